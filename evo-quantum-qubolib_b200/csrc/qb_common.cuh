// qb_common.cuh -- shared device types and helpers of the exhaustive QUBO kernels.
//
// State encoding: X = MSB-first integer of the state, variable i <-> bit (n-1-i).
// Problem data on the device: W (n x n doubles, row-major) with W[i][j] = Q_ij + Q_ji for
// i != j and W[i][i] = Q_ii, so that E(x) = sum_i W_ii x_i + sum_{i<j} W_ij x_i x_j.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qb {

constexpr int kMaxN = 62;

// error flags raised by kernels (bitwise or-ed into a device word)
constexpr unsigned kErrTimeout = 1u;
constexpr unsigned kErrBadArg = 2u;
constexpr unsigned kErrCandOverflow = 4u;

struct ProblemDev {
  int n;
  const double* W;  // n*n
};

// tie rules (values match QB_TIE_* in include/qubo_b200.h)
constexpr int kTieQBF = 0;
constexpr int kTieQBF1 = 1;
constexpr int kTieNatural = 2;

struct TieRule {
  int kind;
  int n;
  int k;  // QBF: leading natural-order task bits
  int A;  // QBF: inverse-Gray ranked prefix bits; QB_F1: prefix bits (n - k - 18)
  int B;  // QBF: trailing natural-order bits
};

// record geometry: which states a pass-1 record covers
constexpr int kGeomGray = 1;
constexpr int kGeomTC = 2;
constexpr int kGeomBlock = 3;  // plain blocks of 2^f consecutive X (exact form)

struct RecGeom {
  int kind;
  int n;
  int a, b;       // Gray form split (b >= 13)
  int sbits;      // Gray form: log2 prefix steps per record
  int cbbits;     // Gray form: log2 column blocks (b - 13)
  int gubits;     // Gray form: log2 record groups per work unit
  int gl;         // TC form: log2 tiles per record
  int fbits;      // block geometry: log2 states per record
};

__host__ __device__ __forceinline__ uint64_t mask64(int b) {
  return b >= 64 ? ~0ull : ((1ull << b) - 1ull);
}

__host__ __device__ __forceinline__ uint64_t gray64(uint64_t i) { return i ^ (i >> 1); }

// inverse Gray code: i with gray64(i) == g
__host__ __device__ __forceinline__ uint64_t grayrank64(uint64_t g) {
  g ^= g >> 1;
  g ^= g >> 2;
  g ^= g >> 4;
  g ^= g >> 8;
  g ^= g >> 16;
  g ^= g >> 32;
  return g;
}

__host__ __device__ __forceinline__ uint64_t tie_key(const TieRule& r, uint64_t X) {
  switch (r.kind) {
    case kTieQBF: {
      uint64_t task = r.k ? (X >> (r.A + r.B)) : 0ull;
      uint64_t mid = (X >> r.B) & mask64(r.A);
      uint64_t low = X & mask64(r.B);
      return (task << (r.A + r.B)) | (grayrank64(mid) << r.B) | low;
    }
    case kTieQBF1: {
      // k task bits (natural order), then QB_F1's thread id of the 18-bit suffix
      // (256 x 64 grid, 16 columns per thread: tid = (s >> 10) * 64 + (s & 63)), then the
      // Gray step of the A-bit prefix
      uint64_t task = r.k ? (X >> (r.A + 18)) : 0ull;
      uint64_t s = X & mask64(18);
      uint64_t p = (X >> 18) & mask64(r.A);
      uint64_t tid = ((s >> 10) << 6) | (s & 63ull);
      return (task << (14 + r.A)) | (tid << r.A) | grayrank64(p);
    }
    default:
      return X;
  }
}

// record index -> (base state, free-bit mask)
__host__ __device__ __forceinline__ void record_states(const RecGeom& g, uint64_t r, uint64_t* base,
                                                       uint64_t* freem) {
  if (g.kind == kGeomGray) {
    // r = (unit << (gubits + 3)) | (group << 3) | warp, unit = (chunk << cbbits) | cb
    uint64_t w = r & 7ull;
    uint64_t rest = r >> 3;
    uint64_t gi = rest & mask64(g.gubits);
    uint64_t unit = rest >> g.gubits;
    uint64_t cb = unit & mask64(g.cbbits);
    uint64_t I = ((unit >> g.cbbits) << g.gubits) | gi;
    *base = (gray64(I) << (g.sbits + g.b)) | (cb << 13) | (w << 10);
    *freem = (mask64(g.sbits) << g.b) | mask64(10);
  } else if (g.kind == kGeomTC) {
    // r = (block << 3) | (column half h << 2) | TMEM lane quarter q: the Gray tiles of
    // block J (t >> gl = gray(J), low gl bits of t free), rows 32q..32q+31 (y's top 2
    // bits = q), columns 128h..128h+127 (u's top bit = h)
    uint64_t q = r & 3ull;
    uint64_t h = (r >> 2) & 1ull;
    uint64_t J = r >> 3;
    *base = (gray64(J) << (15 + g.gl)) | (q << 13) | (h << 7);
    *freem = (mask64(g.gl) << 15) | (mask64(5) << 8) | mask64(7);
  } else {
    *base = r << g.fbits;
    *freem = mask64(g.fbits);
  }
}

// order-preserving map float -> uint32 (for integer min reductions)
__host__ __device__ __forceinline__ uint32_t f2key(float f) {
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f);
#else
  union { float f; uint32_t u; } c; c.f = f; u = c.u;
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float key2f(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  union { float f; uint32_t u; } c; c.u = u; return c.f;
#endif
}

// trailing zeros of 1 <= l < 32 (folds to a constant for an unrolled l): the prefix bit
// flipped by step l of an aligned group of 32 Gray steps
__host__ __device__ constexpr int ctz5(int l) { return (l & 1) ? 0 : (l & 2) ? 1 : (l & 4) ? 2 : (l & 8) ? 3 : 4; }

#ifdef __CUDACC__
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ float fmin3(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  uint64_t ra = *reinterpret_cast<uint64_t*>(&a);
  uint64_t rb = *reinterpret_cast<uint64_t*>(&b);
  uint64_t rc;
  asm("add.f32x2 %0, %1, %2;" : "=l"(rc) : "l"(ra), "l"(rb));
  return *reinterpret_cast<float2*>(&rc);
}

__device__ __forceinline__ float warp_min_f(float v) {
  uint32_t k = f2key(v);
  k = __reduce_min_sync(0xffffffffu, k);
  return key2f(k);
}
#endif

}  // namespace qb
