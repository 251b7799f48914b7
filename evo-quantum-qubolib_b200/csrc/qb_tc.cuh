// qb_tc.cuh -- tensor-core (tcgen05) form of the exhaustive search.
//
// The state X splits into three groups of bits:
//   t = X >> 15          (n_T = n - 15 bits; one tile per value, visited in Gray order)
//   y = (X >> 8) & 127   (7 bits: the 128 rows of an MMA tile, one TMEM lane each)
//   u = X & 255          (8 bits: the 256 columns of an MMA tile)
// and the energy as
//   E(t, y, u) = R_t(y) + C_t(u) + y^T V u
//   R_t(y) = energy of the (t, y) variables alone            (per row, per tile)
//   C_t(u) = E_U(u) + (t^T W_TU) u                            (per column, per tile)
//   V      = couplings between the y and u variables          (fixed)
// One tcgen05.mma (kind::f16, M=128, N=256, K=16, fp32 accumulators in TMEM) computes
// D[y][u] = y^T V u + C_t(u) for all 32768 states of a tile:
//   A[y][2i+d] = y_i * s_d         B[u][2i+d] = digit_d((V u)_i)      i < 7, d in {0,1}
//   A[y][14+d] = s_d               B[u][14+d] = digit_d(C_t(u))
// with digits v = d0 + s_1 d1 (integer Q: s = (1, 2048), d0 in [0, 2048), exact in fp16;
// float Q: s = (1, 1), d0 + d1 = fp16 hi/lo split of v).  A is constant; per tile only
// the two C columns of B change.  The epilogue reads each row's 256 accumulators
// (tcgen05.ld), takes the row minimum with 3-input fp32 min, adds R_t(y) and keeps the
// running minimum; every 2^gl tiles each epilogue warp writes one record (32 rows x 128
// columns x 2^gl tiles).
//
// Roles (one persistent CTA per SM, 384 threads):
//   warp 0      tile walk: Gray update of t, per-tile row increment and C tables
//   warp 1      TMEM allocation and MMA issue (one elected thread)
//   warps 2-3   B producers: C_t(u) digits into the B stage (generic stores + proxy fence)
//   warps 4-11  epilogue: warp w reads TMEM lanes 32*(w%4).. and column half (w-4)/4
// Pipelines: 8 tile-parameter slots, 4 B stages, 2 accumulator stages (2 x 256 TMEM
// columns), all on mbarriers.  Every wait is bounded (%globaltimer): on timeout the
// waiting role raises an error flag, the CTA drains and frees TMEM, and the host reports
// QB_ETIMEOUT.
//
// Integer Q with sum|Q| <= 2^22 is exact (all partial sums stay below 2^24 in fp32).
// Otherwise every value is within tc_error_bound() of the exact energy.
#pragma once
#include <cuda_fp16.h>

#include "qb_common.cuh"

namespace qb {

constexpr double kTcIntMaxAbsSum = 4194304.0;  // 2^22
constexpr int kTcThreads = 384;
constexpr int kTcParamSlots = 8;
constexpr int kTcBStages = 4;
constexpr int kTcMaxNT = kMaxN - 15;
constexpr uint64_t kTcWaitLimitNs = 2000000000ull;  // 2 s per wait

struct TcPlan {
  int n = 0, nt = 0, gl = 0;
  bool is_int = false;
  bool exact = false;      // integer digits (exact arithmetic)
  double scale = 1.0;      // power of two applied to W on the device (float digits)
  double eps = 0.0;        // per-state error bound, unscaled units
  uint64_t tile_begin = 0, tile_end = 0;  // this shard's Gray tile indices
  uint64_t rec_begin = 0, rec_count = 0, states = 0;
  int ctas = 0;
};

struct TcParams {
  int n, nt, gl;
  int exact;
  float inv_scale;
  const double* W;          // scaled W, n*n
  uint64_t tile_begin;      // shard start (aligned to 2^gl)
  uint64_t groups;          // record groups in this shard
  uint64_t groups_per_cta;  // contiguous groups per CTA (last CTA may have fewer)
  float* rec;               // rec[0] = record (tile_begin >> gl) << 3
  unsigned* err;            // error word
};

inline bool tc_supported(int n) { return n >= 15 && n <= kMaxN; }

// per-state error bound of the float-digit path (unscaled units)
inline double tc_error_bound(double abs_sum) { return 256.0 * abs_sum * 5.9604644775390625e-08 + 1e-300; }

inline void tc_plan(int n, bool is_int, double abs_sum, int shard_idx, int shard_cnt, TcPlan* p) {
  p->n = n;
  p->nt = n - 15;
  p->is_int = is_int;
  p->exact = is_int && abs_sum <= kTcIntMaxAbsSum;
  if (p->exact) {
    p->scale = 1.0;
    p->eps = 0.0;
  } else {
    // largest power of two with scale * abs_sum <= 2^14 (fp16 digits stay in range)
    int e = 14 - (int)std::ceil(std::log2(std::max(abs_sum, 1e-30)));
    e = std::max(-60, std::min(60, e));
    p->scale = std::ldexp(1.0, e);
    p->eps = tc_error_bound(abs_sum);
  }
  p->gl = std::max(0, std::min(p->nt, n - 15 - 19));  // at most 2^22 records
  uint64_t groups = 1ull << (p->nt - p->gl);
  unsigned __int128 g = groups;
  uint64_t gb = (uint64_t)(g * (unsigned)shard_idx / (unsigned)shard_cnt);
  uint64_t ge = (uint64_t)(g * (unsigned)(shard_idx + 1) / (unsigned)shard_cnt);
  p->tile_begin = gb << p->gl;
  p->tile_end = ge << p->gl;
  p->rec_begin = gb << 3;
  p->rec_count = (ge - gb) << 3;
  p->states = (p->tile_end - p->tile_begin) << 15;
}

// scratch: error word (16 B) + scaled W
inline size_t tc_scratch_bytes(const TcPlan& p) { return 16 + (size_t)p.n * p.n * sizeof(double); }

#ifdef __CUDACC__
// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false on timeout (or when another role already gave up)
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try_wait(b, parity)) return true;
    if ((it & 63) == 63) {
      if (*abort_flag) return false;
      if (globaltimer_ns() - t0 > kTcWaitLimitNs) return false;
    }
  }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// K-major, no-swizzle shared-memory matrix descriptor: core matrices of 8 rows x 16 bytes,
// LBO = distance between K-adjacent core matrices, SBO = between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version for tcgen05
  return d;         // base offset 0, relative LBO, no swizzle
}

// instruction descriptor, kind::f16: A = B = f16, D = f32, both K-major, M = 128, N = 256
constexpr uint32_t kTcIdesc = (1u << 4) | (0u << 7) | (0u << 10) | ((256u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(0)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

#define QB_TC_LD32(taddr, r)                                                                                      \
  asm volatile(                                                                                                   \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18," \
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                                               \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),           \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),     \
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),   \
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])    \
      : "r"(taddr))

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float min32(const uint32_t* r) {
  float m0 = fmin3(__uint_as_float(r[0]), __uint_as_float(r[1]), __uint_as_float(r[2]));
  float m1 = fmin3(__uint_as_float(r[3]), __uint_as_float(r[4]), __uint_as_float(r[5]));
  float m2 = fmin3(__uint_as_float(r[6]), __uint_as_float(r[7]), __uint_as_float(r[8]));
  float m3 = fmin3(__uint_as_float(r[9]), __uint_as_float(r[10]), __uint_as_float(r[11]));
  float m4 = fmin3(__uint_as_float(r[12]), __uint_as_float(r[13]), __uint_as_float(r[14]));
  float m5 = fmin3(__uint_as_float(r[15]), __uint_as_float(r[16]), __uint_as_float(r[17]));
  float m6 = fmin3(__uint_as_float(r[18]), __uint_as_float(r[19]), __uint_as_float(r[20]));
  float m7 = fmin3(__uint_as_float(r[21]), __uint_as_float(r[22]), __uint_as_float(r[23]));
  float m8 = fmin3(__uint_as_float(r[24]), __uint_as_float(r[25]), __uint_as_float(r[26]));
  float m9 = fmin3(__uint_as_float(r[27]), __uint_as_float(r[28]), __uint_as_float(r[29]));
  float n0 = fmin3(m0, m1, m2);
  float n1 = fmin3(m3, m4, m5);
  float n2 = fmin3(m6, m7, m8);
  float n3 = fmin3(m9, __uint_as_float(r[30]), __uint_as_float(r[31]));
  return fmin3(n0, n1, fminf(n2, n3));
}

// offset of element (row, k) of a 16-column f16 operand in the K-major no-swizzle layout
__device__ __forceinline__ uint32_t kmaj_off(uint32_t row, uint32_t k) {
  return (row >> 3) * 256u + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// split v into two fp16 digits
__device__ __forceinline__ __half2 digits(float v, int exact) {
  if (exact) {
    float d1 = floorf(v * (1.0f / 2048.0f));
    float d0 = v - 2048.0f * d1;
    return __halves2half2(__float2half_rn(d0), __float2half_rn(d1));
  }
  __half hi = __float2half_rn(v);
  __half lo = __float2half_rn(v - __half2float(hi));
  return __halves2half2(lo, hi);
}

struct TcSlot {
  float F[32];  // F[0..15]: C contribution of the low 4 u bits, F[16..31]: high 4 bits
  double d;     // W_kk + field of the flipped tile variable before the flip
  int k;        // flipped tile bit (-1: none)
  float sgn;    // +1 when the bit turns on
};

struct TcSmemLayout {
  uint32_t a_off, b_off, bar_off, slot_off, eu_off, misc_off, hy_off, w_off, total;
};

__host__ __device__ inline TcSmemLayout tc_layout(int n) {
  TcSmemLayout L;
  uint32_t o = 0;
  L.a_off = o;
  o += 128 * 32;  // A: 128 rows x 16 f16
  L.b_off = o;
  o += kTcBStages * 256 * 32;
  L.bar_off = o;
  o += (2 * kTcParamSlots + 2 * kTcBStages + 4) * 8;
  L.slot_off = o;
  o += kTcParamSlots * sizeof(TcSlot);
  L.eu_off = o;
  o += 256 * 4;
  L.misc_off = o;
  o += 64;
  L.hy_off = o;
  o += (uint32_t)(n - 15) * 128 * 8;
  L.w_off = o;
  o += (uint32_t)n * n * 8;
  L.total = o;
  return L;
}

__global__ void __launch_bounds__(kTcThreads, 1) tc_pass1_kernel(TcParams P) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int n = P.n, nt = P.nt;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const TcSmemLayout L = tc_layout(n);
  unsigned char* Asm = sm + L.a_off;
  unsigned char* Bsm = sm + L.b_off;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + L.bar_off);
  uint64_t* p_full = bars;
  uint64_t* p_empty = p_full + kTcParamSlots;
  uint64_t* b_full = p_empty + kTcParamSlots;
  uint64_t* b_empty = b_full + kTcBStages;
  uint64_t* acc_full = b_empty + kTcBStages;
  uint64_t* acc_empty = acc_full + 2;
  TcSlot* slots = reinterpret_cast<TcSlot*>(sm + L.slot_off);
  float* EU = reinterpret_cast<float*>(sm + L.eu_off);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L.misc_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L.misc_off + 4);
  double* ET0 = reinterpret_cast<double*>(sm + L.misc_off + 8);
  double* hY = reinterpret_cast<double*>(sm + L.hy_off);
  double* Ws = reinterpret_cast<double*>(sm + L.w_off);

  // this CTA's record groups and tiles (Gray indices)
  const uint64_t g0 = (uint64_t)blockIdx.x * P.groups_per_cta;
  if (g0 >= P.groups) return;  // uniform per CTA
  const uint64_t g1 = min(P.groups, g0 + P.groups_per_cta);
  const uint64_t i_begin = P.tile_begin + (g0 << P.gl);
  const uint64_t ntiles = (g1 - g0) << P.gl;
  const uint64_t t0 = gray64(i_begin);
  const float s1 = P.exact ? 2048.0f : 1.0f;

  // ---------------------------------------------------------------- set-up
  for (int i = tid; i < n * n; i += kTcThreads) Ws[i] = P.W[i];
  if (tid == 0) {
    for (int s = 0; s < kTcParamSlots; ++s) {
      mbar_init(&p_full[s], 1);
      mbar_init(&p_empty[s], 10);  // 2 producer warps + 8 epilogue warps
    }
    for (int s = 0; s < kTcBStages; ++s) {
      mbar_init(&b_full[s], 2);
      mbar_init(&b_empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], 8);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  // variables: t bit k <-> n-16-k, y bit i <-> n-9-i, u bit j <-> n-1-j
  // A operand (constant)
  for (int e = tid; e < 128 * 16; e += kTcThreads) {
    int y = e >> 4, k = e & 15;
    float v;
    if (k < 14)
      v = ((y >> (k >> 1)) & 1) ? ((k & 1) ? s1 : 1.0f) : 0.0f;
    else
      v = (k & 1) ? s1 : 1.0f;
    *reinterpret_cast<__half*>(Asm + kmaj_off(y, k)) = __float2half_rn(v);
  }
  // B operand, coupling columns (same in every stage)
  for (int e = tid; e < 256 * 7; e += kTcThreads) {
    int u = e / 7, i = e % 7;
    const double* row = Ws + (n - 9 - i) * n;
    double v = 0.0;
    for (int j = 0; j < 8; ++j)
      if ((u >> j) & 1) v += row[n - 1 - j];
    __half2 dg = digits((float)v, P.exact);
    for (int s = 0; s < kTcBStages; ++s)
      *reinterpret_cast<__half2*>(Bsm + s * 256 * 32 + kmaj_off(u, 2 * i)) = dg;
  }
  // E_U(u)
  for (int u = tid; u < 256; u += kTcThreads) {
    double e = 0.0;
    for (int j = 0; j < 8; ++j) {
      if (!((u >> j) & 1)) continue;
      const double* row = Ws + (n - 1 - j) * n;
      e += row[n - 1 - j];
      for (int j2 = 0; j2 < j; ++j2)
        if ((u >> j2) & 1) e += row[n - 1 - j2];
    }
    EU[u] = (float)e;
  }
  // hY[k][y] = sum_i y_i W(t var k, y var i)
  for (int e = tid; e < nt * 128; e += kTcThreads) {
    int k = e >> 7, y = e & 127;
    const double* row = Ws + (n - 16 - k) * n;
    double v = 0.0;
    for (int i = 0; i < 7; ++i)
      if ((y >> i) & 1) v += row[n - 9 - i];
    hY[e] = v;
  }
  if (tid == 0) {  // E_T(t0)
    double e = 0.0;
    for (int k = 0; k < nt; ++k) {
      if (!((t0 >> k) & 1)) continue;
      const double* row = Ws + (n - 16 - k) * n;
      e += row[n - 16 - k];
      for (int k2 = 0; k2 < k; ++k2)
        if ((t0 >> k2) & 1) e += row[n - 16 - k2];
    }
    *ET0 = e;
  }
  fence_proxy_async();  // A / B stores (generic proxy) -> visible to tcgen05.mma
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  bool ok = true;
  if (warp == 0) {
    // ---------------------------------------------------------- tile walk
    double h0 = 0.0, h1 = 0.0, f = 0.0;  // fields of t bits lane, lane+32; f_lane (lane < 8)
    const int m0 = lane, m1 = lane + 32;
    for (int k = 0; k < nt; ++k) {
      if (!((t0 >> k) & 1)) continue;
      const double* row = Ws + (n - 16 - k) * n;
      if (m0 < nt && m0 != k) h0 += row[n - 16 - m0];
      if (m1 < nt && m1 != k) h1 += row[n - 16 - m1];
      if (lane < 8) f += row[n - 1 - lane];
    }
    for (uint64_t j = 0; j < ntiles && ok; ++j) {
      const int s = (int)(j % kTcParamSlots);
      const uint32_t ph = (uint32_t)((j / kTcParamSlots) & 1);
      ok = mbar_wait(&p_empty[s], ph ^ 1u, abort_flag);
      if (!ok) break;
      TcSlot& sl = slots[s];
      if (j == 0) {
        if (lane == 0) {
          sl.k = -1;
          sl.sgn = 0.f;
          sl.d = 0.0;
        }
      } else {
        const uint64_t i = i_begin + j;
        const int kb = __ffsll((long long)i) - 1;
        const bool on = (gray64(i) >> kb) & 1;
        const double sg = on ? 1.0 : -1.0;
        const double hk = __shfl_sync(0xffffffffu, kb < 32 ? h0 : h1, kb & 31);
        const double* row = Ws + (n - 16 - kb) * n;
        if (lane == 0) {
          sl.k = kb;
          sl.sgn = (float)sg;
          sl.d = row[n - 16 - kb] + hk;
        }
        if (m0 < nt && m0 != kb) h0 += sg * row[n - 16 - m0];
        if (m1 < nt && m1 != kb) h1 += sg * row[n - 16 - m1];
        if (lane < 8) f += sg * row[n - 1 - lane];
      }
      // C tables: F[l] (l < 16) = sum of f_j over bits j of l; F[16 + l] over bits j+4
      double acc = 0.0;
      const int base = lane < 16 ? 0 : 4;
      for (int jb = 0; jb < 4; ++jb) {
        double fj = __shfl_sync(0xffffffffu, f, base + jb);
        if (((lane & 15) >> jb) & 1) acc += fj;
      }
      sl.F[lane] = (float)acc;
      __syncwarp();
      if (lane == 0) mbar_arrive(&p_full[s]);
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issue
    if (lane == 0) {
      const uint64_t adesc = umma_desc(smem_u32(Asm), 128, 256);
      uint64_t issued = 0;
      for (uint64_t j = 0; j < ntiles && ok; ++j) {
        const int bs = (int)(j % kTcBStages);
        const int as = (int)(j & 1);
        ok = mbar_wait(&b_full[bs], (uint32_t)((j / kTcBStages) & 1), abort_flag) &&
             mbar_wait(&acc_empty[as], (uint32_t)(((j >> 1) & 1) ^ 1), abort_flag);
        if (!ok) break;
        tc_fence_after();
        const uint64_t bdesc = umma_desc(smem_u32(Bsm + bs * 256 * 32), 128, 256);
        tc_mma(tmem + (uint32_t)as * 256u, adesc, bdesc);
        tc_commit(&b_empty[bs]);
        tc_commit(&acc_full[as]);
        issued = j + 1;
      }
      if (issued) {  // let the last MMA finish before the CTA can release TMEM
        const uint64_t j = issued - 1;
        mbar_wait(&b_empty[j % kTcBStages], (uint32_t)((j / kTcBStages) & 1), abort_flag);
      }
    }
    __syncwarp();
  } else if (warp < 4) {
    // ---------------------------------------------------------- B producers (C_t columns)
    const int pt = tid - 64;  // 0..63
    for (uint64_t j = 0; j < ntiles && ok; ++j) {
      const int s = (int)(j % kTcParamSlots);
      const int bs = (int)(j % kTcBStages);
      ok = mbar_wait(&p_full[s], (uint32_t)((j / kTcParamSlots) & 1), abort_flag);
      float c[4];
      if (ok) {
        const TcSlot& sl = slots[s];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int u = pt + 64 * r;
          c[r] = EU[u] + sl.F[u & 15] + sl.F[16 + (u >> 4)];
        }
        ok = mbar_wait(&b_empty[bs], (uint32_t)(((j / kTcBStages) & 1) ^ 1), abort_flag);
      }
      if (!ok) break;
      unsigned char* Bst = Bsm + bs * 256 * 32;
#pragma unroll
      for (int r = 0; r < 4; ++r)
        *reinterpret_cast<__half2*>(Bst + kmaj_off(pt + 64 * r, 14)) = digits(c[r], P.exact);
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&b_full[bs]);
        mbar_arrive(&p_empty[s]);
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int ew = warp - 4;  // 0..7
    const int q = warp & 3;   // TMEM lane quarter (warp id % 4)
    const int half = ew >> 2; // column half
    const int y = q * 32 + lane;
    double R = *ET0;
    {
      const double* yr = Ws + (n - 9) * n;  // placeholder row pointer (unused when y == 0)
      (void)yr;
      for (int i = 0; i < 7; ++i) {
        if (!((y >> i) & 1)) continue;
        const double* row = Ws + (n - 9 - i) * n;
        R += row[n - 9 - i];
        for (int i2 = 0; i2 < i; ++i2)
          if ((y >> i2) & 1) R += row[n - 9 - i2];
      }
      for (int k = 0; k < nt; ++k)
        if ((t0 >> k) & 1) R += hY[k * 128 + y];
    }
    const float inv = P.inv_scale;
    const float inf = __int_as_float(0x7f800000);
    float rmin = inf;
    const uint64_t gmask = (1ull << P.gl) - 1ull;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    for (uint64_t j = 0; j < ntiles && ok; ++j) {
      const int s = (int)(j % kTcParamSlots);
      const int as = (int)(j & 1);
      ok = mbar_wait(&p_full[s], (uint32_t)((j / kTcParamSlots) & 1), abort_flag);
      if (!ok) break;
      {
        const TcSlot& sl = slots[s];
        if (sl.k >= 0) R += (double)sl.sgn * (sl.d + hY[sl.k * 128 + y]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&p_empty[s]);
      ok = mbar_wait(&acc_full[as], (uint32_t)((j >> 1) & 1), abort_flag);
      if (!ok) break;
      tc_fence_after();
      const uint32_t ta = tmem + lane_base + (uint32_t)as * 256u + (uint32_t)half * 128u;
      uint32_t ra[32], rb[32];
      QB_TC_LD32(ta, ra);
      QB_TC_LD32(ta + 32, rb);
      tc_wait_ld();
      float m = fminf(min32(ra), min32(rb));
      QB_TC_LD32(ta + 64, ra);
      QB_TC_LD32(ta + 96, rb);
      tc_wait_ld();
      m = fmin3(m, min32(ra), min32(rb));
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[as]);
      rmin = fminf(rmin, m + (float)R);
      const uint64_t i = i_begin + j;
      if ((i & gmask) == gmask) {
        const float wm = warp_min_f(rmin);
        if (lane == 0) {
          const uint64_t J = (i >> P.gl) - (P.tile_begin >> P.gl);
          P.rec[(J << 3) | ((uint64_t)half << 2) | (uint64_t)q] = wm * inv;
        }
        rmin = inf;
      }
    }
  }
  if (!ok) {
    *abort_flag = 1;
    atomicOr(P.err, kErrTimeout);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
  }
}

// scale W into the scratch buffer (float digits keep magnitudes inside the fp16 range)
__global__ void tc_scale_w_kernel(const double* __restrict__ W, double* __restrict__ out, int nn, double scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) out[i] = W[i] * scale;
}

inline int tc_launch(const TcPlan& p, ProblemDev pd, float* rec, void* scratch, cudaStream_t st, int sms,
                     int* kernels) {
  unsigned* err = static_cast<unsigned*>(scratch);
  double* Wsc = reinterpret_cast<double*>(static_cast<char*>(scratch) + 16);
  if (cudaMemsetAsync(err, 0, 16, st) != cudaSuccess) return 4;
  tc_scale_w_kernel<<<8, 256, 0, st>>>(pd.W, Wsc, p.n * p.n, p.scale);
  ++*kernels;
  const uint64_t groups = (p.tile_end - p.tile_begin) >> p.gl;
  if (!groups) return cudaGetLastError() == cudaSuccess ? 0 : 4;
  uint64_t ctas = std::min<uint64_t>((uint64_t)sms, groups);
  uint64_t gpc = (groups + ctas - 1) / ctas;
  ctas = (groups + gpc - 1) / gpc;
  TcParams P{};
  P.n = p.n;
  P.nt = p.nt;
  P.gl = p.gl;
  P.exact = p.exact ? 1 : 0;
  P.inv_scale = (float)(1.0 / p.scale);
  P.W = Wsc;
  P.tile_begin = p.tile_begin;
  P.groups = groups;
  P.groups_per_cta = gpc;
  P.rec = rec;
  P.err = err;
  const TcSmemLayout L = tc_layout(p.n);
  // at least 120 KB so that one CTA (and one 512-column TMEM allocation) runs per SM
  const size_t smem = std::max<size_t>(L.total, 120 * 1024) + 1024;
  if (cudaFuncSetAttribute(tc_pass1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 4;
  tc_pass1_kernel<<<(unsigned)ctas, kTcThreads, smem, st>>>(P);
  ++*kernels;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

inline int tc_check_error(void* scratch, cudaStream_t st) {
  unsigned e = 0;
  if (cudaMemcpyAsync(&e, scratch, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess) return 4;
  if (cudaStreamSynchronize(st) != cudaSuccess) return 4;
  return (e & kErrTimeout) ? 5 : 0;
}
#endif

}  // namespace qb
