// qb_gray.cuh -- plain Gray-code form of the exhaustive search (SIMT, fp32 arithmetic).
//
// Split the state into a prefix p (variables 0..a-1, the top a bits of X) and a suffix s
// (the low b bits).  Following the reference's method (src/qubo_lib/solvers/qbf.py:188-230),
// prefixes are visited in Gray order, step i having p = i ^ (i >> 1), and every suffix
// keeps its running energy.  On B200 each thread owns 32 suffixes s = (s_hi << 5) | c and
// splits their energy as
//     E(p, s) = A_t(p) + e_t[c] + G(p)[c]
//   e_t[c]  = E_suf(s)                              (32 registers, fixed per thread)
//   A_t(p)  = sum_{k in p} alpha_k(s_hi)            (cross term with the thread's high
//                                                    suffix bits; one update per Gray step)
//   G(p)[c] = E_pre(p) + sum_{k in p} beta_k[c]     (cross term with the 5 low suffix bits,
//                                                    shared by every thread; a table)
// so a Gray step costs each thread one scalar update, 16 packed adds (add.f32x2) and a
// 3-input-min tree over its 32 energies.  A CTA holds 256 threads x 32 suffixes = 2^13
// consecutive suffixes ("column block"); a unit of work is (column block, run of prefix
// steps).  Every aligned group of 2^sbits steps, each warp writes the minimum over its
// 1024 suffixes x 2^sbits prefixes as one record (record_states, kGeomGray).
//
// Arithmetic is fp32.  Integer Q with sum|Q| < 2^24 is exact; otherwise every value is
// within gray_error_bound() of the exact energy and pass 2 re-evaluates in FP64.
#pragma once
#include "qb_common.cuh"

namespace qb {

constexpr int kGrayThreads = 256;
constexpr int kGrayStage = 128;  // G-table rows staged in shared memory per buffer

struct GrayParams {
  ProblemDev P;
  int a, b;           // prefix / suffix bits (b >= 13, 5 <= a <= 24)
  int cbbits;         // b - 13
  int sbits;          // log2 prefix steps per record (>= 5)
  int gubits;         // log2 record groups per unit; steps per unit = 2^(gubits + sbits) >= 128
  uint64_t unit_begin;
  const float* gtab;  // [2^a][32]
  float* rec;         // record minima; rec[0] holds record (unit_begin << (gubits + 3))
};

// per-state error bound of the fp32 path (see the header comment)
inline double gray_error_bound(double abs_sum) { return 300.0 * abs_sum * 5.9604644775390625e-08; }

// G(p)[c] for the Gray steps i in [lo, hi), lane = c.  The CTA's warps take contiguous
// sub-ranges and walk them in Gray order: at the first step of a sub-range a warp computes
// E_pre(p), the prefix fields h_l = sum_{m in p, m != l} W_lm (lane l < a) and
// sum_{k in p} beta_k[c] from scratch in FP64, then each step flips one prefix variable k:
//   E_pre += s (W_kk + h_k),  sum beta += s beta_k[c],  h_l += s W_lk (l != k)
// (s = +1 when k turns on).  smem: gray_gtab_smem(n, a).
__device__ __forceinline__ void gray_gtab_body(const ProblemDev& P, int a, float* __restrict__ gtab, uint64_t lo,
                                               uint64_t hi, double* gtab_smem) {
  const int n = P.n;
  double* Ws = gtab_smem;      // n*n
  double* beta = Ws + n * n;   // a * 32
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) Ws[i] = P.W[i];
  __syncthreads();
  for (int i = threadIdx.x; i < a * 32; i += blockDim.x) {
    int k = i >> 5, c = i & 31;
    double s = 0.0;
    for (int j = 0; j < 5; ++j)
      if ((c >> j) & 1) s += Ws[k * n + (n - 1 - j)];
    beta[i] = s;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint64_t len = (hi - lo + nw - 1) / nw;
  const uint64_t w0 = lo + (uint64_t)warp * len;
  const uint64_t w1 = min(hi, w0 + len);
  if (w0 >= w1) return;  // uniform per warp
  const uint64_t p0 = gray64(w0);
  double h = 0.0, ep = 0.0, bs = 0.0;
  if (lane < a) {
    const double* row = Ws + lane * n;
    for (int m = 0; m < a; ++m)
      if (m != lane && ((p0 >> (a - 1 - m)) & 1)) h += row[m];
    if ((p0 >> (a - 1 - lane)) & 1) ep = row[lane] + 0.5 * h;  // E_pre = sum_k in p (W_kk + h_k / 2)
  }
  for (int off = 16; off; off >>= 1) ep += __shfl_xor_sync(0xffffffffu, ep, off);
  for (int k = 0; k < a; ++k)
    if ((p0 >> (a - 1 - k)) & 1) bs += beta[k * 32 + lane];
  gtab[w0 * 32 + lane] = (float)(ep + bs);
  for (uint64_t i = w0 + 1; i < w1; ++i) {
    const int kb = __ffsll((long long)i) - 1;
    const int k = a - 1 - kb;
    const double sg = ((gray64(i) >> kb) & 1) ? 1.0 : -1.0;
    const double hk = __shfl_sync(0xffffffffu, h, k);
    ep += sg * (Ws[k * n + k] + hk);
    bs += sg * beta[k * 32 + lane];
    if (lane < a && lane != k) h += sg * Ws[lane * n + k];
    gtab[i * 32 + lane] = (float)(ep + bs);
  }
}

__global__ void gray_gtab_kernel(ProblemDev P, int a, int b, float* __restrict__ gtab) {
  extern __shared__ double gtab_smem[];
  (void)b;
  const uint64_t steps = 1ull << a;
  const uint64_t per = (steps + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = (uint64_t)blockIdx.x * per;
  gray_gtab_body(P, a, gtab, min(lo, steps), min(lo + per, steps), gtab_smem);
}

inline size_t gray_gtab_smem(int n, int a) { return (size_t)(n * n + a * 32) * sizeof(double); }

// shared-memory carve-out, in this order so that the float4-read staging buffer sits at
// offset 0 (16-byte aligned) and every double array at a multiple of 8 bytes
inline size_t gray_pass1_smem(int n, int a) {
  return 2 * kGrayStage * 32 * sizeof(float)          // staged G rows
         + 32 * sizeof(double)                        // E_lo
         + (size_t)a * kGrayThreads * sizeof(double)  // alpha (fp64, resync)
         + (size_t)n * n * sizeof(double)              // W
         + (size_t)a * kGrayThreads * sizeof(float);  // alpha (fp32, per step)
}

// One CTA searches work unit g.unit_begin + unit_local and writes its records.
__device__ __forceinline__ void gray_unit_body(const GrayParams& g, uint64_t unit_local, unsigned char* smem_raw) {
  const int n = g.P.n, a = g.a, b = g.b;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  float* gbuf = reinterpret_cast<float*>(smem_raw);
  double* Elo = reinterpret_cast<double*>(gbuf + 2 * kGrayStage * 32);
  double* alpha_d = Elo + 32;
  double* Ws = alpha_d + a * kGrayThreads;
  float* alpha_f = reinterpret_cast<float*>(Ws + n * n);

  const uint64_t unit = g.unit_begin + unit_local;
  const uint64_t cb = unit & mask64(g.cbbits);
  const uint64_t chunk = unit >> g.cbbits;
  const int ubits = g.gubits + g.sbits;
  const uint32_t i0 = (uint32_t)(chunk << ubits);
  const uint32_t S = 1u << ubits;

  for (int i = t; i < n * n; i += kGrayThreads) Ws[i] = g.P.W[i];
  __syncthreads();
  if (t < 32) {  // energy of the 5 low suffix variables for pattern c = t
    double e = 0.0;
    for (int j = 0; j < 5; ++j) {
      if (!((t >> j) & 1)) continue;
      int v = n - 1 - j;
      e += Ws[v * n + v];
      for (int j2 = 0; j2 < j; ++j2)
        if ((t >> j2) & 1) e += Ws[v * n + (n - 1 - j2)];
    }
    Elo[t] = e;
  }
  // thread's high suffix bits: s = (shi << 5) | c, s-bit m <-> variable n-1-m
  const uint64_t shi = (cb << 8) | (uint64_t)t;
  double ehi = 0.0, w5[5] = {0, 0, 0, 0, 0};
  for (int m = 5; m < b; ++m) {
    if (!((shi >> (m - 5)) & 1)) continue;
    int v = n - 1 - m;
    const double* row = Ws + v * n;
    ehi += row[v];
    for (int m2 = 5; m2 < m; ++m2)
      if ((shi >> (m2 - 5)) & 1) ehi += row[n - 1 - m2];
    for (int j = 0; j < 5; ++j) w5[j] += row[n - 1 - j];
  }
  for (int k = 0; k < a; ++k) {
    double s = 0.0;
    const double* row = Ws + k * n;
    for (int m = 5; m < b; ++m)
      if ((shi >> (m - 5)) & 1) s += row[n - 1 - m];
    alpha_d[k * kGrayThreads + t] = s;
    alpha_f[k * kGrayThreads + t] = (float)s;
  }
  __syncthreads();
  float alo[5];  // fp32 cross terms of the 5 low prefix bits (variables a-1-k), fixed per thread
#pragma unroll
  for (int k = 0; k < 5; ++k) alo[k] = alpha_f[(a - 1 - k) * kGrayThreads + t];
  float2 e2[16];
#pragma unroll
  for (int c2 = 0; c2 < 16; ++c2) {
    double v0 = ehi + Elo[2 * c2], v1 = ehi + Elo[2 * c2 + 1];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      if (((2 * c2) >> j) & 1) v0 += w5[j];
      if (((2 * c2 + 1) >> j) & 1) v1 += w5[j];
    }
    e2[c2] = make_float2((float)v0, (float)v1);
  }

  // stage the first block of G rows
  const float4* gsrc = reinterpret_cast<const float4*>(g.gtab + (size_t)i0 * 32);
  float4* gdst = reinterpret_cast<float4*>(gbuf);
#pragma unroll
  for (int q = 0; q < 4; ++q) gdst[t + q * kGrayThreads] = gsrc[t + q * kGrayThreads];
  __syncthreads();

  const float inf = __int_as_float(0x7f800000);
  float rmin = inf;
  const uint32_t rmask = (1u << g.sbits) - 1u;
  const uint64_t rec_unit_base = ((unit - g.unit_begin) << (g.gubits + 3));
  const uint32_t nblk = S / kGrayStage;
  for (uint32_t blk = 0; blk < nblk; ++blk) {
    const uint32_t ib = i0 + blk * kGrayStage;
    // exact prefix cross term at the block start (fp64), then fp32 steps
    float A;
    {
      const uint32_t p = ib ^ (ib >> 1);
      double ad = 0.0;
      for (int k = 0; k < a; ++k)
        if ((p >> (a - 1 - k)) & 1) ad += alpha_d[k * kGrayThreads + t];
      A = (float)ad;
    }
    float4 nxt[4];
    const bool more = blk + 1 < nblk;
    if (more) {
      const float4* src = reinterpret_cast<const float4*>(g.gtab + (size_t)(ib + kGrayStage) * 32);
#pragma unroll
      for (int q = 0; q < 4; ++q) nxt[q] = src[t + q * kGrayThreads];
    }
    const float* cur = gbuf + (blk & 1) * kGrayStage * 32;
    // 4 aligned groups of 32 steps.  Inside a group the flipped prefix bit of step l > 0 is
    // kb = ctz(l) and its new state is !bit(kb + 1) of the step index: both constants of
    // the unrolled step for kb < 4; for kb = 4 bit 5 is the group's parity (the block
    // starts at a multiple of 128).  A group's first step flips a bit >= 5 (general code).
    for (int grp = 0; grp < kGrayStage / 32; ++grp) {
      const uint32_t ig = ib + (uint32_t)grp * 32u;
      if (grp) {
        const int kb = __ffs(ig) - 1;
        const int var = a - 1 - kb;
        const float al = alpha_f[var * kGrayThreads + t];
        A = ((ig ^ (ig >> 1)) >> kb) & 1 ? A + al : A - al;
      }
      const float a4 = (grp & 1) ? -alo[4] : alo[4];
      const float* crow = cur + grp * 32 * 32;
#pragma unroll
      for (int l = 0; l < 32; ++l) {
        if (l) {
          const int kb = ctz5(l);
          if (kb < 4)
            A = ((l >> (kb + 1)) & 1) ? A - alo[kb] : A + alo[kb];
          else
            A += a4;
        }
        const float4* row = reinterpret_cast<const float4*>(crow + l * 32);
        float2 v[16];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          float4 gg = row[q];
          v[2 * q] = fadd2(e2[2 * q], make_float2(gg.x, gg.y));
          v[2 * q + 1] = fadd2(e2[2 * q + 1], make_float2(gg.z, gg.w));
        }
        float m0 = fmin3(v[0].x, v[0].y, v[1].x);
        float m1 = fmin3(v[1].y, v[2].x, v[2].y);
        float m2 = fmin3(v[3].x, v[3].y, v[4].x);
        float m3 = fmin3(v[4].y, v[5].x, v[5].y);
        float m4 = fmin3(v[6].x, v[6].y, v[7].x);
        float m5 = fmin3(v[7].y, v[8].x, v[8].y);
        float m6 = fmin3(v[9].x, v[9].y, v[10].x);
        float m7 = fmin3(v[10].y, v[11].x, v[11].y);
        float m8 = fmin3(v[12].x, v[12].y, v[13].x);
        float m9 = fmin3(v[13].y, v[14].x, v[14].y);
        float n0 = fmin3(m0, m1, m2);
        float n1 = fmin3(m3, m4, m5);
        float n2 = fmin3(m6, m7, m8);
        float n3 = fmin3(m9, v[15].x, v[15].y);
        float mm = fmin3(n0, n1, fminf(n2, n3));
        rmin = fminf(rmin, mm + A);
      }
      const uint32_t ilast = ig + 31u;
      if ((ilast & rmask) == rmask) {  // end of an aligned record group (sbits >= 5; uniform)
        float wmin = warp_min_f(rmin);
        if (lane == 0) {
          const uint64_t gi = (uint64_t)((ilast - i0) >> g.sbits);
          g.rec[rec_unit_base | (gi << 3) | (uint64_t)warp] = wmin;
        }
        rmin = inf;
      }
    }
    if (more) {
      float4* dst = reinterpret_cast<float4*>(gbuf + ((blk + 1) & 1) * kGrayStage * 32);
#pragma unroll
      for (int q = 0; q < 4; ++q) dst[t + q * kGrayThreads] = nxt[q];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kGrayThreads, 2) gray_pass1_kernel(GrayParams g) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  gray_unit_body(g, blockIdx.x, smem_raw);
}

}  // namespace qb
