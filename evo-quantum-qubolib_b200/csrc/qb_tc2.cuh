// qb_tc2.cuh -- tensor-core form with two states per accumulator (tile pairs): one problem,
// or (16-bit form) the work items of a batch.
//
// Same decomposition as qb_tc.cuh (t: tile index in Gray order, y: the 128 MMA rows, u: the
// 256 MMA columns; E(t, y, u) = R_t(y) + C_t(u) + y^T V u), but the Gray-ordered tiles are
// taken in pairs (i, i + 1) with i even.  Their tile values t and t' = t ^ 1 differ in t
// bit 0 (variable n-16) alone, so
//   E(t', y, u) = R_t'(y) + D(y, u) + s * gamma(u),   D(y, u) = y^T V u + C_t(u)
//   gamma(u)    = sum_j W[n-16][n-1-j] u_j          (the couplings of variable n-16 with u)
//   s           = +1 if t bit 0 is 0, else -1       (bit 0 of gray(i) = (i >> 1) & 1)
// One MMA computes D for tile t; the epilogue reads each accumulator once and derives the
// partner tile's value from it.  Every TMEM accumulator thus stands for two states, which
// halves the MMAs, accumulator round trips and TMEM loads per state.  Measured on B200
// (n = 36 TSP QUBO, 2^36 states): fp32 pair form 3.83 ms, 16-bit pair form (below) 2.36 ms,
// against 3.8-3.95 ms for one state per accumulator; the 16-bit pair form is the default
// where it applies, and qb_autotune times both forms.
//
// Roles, pipelines, records and bounded waits are those of tc_pass1_kernel<false>
// (qb_tc.cuh), with "tile" replaced by "pair" in the MMA, B-stage and accumulator
// pipelines: per pair the B producer writes the column-term digits of tile t and the row
// terms of both tiles.  acc_full takes two arrivals, the MMA's commit and the MMA thread's
// own arrive after it saw the pair's B stage full, so the epilogue's acquire of acc_full
// also orders the row terms and it needs no wait on the B stage.  Records: per block of
// 2^gl tiles (2^(gl-1) pairs, gl >= 5) 8 records, as in qb_tc.cuh (kGeomTC); a pair never
// straddles two blocks.
//
// fp32 pair form (tc_pair_fp32_kernel): the partner's values by one fma per state (gamma of the 5
// low u bits as constant operands, the 3 high u bits added to each 32-column chunk's minimum)
// and 3-input fp32 minima.
//
// 16-bit pair form (tc_pair_kernel<kItems>: one problem, or the batch's work items;
// tc2_u16_eligible, tc2_u16_quantized).  As in the one-state 16-bit epilogue (qb_tc.cuh,
// tc_u16_eligible) the accumulator is an integer in [2^23, 2^24) whose fp32 pattern holds a
// 16-bit value in its low half, loaded two columns per register (.pack::16b).  Here the MMA
// computes F = D~ + 2^23 - Dlow_s with D~(y, u) = D(y, u) + s * X(u), X the gamma of the chunk
// bits u4, u5, u6 and Dlow_s = Dmin + min_u s * X(u): the column term carries s * X(u).  In a
// warp's 64 registers (u = 128 hh + 32 L + 2 j + half, register j of load L) the chunk
// c = (u4, u5, u6) = (j >> 3, L) and the position k = j & 7 (u1, u2, u3) with the half bit u0
// index an 8 x 8 grid, and
//   tile t:   D  - Dmin = (F mod 2^16) - s * X(c) + (Dlow_s - Dmin)       per-chunk correction
//   tile t':  D' - Dmin = (F mod 2^16) + s * (gamma - X)(k, u0, hh) + (Dlow_s - Dmin)
//                                                                      per-position correction
// so tile t takes the packed minimum over each chunk (8 registers) plus one add.u16x2 per
// chunk, and tile t' the packed minimum over the 8 chunks at each position plus one add.u16x2
// per position: 64 packed 3-input minimum inputs and 16 adds per 64 registers (8192 states),
// against 64 adds more when the partner's values are formed register by register.  Every
// corrected value is D - Dmin of a state, in [0, Dmax - Dmin]; the uncorrected ones lie in
// [0, Dmax - Dmin + sum_{b=4..6} |gamma_b|] < 2^16 (the eligibility condition), so packed
// 16-bit minima and mod-2^16 adds are exact.  Each warp's pairs share one parity, hence one
// sign s and one set of 16 corrections, kept in registers.  The column term's constant part
// E_U(u) + s X(u) + 2^23 - Dlow_s sits in three constant K slots of each B stage (a stage
// always holds pairs of one parity); the producer writes only the tile-dependent part
// T(u) = (t^T W_TU) u as two digits per pair.
//
// Exactness: for integer Q with sum|Q| <= 2^22, D + s*gamma(u) = y^T V u + C_t'(u) is an
// integer of magnitude at most sum|Q| (it is the accumulator tile t' would have had), so the
// fma is exact.  For float Q, gamma in fp32, its partial sums g5, the fma and the chunk
// offset add at most 8 roundings of 2^-24 relative to sum|Q| (scaled units) to the error
// bound of the digit contraction; tc2_error_bound() includes them.
#pragma once
#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>

#include "qb_tc.cuh"

namespace qb {

// per-state error bound of the float-digit pair form (unscaled units)
inline double tc2_error_bound(double abs_sum) { return 264.0 * abs_sum * 5.9604644775390625e-08 + 1e-300; }

// the 16-bit pair form's constants of one problem (one sign per accumulator stage: [0] for
// s = +1, [1] for s = -1), in the problem's units
struct Tc2Tab {
  float gx[3];               // gamma of the chunk bits u4, u5, u6
  float k0s[2];              // 2^23 - Dlow_s, the offset of the column term
  float dmin;                // lower bound of every accumulator value D
  uint32_t corr_t[2][8];     // tile t: correction of chunk c (u4 = c & 1, u5, u6 = c >> 1), both halves
  uint32_t corr_p[2][2][8];  // partner: correction of position k (u1..u3) in column half hh (u7)
};

struct Tc2Params {
  TcParams P;       // n, nt, gl, stall, exact, inv_scale, W, tile_begin, groups, groups_per_cta, rec, err
  alignas(8) float g5[32];     // fp32 form: gamma of register k of a 32-column chunk, sum_{j < 5} w_j k_j
  float whi[3];     // fp32 form: w_5, w_6, w_7, the gamma of u bits 5..7 (scaled W)
  Tc2Tab tab;       // 16-bit form, one problem (tc_pair_kernel<false>)
  const Tc2Tab* tabs;  // 16-bit form, work items: per item (tc_pair_kernel<true>)
};

// u bits that form the 16-bit pair epilogue's chunks (their gamma is folded into the MMA)
constexpr int kTc2ChunkBits[3] = {4, 5, 6};

// The 16-bit pair form applies (integer Q on the exact path; W unscaled, n x n FP64): the
// problems of the one-state 16-bit epilogue with room for the chunk offsets,
// Dmax - Dmin + sum over the chunk bits b of |gamma_b| < 2^16.
inline bool tc2_u16_eligible(int n, const double* W, float* dmin) {
  double span = 0.0;
  if (!tc_u16_eligible(n, W, dmin, &span)) return false;
  double gx = 0.0;
  for (int b : kTc2ChunkBits) gx += std::fabs(W[(size_t)(n - 16) * n + (n - 1 - b)]);
  return span + gx <= 65535.0;
}

// The 16-bit pair form off the exact path (float Q, or integer Q with sum|Q| > 2^22).  The
// kernel then works in units of 1/sigma, sigma a power of two applied to W: every MMA operand
// (the y coupling rows, T(u), the column term's constant part, the gammas of the corrections)
// is rounded to an integer in those units, so the accumulators are integers and the 16-bit
// epilogue stays exact on the rounded values.  Per state the roundings add at most 4.5 units
// (seven y rows, T and E_U at 0.5 each), the partner's rounded gammas 4 more, the row term's
// bias 0.5, plus fp32 rounding of the row terms and of T below 2^-18 sum|Q| sigma; eps =
// 10 / sigma + 2^-16 sum|Q| bounds it (unscaled) and pass 2 re-walks every record within
// 2 eps of the minimum in FP64.  Applies when, at the largest such sigma, every y coupling
// row stays within +-2047 units, the value span with the chunk offsets and a 40-unit margin
// within 2^16 units, and the span covers at least 1024 units.  W: the unscaled n x n FP64 W.
// On success: sigma, dmin (the lower bound of the rounded values in units, an integer) and eps.
inline bool tc2_u16_quantized(int n, const double* W, double abs_sum, double* sigma, float* dmin, double* eps) {
  if (n < 20) return false;
  double lo = 0.0, hi = 0.0, rowmax = 0.0;
  auto add = [&](double w) {
    if (w < 0) lo += w;
    else hi += w;
  };
  for (int i = 0; i < 7; ++i) {
    double rp = 0.0, rn = 0.0;
    for (int j = 0; j < 8; ++j) {
      const double w = W[(size_t)(n - 9 - i) * n + (n - 1 - j)];
      if (w < 0) rn -= w;
      else rp += w;
      add(w);
    }
    rowmax = std::max(rowmax, std::max(rp, rn));
  }
  for (int j = 0; j < 8; ++j) {
    const int a = n - 1 - j;
    add(W[(size_t)a * n + a]);
    for (int j2 = 0; j2 < j; ++j2) add(W[(size_t)a * n + (n - 1 - j2)]);
    for (int t = 0; t < n - 15; ++t) add(W[(size_t)t * n + a]);
  }
  double gA = 0.0;
  for (int b : kTc2ChunkBits) gA += std::fabs(W[(size_t)(n - 16) * n + (n - 1 - b)]);
  const double span = hi - lo;
  if (!(span > 0.0) || !std::isfinite(span + gA)) return false;
  double lim = (65535.0 - 40.0) / (span + gA);
  if (rowmax > 0.0) lim = std::min(lim, 2047.0 / rowmax);
  double sg = std::ldexp(1.0, (int)std::floor(std::log2(lim)));
  while (sg * rowmax > 2047.0 || sg * (span + gA) + 40.0 > 65535.0) sg *= 0.5;
  if (sg * span < 1024.0) return false;  // too coarse: most records would become candidates
  *sigma = sg;
  *dmin = (float)(std::floor(sg * lo) - 12.0);
  *eps = 10.0 / sg + std::ldexp(abs_sum, -16);
  return true;
}


// the 16-bit pair form's constants from gamma (integers in the kernel's units, rounded here)
// and Dmin
inline void tc2_u16_tables(const float* gamma, float dmin, Tc2Tab* Q) {
  Q->dmin = dmin;
  int64_t g[8];
  for (int j = 0; j < 8; ++j) g[j] = (int64_t)std::llrint(gamma[j]);
  for (int b = 0; b < 3; ++b) Q->gx[b] = (float)g[kTc2ChunkBits[b]];
  for (int neg = 0; neg < 2; ++neg) {
    const int64_t s = neg ? -1 : 1;
    int64_t lo = 0;  // min over the chunk bits of s * X(u) = Dlow_s - Dmin
    for (int b = 0; b < 3; ++b) lo += std::min<int64_t>(0, s * g[kTc2ChunkBits[b]]);
    Q->k0s[neg] = (float)(8388608.0 - ((double)dmin + (double)lo));
    for (int c = 0; c < 8; ++c) {
      const int64_t x = ((c & 1) ? g[4] : 0) + ((c & 2) ? g[5] : 0) + ((c & 4) ? g[6] : 0);
      const uint32_t v = (uint32_t)((lo - s * x) & 0xffff);
      Q->corr_t[neg][c] = v | (v << 16);
    }
    for (int hh = 0; hh < 2; ++hh)
      for (int k = 0; k < 8; ++k) {
        uint32_t h[2];
        for (int d = 0; d < 2; ++d) {
          const int64_t gp = (d ? g[0] : 0) + ((k & 1) ? g[1] : 0) + ((k & 2) ? g[2] : 0) + ((k & 4) ? g[3] : 0) +
                             (hh ? g[7] : 0);
          h[d] = (uint32_t)((s * gp + lo) & 0xffff);
        }
        Q->corr_p[neg][hh][k] = h[0] | (h[1] << 16);
      }
  }
}

#ifdef __CUDACC__

// min over k of (D_k + s * g5[k]) for one 32-column chunk, two registers per packed fma
// (fma.rn.f32x2: the same rounding as two scalar fmas); g5 pairs are read from the parameter
// space with a constant index
__device__ __forceinline__ float min32_shift(const uint32_t* r, const Tc2Params& Q, float s) {
  float v[32];
  const uint64_t ss = ((uint64_t)__float_as_uint(s) << 32) | __float_as_uint(s);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const uint64_t g = *reinterpret_cast<const uint64_t*>(&Q.g5[2 * k]);
    const uint64_t d = ((uint64_t)r[2 * k + 1] << 32) | r[2 * k];
    uint64_t o;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(o) : "l"(g), "l"(ss), "l"(d));
    v[2 * k] = __uint_as_float((uint32_t)o);
    v[2 * k + 1] = __uint_as_float((uint32_t)(o >> 32));
  }
  float m0 = fmin3(v[0], v[1], v[2]);
  float m1 = fmin3(v[3], v[4], v[5]);
  float m2 = fmin3(v[6], v[7], v[8]);
  float m3 = fmin3(v[9], v[10], v[11]);
  float m4 = fmin3(v[12], v[13], v[14]);
  float m5 = fmin3(v[15], v[16], v[17]);
  float m6 = fmin3(v[18], v[19], v[20]);
  float m7 = fmin3(v[21], v[22], v[23]);
  float m8 = fmin3(v[24], v[25], v[26]);
  float m9 = fmin3(v[27], v[28], v[29]);
  float n0 = fmin3(m0, m1, m2);
  float n1 = fmin3(m3, m4, m5);
  float n2 = fmin3(m6, m7, m8);
  float n3 = fmin3(m9, v[30], v[31]);
  return fmin3(n0, n1, fminf(n2, n3));
}

__device__ __forceinline__ uint32_t uadd2(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("add.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));  // per half, mod 2^16
  return d;
}

// packed unsigned 16-bit minimum of 8 registers (3-input minima)
__device__ __forceinline__ uint32_t umin8(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t e, uint32_t f,
                                          uint32_t g, uint32_t h) {
  return __vimin3_u16x2(__vimin3_u16x2(a, b, c), __vimin3_u16x2(d, e, f), umin2(g, h));
}

__global__ void __launch_bounds__(kTcThreads, 1) tc_pair_fp32_kernel(const __grid_constant__ Tc2Params Q) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  const TcParams& P = Q.P;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const TcSmemLayout L = tc_layout(P.n);
  unsigned char* Asm = tc_smem + L.a_off;
  unsigned char* Bsm = tc_smem + L.b_off;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tc_smem + L.bar_off);
  uint64_t* p_full = bars;
  uint64_t* p_empty = p_full + kTcParamSlots;
  uint64_t* b_full = p_empty + kTcParamSlots;
  uint64_t* b_empty = b_full + kTcBStages;
  uint64_t* acc_full = b_empty + kTcBStages;
  uint64_t* acc_empty = acc_full + kTcStages;
  TcSlot* slots = reinterpret_cast<TcSlot*>(tc_smem + L.slot_off);
  float* EU = reinterpret_cast<float*>(tc_smem + L.eu_off);
  float* EY = reinterpret_cast<float*>(tc_smem + L.ey_off);
  float* Rs = reinterpret_cast<float*>(tc_smem + L.rs_off);            // tile t of each pair
  float* Rs2 = reinterpret_cast<float*>(tc_smem + L.total);            // tile t' of each pair
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + L.misc_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tc_smem + L.misc_off + 4);
  double* LO = reinterpret_cast<double*>(tc_smem + L.lo_off);
  double* Ws = reinterpret_cast<double*>(tc_smem + L.w_off);

  const uint64_t g0 = (uint64_t)blockIdx.x * P.groups_per_cta;
  if (g0 >= P.groups) return;  // uniform per CTA
  const uint64_t g1 = min(P.groups, g0 + P.groups_per_cta);
  const int n = P.n, nt = P.nt, gl = P.gl, exact = P.exact;
  const uint64_t i_begin = P.tile_begin + (g0 << gl), ntiles = (g1 - g0) << gl;
  float* rec = P.rec + (g0 << 3);
  const uint64_t t0 = gray64(i_begin);
  const float s1 = exact ? 2048.0f : 1.0f;

  if (tid == 0) {
    for (int s = 0; s < kTcParamSlots; ++s) {
      mbar_init(&p_full[s], 1);
      mbar_init(&p_empty[s], 1);
    }
    for (int s = 0; s < kTcBStages; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
    }
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&acc_full[s], 2);  // the MMA's commit and the MMA thread (after it saw the B stage full)
      mbar_init(&acc_empty[s], kTcEpiWarps / 2);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  for (int i = tid; i < n * n; i += kTcThreads) Ws[i] = P.W[i];
  for (uint64_t r = (uint64_t)tid; r < ((ntiles >> gl) << 3); r += kTcThreads) rec[r] = __int_as_float(0x7f800000);
  __syncthreads();
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
  for (int e = tid; e < kTcN * 7; e += kTcThreads) {
    int u = e / 7, i = e % 7;
    const double* row = Ws + (n - 9 - i) * n;
    double v = 0.0;
    for (int j = 0; j < 8; ++j)
      if ((u >> j) & 1) v += row[n - 1 - j];
    __half2 dg = digits((float)v, exact);
    for (int s = 0; s < kTcBStages; ++s)
      *reinterpret_cast<__half2*>(Bsm + s * kTcN * 32 + kmaj_off(u, 2 * i)) = dg;
  }
  for (int u = tid; u < kTcN; u += kTcThreads) {
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
  for (int y = tid; y < 128; y += kTcThreads) {
    double e = 0.0;
    for (int i = 0; i < 7; ++i) {
      if (!((y >> i) & 1)) continue;
      const double* row = Ws + (n - 9 - i) * n;
      e += row[n - 9 - i];
      for (int i2 = 0; i2 < i; ++i2)
        if ((y >> i2) & 1) e += row[n - 9 - i2];
    }
    EY[y] = (float)e;
  }
  for (int e = tid; e < 32 * 16; e += kTcThreads) {
    const int p = e >> 4, c = e & 15;
    double v = 0.0;
    if (c == 15) {
      for (int k = 0; k < 5; ++k) {
        if (!((p >> k) & 1)) continue;
        const double* row = Ws + (n - 16 - k) * n;
        v += row[n - 16 - k];
        for (int k2 = 0; k2 < k; ++k2)
          if ((p >> k2) & 1) v += row[n - 16 - k2];
      }
    } else {
      const int col = c < 8 ? n - 1 - c : n - 9 - (c - 8);
      for (int k = 0; k < 5; ++k)
        if ((p >> k) & 1) v += Ws[(n - 16 - k) * n + col];
    }
    LO[e] = v;
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t npairs = (uint32_t)(ntiles >> 1);

  bool ok = true;
  if (warp == 0 && P.stall) {
    // test hook (QB_FLAG_TEST_STALL): nothing is published, every other wait runs out
  } else if (warp == 0) {
    // ------------------------------------------------------------ tile walk (every tile)
    const int nh = nt - 5;
    double fh[8], gh[7], c[5], eh = 0.0, h0 = 0.0, h1 = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) fh[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 7; ++k) gh[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) c[k] = 0.0;
    const uint64_t th0 = t0 >> 5;
    for (int m = 0; m < nh; ++m) {
      if (!((th0 >> m) & 1)) continue;
      const double* row = Ws + (n - 21 - m) * n;
      eh += row[n - 21 - m];
      for (int m2 = 0; m2 < m; ++m2)
        if ((th0 >> m2) & 1) eh += row[n - 21 - m2];
      if (lane < nh && lane != m) h0 += row[n - 21 - lane];
      if (lane + 32 < nh && lane + 32 != m) h1 += row[n - 21 - lane - 32];
#pragma unroll
      for (int k = 0; k < 8; ++k) fh[k] += row[n - 1 - k];
#pragma unroll
      for (int k = 0; k < 7; ++k) gh[k] += row[n - 9 - k];
#pragma unroll
      for (int k = 0; k < 5; ++k) c[k] += row[n - 16 - k];
    }
    for (uint64_t j0 = 0; j0 < ntiles && ok; j0 += 32) {
      const uint64_t i0 = i_begin + j0;
      if (j0 > 0) {
        const int kb = __ffsll((long long)i0) - 1;
        const int m = kb - 5;
        const double sg = ((gray64(i0) >> kb) & 1) ? 1.0 : -1.0;
        const double hm = __shfl_sync(0xffffffffu, m < 32 ? h0 : h1, m & 31);
        const double* row = Ws + (n - 21 - m) * n;
        eh += sg * (row[n - 21 - m] + hm);
        if (lane < nh && lane != m) h0 += sg * row[n - 21 - lane];
        if (lane + 32 < nh && lane + 32 != m) h1 += sg * row[n - 21 - lane - 32];
#pragma unroll
        for (int k = 0; k < 8; ++k) fh[k] += sg * row[n - 1 - k];
#pragma unroll
        for (int k = 0; k < 7; ++k) gh[k] += sg * row[n - 9 - k];
#pragma unroll
        for (int k = 0; k < 5; ++k) c[k] += sg * row[n - 16 - k];
      }
      const uint64_t j = j0 + (uint64_t)lane;
      const int tl = (int)(gray64(i0 + (uint64_t)lane) & 31ull);
      const double* lo = LO + tl * 16;
      double et = eh + lo[15];
#pragma unroll
      for (int k = 0; k < 5; ++k)
        if ((tl >> k) & 1) et += c[k];
      const int s = (int)(j % kTcParamSlots);
      ok = mbar_wait(&p_empty[s], (uint32_t)(((j / kTcParamSlots) & 1) ^ 1), abort_flag);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      TcSlot& sl = slots[s];
#pragma unroll
      for (int k = 0; k < 8; ++k) sl.f[k] = (float)(fh[k] + lo[k]);
#pragma unroll
      for (int k = 0; k < 7; ++k) sl.g[k] = (float)(gh[k] + lo[8 + k]);
      sl.et = (float)et;
      mbar_arrive(&p_full[s]);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issue (one per pair)
    if (lane == 0) {
      const uint64_t adesc = umma_desc(smem_u32(Asm), 128, 256);
      const uint64_t bdesc0 = umma_desc(smem_u32(Bsm), 128, 256);
      for (uint32_t p0 = 0; p0 < npairs && ok; p0 += kTcBStages) {
        const uint32_t pb = (p0 >> 3) & 1u;
#pragma unroll
        for (int k = 0; k < kTcBStages; ++k) {
          const uint32_t as = (uint32_t)k & 1u;
          ok = mbar_wait(&b_full[k], pb, abort_flag) &&
               mbar_wait_short(&acc_empty[as], (((uint32_t)k >> 1) & 1u) ^ 1u, abort_flag);
          if (!ok) break;
          tc_fence_after();
          if (p0 + (uint32_t)k >= (uint32_t)kTcStages) mbar_arrive(&b_empty[(k + kTcBStages - kTcStages) % kTcBStages]);
          tc_mma(tmem + as * (uint32_t)kTcN, adesc, bdesc0 + (uint64_t)(k * (kTcN * 32 / 16)));
          tc_commit(&acc_full[as]);
          // the second arrival on acc_full: this thread has seen the B stage full, so the
          // epilogue's acquire of acc_full also orders the row terms written with the stage
          mbar_arrive(&acc_full[as]);
        }
      }
    }
    __syncwarp();
  } else if (warp < 4) {
    // ------------------------------------------------------------ B producers (per pair)
    // warp 2 + (p & 1) fills pair p: the C_t(u) digits of tile 2p (rows u = lane + 32 r) and
    // the row terms of tiles 2p and 2p + 1 (rows y = lane + 32 r)
    for (uint32_t p = (uint32_t)(warp - 2); p < npairs && ok; p += 2) {
      const uint32_t ja = 2 * p, jb = ja + 1;
      const uint32_t sa = ja & (uint32_t)(kTcParamSlots - 1), sb = jb & (uint32_t)(kTcParamSlots - 1);
      const uint32_t bs = p & (uint32_t)(kTcBStages - 1);
      ok = mbar_wait(&p_full[sa], (ja >> 6) & 1u, abort_flag) && mbar_wait(&p_full[sb], (jb >> 6) & 1u, abort_flag);
      if (!ok) break;
      __half2 dg[8];
      float ra[4], rb[4];
      {
        const TcSlot& sl = slots[sa];
        float s5 = 0.f;
#pragma unroll
        for (int jb5 = 0; jb5 < 5; ++jb5)
          if ((lane >> jb5) & 1) s5 += sl.f[jb5];
        const float f5 = sl.f[5], f6 = sl.f[6], f7 = sl.f[7];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          float cr = s5;
          if (r & 1) cr += f5;
          if (r & 2) cr += f6;
          if (r & 4) cr += f7;
          dg[r] = digits(EU[lane + 32 * r] + cr, exact);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const TcSlot& sl = slots[h ? sb : sa];
        float g5 = sl.et;
#pragma unroll
        for (int i = 0; i < 5; ++i)
          if ((lane >> i) & 1) g5 += sl.g[i];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          float v = g5;
          if (r & 1) v += sl.g[5];
          if (r & 2) v += sl.g[6];
          (h ? rb : ra)[r] = v + EY[lane + 32 * r];
        }
      }
      ok = mbar_wait(&b_empty[bs], ((p >> 3) & 1u) ^ 1u, abort_flag);
      if (!ok) break;
      unsigned char* Bst = Bsm + bs * kTcN * 32;
#pragma unroll
      for (int r = 0; r < 8; ++r) *reinterpret_cast<__half2*>(Bst + kmaj_off(lane + 32 * r, 14)) = dg[r];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        Rs[bs * 128 + lane + 32 * r] = ra[r];
        Rs2[bs * 128 + lane + 32 * r] = rb[r];
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&b_full[bs]);
        mbar_arrive(&p_empty[sa]);
        mbar_arrive(&p_empty[sb]);
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;
    const int cq = (warp - 4) >> 2;
    const int y = q * 32 + lane;
    const float inf = __int_as_float(0x7f800000);
    float rmin = inf;
    const uint32_t sp = (uint32_t)cq >> 1;   // pair parity = accumulator stage
    const uint32_t hh = (uint32_t)cq & 1u;   // column half: u bit 7
    const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + sp * (uint32_t)kTcN + hh * 128u;
    // gamma of u bits 5..7 for the four 32-column chunks of this half
    float ghi[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) ghi[c] = ((c & 1) ? Q.whi[0] : 0.f) + ((c & 2) ? Q.whi[1] : 0.f) + (hh ? Q.whi[2] : 0.f);
    // records every 2^gl tiles = 2^(gl-1) pairs, 2^(gl-2) of this warp's parity
    uint32_t rec_left = 1u << (gl - 2);
    uint32_t Jrec = 0;
    for (uint32_t p = sp; p < npairs && ok; p += 2) {
      const uint32_t bs = p & (uint32_t)(kTcBStages - 1);
      // s = +1 when tile 2p has t bit 0 clear (its partner sets the bit); i_begin is even
      const float s = (((i_begin >> 1) + p) & 1ull) ? -1.0f : 1.0f;
      // acc_full completes after the MMA thread saw this pair's B stage full
      ok = mbar_wait(&acc_full[sp], (p >> 1) & 1u, abort_flag);
      if (!ok) break;
      const float R1 = Rs[bs * 128 + y];
      const float R2 = Rs2[bs * 128 + y];
      tc_fence_after();
      uint32_t ra[32], rb[32];
      QB_TC_LD32(tbase, ra);
      QB_TC_LD32(tbase + 32, rb);
      tc_wait_ld();
      reg_fence32(ra);
      reg_fence32(rb);
      float m1 = fminf(min32(ra), min32(rb));
      float m2 = fminf(fmaf(ghi[0], s, min32_shift(ra, Q, s)), fmaf(ghi[1], s, min32_shift(rb, Q, s)));
      QB_TC_LD32(tbase + 64, ra);
      QB_TC_LD32(tbase + 96, rb);
      tc_wait_ld();
      reg_fence32(ra);
      reg_fence32(rb);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[sp]);
      m1 = fminf(m1, fminf(min32(ra), min32(rb)));
      m2 = fmin3(m2, fmaf(ghi[2], s, min32_shift(ra, Q, s)), fmaf(ghi[3], s, min32_shift(rb, Q, s)));
      rmin = fmin3(rmin, m1 + R1, m2 + R2);
      if (--rec_left == 0) {
        const float wm = warp_min_f(rmin) * P.inv_scale;
        if (lane == 0) {
          float* dst = rec + (((uint64_t)Jrec << 3) | ((uint64_t)hh << 2) | (uint64_t)q);
          if (wm >= 0.f)
            atomicMin(reinterpret_cast<int*>(dst), __float_as_int(wm));
          else
            atomicMax(reinterpret_cast<unsigned*>(dst), __float_as_uint(wm));
        }
        ++Jrec;
        rec_left = 1u << (gl - 2);
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


// The 16-bit pair form.  kItems = false: one problem, each CTA a contiguous run of its record
// blocks (one work item), its constants in Q.tab; kItems = true: the CTA's list of work items
// (runs of record blocks of the batch's problems, qb_batch.cuh), Q.tabs[it] the constants of
// item it's problem, as tc_pass1_kernel<true> does for one state per accumulator.  Every role
// walks the CTA's tiles in the same order; barrier slots, B stages and phases follow the
// CTA-wide tile counter jbase (a multiple of 32: every item has a multiple of 2^gl >= 32
// tiles), pairs the pair counter jbase / 2.  Between items all roles meet at a CTA barrier
// with the pipelines empty (the MMA thread waits for its last MMA), so the per-item tables,
// B operand columns and constants can be rewritten.  W is in the problem's units (scaled by
// sigma off the exact path).
template <bool kItems>
__global__ void __launch_bounds__(kTcThreads, 1) tc_pair_kernel(const __grid_constant__ Tc2Params Q) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  const TcParams& P = Q.P;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const TcSmemLayout L = tc_layout(kItems ? P.n_max : P.n);  // only the W block grows with n
  unsigned char* Asm = tc_smem + L.a_off;
  unsigned char* Bsm = tc_smem + L.b_off;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tc_smem + L.bar_off);
  uint64_t* p_full = bars;
  uint64_t* p_empty = p_full + kTcParamSlots;
  uint64_t* b_full = p_empty + kTcParamSlots;
  uint64_t* b_empty = b_full + kTcBStages;
  uint64_t* acc_full = b_empty + kTcBStages;
  uint64_t* acc_empty = acc_full + kTcStages;
  TcSlot* slots = reinterpret_cast<TcSlot*>(tc_smem + L.slot_off);
  float* EU = reinterpret_cast<float*>(tc_smem + L.eu_off);
  float* EY = reinterpret_cast<float*>(tc_smem + L.ey_off);
  float* Rs = reinterpret_cast<float*>(tc_smem + L.rs_off);  // tile t of each pair
  float* Rs2 = reinterpret_cast<float*>(tc_smem + L.total);  // tile t' of each pair
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + L.misc_off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tc_smem + L.misc_off + 4);
  double* LO = reinterpret_cast<double*>(tc_smem + L.lo_off);
  double* Ws = reinterpret_cast<double*>(tc_smem + L.w_off);

  // this CTA's work: one run of record blocks of one problem, or a list of items
  uint32_t it_lo = 0, it_hi = 1;
  TcItem one{};
  if (kItems) {
    it_lo = P.item_first[blockIdx.x];
    it_hi = P.item_first[blockIdx.x + 1];
    if (it_lo >= it_hi) return;  // uniform per CTA
  } else {
    const uint64_t g0 = (uint64_t)blockIdx.x * P.groups_per_cta;
    if (g0 >= P.groups) return;  // uniform per CTA
    const uint64_t g1 = min(P.groups, g0 + P.groups_per_cta);
    one = TcItem{P.W, P.rec + (g0 << 3), P.tile_begin + (g0 << P.gl), (g1 - g0) << P.gl, P.n, P.gl, P.exact,
                 P.inv_scale};
  }

  if (tid == 0) {
    for (int s = 0; s < kTcParamSlots; ++s) {
      mbar_init(&p_full[s], 1);
      mbar_init(&p_empty[s], 1);
    }
    for (int s = 0; s < kTcBStages; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
    }
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&acc_full[s], 2);  // the MMA's commit and the MMA thread (after it saw the B stage full)
      mbar_init(&acc_empty[s], kTcEpiWarps / 2);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // A operand (constant, the same for every item): A[y][i] = y_i (i < 7); digit weights: T
  // (slots 8, 9) 1, 2048; the constant part (slots 10-12) 1, 2048, 32768
  for (int e = tid; e < 128 * 16; e += kTcThreads) {
    const int y = e >> 4, k = e & 15;
    const float v = k < 7 ? (float)((y >> k) & 1)
                          : (k == 8 || k == 10 ? 1.0f : (k == 9 || k == 11 ? 2048.0f : (k == 12 ? 32768.0f : 0.0f)));
    *reinterpret_cast<__half*>(Asm + kmaj_off(y, k)) = __float2half_rn(v);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  uint32_t jnext = 0;  // CTA-wide tile counter of the next item
  for (uint32_t it = it_lo; it < it_hi; ++it) {
    const TcItem I = kItems ? P.items[it] : one;
    const Tc2Tab& Tb = kItems ? Q.tabs[it] : Q.tab;
    const int n = I.n, nt = n - 15, gl = I.gl;
    const uint64_t i_begin = I.i_begin, ntiles = I.ntiles;
    float* rec = I.rec;
    const uint64_t t0 = gray64(i_begin);
    // the CTA-wide tile and pair counters at the item's start (a compile-time 0 for one
    // problem, so its barrier parities and stages reduce to constants as in a one-item kernel)
    const uint32_t jbase = kItems ? jnext : 0u;
    const uint32_t pbase = jbase >> 1;  // a multiple of 16

    // ------------------------------------------------------------ per-item set-up
    for (int i = tid; i < n * n; i += kTcThreads) Ws[i] = I.W[i];
    for (uint64_t r = (uint64_t)tid; r < ((ntiles >> gl) << 3); r += kTcThreads) rec[r] = __int_as_float(0x7f800000);
    __syncthreads();
    // B operand: coupling rows of the y variables (one exact fp16 integer each), zeros
    for (int e = tid; e < kTcN * 16; e += kTcThreads) {
      const int u = e >> 4, k = e & 15;
      if (k >= 8 && k < 13) continue;  // T's digits (per pair) and the constant digits (below)
      double v = 0.0;
      if (k < 7) {
        const double* row = Ws + (n - 9 - k) * n;
        for (int j = 0; j < 8; ++j)
          if ((u >> j) & 1) v += row[n - 1 - j];
      }
      const __half hv = __float2half_rn((float)rint(v));
      for (int s = 0; s < kTcBStages; ++s) *reinterpret_cast<__half*>(Bsm + s * kTcN * 32 + kmaj_off(u, k)) = hv;
    }
    for (int u = tid; u < kTcN; u += kTcThreads) {
      double e = 0.0;
      for (int j = 0; j < 8; ++j) {
        if (!((u >> j) & 1)) continue;
        const double* row = Ws + (n - 1 - j) * n;
        e += row[n - 1 - j];
        for (int j2 = 0; j2 < j; ++j2)
          if ((u >> j2) & 1) e += row[n - 1 - j2];
      }
      EU[u] = (float)e;
      // the column term's constant part E_U(u) + s X(u) + 2^23 - Dlow_s in three exact digits;
      // B stage bs holds pairs of parity bs & 1 (the pair counter is a multiple of 16), one sign
      const double x = ((u >> 4) & 1 ? (double)Tb.gx[0] : 0.0) + ((u >> 5) & 1 ? (double)Tb.gx[1] : 0.0) +
                       ((u >> 6) & 1 ? (double)Tb.gx[2] : 0.0);
      for (int bs = 0; bs < kTcBStages; ++bs) {
        const uint32_t neg = (uint32_t)(((i_begin >> 1) + (uint64_t)bs) & 1ull);
        const double c = rint(e) + (neg ? -x : x) + (double)Tb.k0s[neg];
        const double d2 = floor(c * (1.0 / 32768.0)), rem = c - 32768.0 * d2;
        const double d1 = floor(rem * (1.0 / 2048.0)), d0 = rem - 2048.0 * d1;
        unsigned char* Bst = Bsm + bs * kTcN * 32;
        *reinterpret_cast<__half*>(Bst + kmaj_off(u, 10)) = __float2half_rn((float)d0);
        *reinterpret_cast<__half*>(Bst + kmaj_off(u, 11)) = __float2half_rn((float)d1);
        *reinterpret_cast<__half*>(Bst + kmaj_off(u, 12)) = __float2half_rn((float)d2);
      }
    }
    for (int y = tid; y < 128; y += kTcThreads) {
      double e = 0.0;
      for (int i = 0; i < 7; ++i) {
        if (!((y >> i) & 1)) continue;
        const double* row = Ws + (n - 9 - i) * n;
        e += row[n - 9 - i];
        for (int i2 = 0; i2 < i; ++i2)
          if ((y >> i2) & 1) e += row[n - 9 - i2];
      }
      EY[y] = (float)e;
    }
    for (int e = tid; e < 32 * 16; e += kTcThreads) {
      const int p = e >> 4, c = e & 15;
      double v = 0.0;
      if (c == 15) {
        for (int k = 0; k < 5; ++k) {
          if (!((p >> k) & 1)) continue;
          const double* row = Ws + (n - 16 - k) * n;
          v += row[n - 16 - k];
          for (int k2 = 0; k2 < k; ++k2)
            if ((p >> k2) & 1) v += row[n - 16 - k2];
        }
      } else {
        const int col = c < 8 ? n - 1 - c : n - 9 - (c - 8);
        for (int k = 0; k < 5; ++k)
          if ((p >> k) & 1) v += Ws[(n - 16 - k) * n + col];
      }
      LO[e] = v;
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t npairs = (uint32_t)(ntiles >> 1);

    bool ok = true;
    if (warp == 0 && P.stall) {
      // test hook (QB_FLAG_TEST_STALL): nothing is published, every other wait runs out
    } else if (warp == 0) {
      // ---------------------------------------------------------- tile walk (every tile)
      const int nh = nt - 5;
      double fh[8], gh[7], c[5], eh = 0.0, h0 = 0.0, h1 = 0.0;
#pragma unroll
      for (int k = 0; k < 8; ++k) fh[k] = 0.0;
#pragma unroll
      for (int k = 0; k < 7; ++k) gh[k] = 0.0;
#pragma unroll
      for (int k = 0; k < 5; ++k) c[k] = 0.0;
      const uint64_t th0 = t0 >> 5;
      for (int m = 0; m < nh; ++m) {
        if (!((th0 >> m) & 1)) continue;
        const double* row = Ws + (n - 21 - m) * n;
        eh += row[n - 21 - m];
        for (int m2 = 0; m2 < m; ++m2)
          if ((th0 >> m2) & 1) eh += row[n - 21 - m2];
        if (lane < nh && lane != m) h0 += row[n - 21 - lane];
        if (lane + 32 < nh && lane + 32 != m) h1 += row[n - 21 - lane - 32];
#pragma unroll
        for (int k = 0; k < 8; ++k) fh[k] += row[n - 1 - k];
#pragma unroll
        for (int k = 0; k < 7; ++k) gh[k] += row[n - 9 - k];
#pragma unroll
        for (int k = 0; k < 5; ++k) c[k] += row[n - 16 - k];
      }
      for (uint64_t j0 = 0; j0 < ntiles && ok; j0 += 32) {
        const uint64_t i0 = i_begin + j0;
        if (j0 > 0) {
          const int kb = __ffsll((long long)i0) - 1;
          const int m = kb - 5;
          const double sg = ((gray64(i0) >> kb) & 1) ? 1.0 : -1.0;
          const double hm = __shfl_sync(0xffffffffu, m < 32 ? h0 : h1, m & 31);
          const double* row = Ws + (n - 21 - m) * n;
          eh += sg * (row[n - 21 - m] + hm);
          if (lane < nh && lane != m) h0 += sg * row[n - 21 - lane];
          if (lane + 32 < nh && lane + 32 != m) h1 += sg * row[n - 21 - lane - 32];
#pragma unroll
          for (int k = 0; k < 8; ++k) fh[k] += sg * row[n - 1 - k];
#pragma unroll
          for (int k = 0; k < 7; ++k) gh[k] += sg * row[n - 9 - k];
#pragma unroll
          for (int k = 0; k < 5; ++k) c[k] += sg * row[n - 16 - k];
        }
        const uint64_t jg = jbase + j0 + (uint64_t)lane;  // CTA-wide tile counter
        const int tl = (int)(gray64(i0 + (uint64_t)lane) & 31ull);
        const double* lo = LO + tl * 16;
        double et = eh + lo[15];
#pragma unroll
        for (int k = 0; k < 5; ++k)
          if ((tl >> k) & 1) et += c[k];
        const int s = (int)(jg % kTcParamSlots);
        ok = mbar_wait(&p_empty[s], (uint32_t)(((jg / kTcParamSlots) & 1) ^ 1), abort_flag);
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        TcSlot& sl = slots[s];
#pragma unroll
        for (int k = 0; k < 8; ++k) sl.f[k] = (float)(fh[k] + lo[k]);
#pragma unroll
        for (int k = 0; k < 7; ++k) sl.g[k] = (float)(gh[k] + lo[8 + k]);
        sl.et = (float)et;
        mbar_arrive(&p_full[s]);
      }
    } else if (warp == 1) {
      // ---------------------------------------------------------- MMA issue (one per pair)
      if (lane == 0) {
        const uint64_t adesc = umma_desc(smem_u32(Asm), 128, 256);
        const uint64_t bdesc0 = umma_desc(smem_u32(Bsm), 128, 256);
        for (uint32_t p0 = 0; p0 < npairs && ok; p0 += kTcBStages) {
          const uint32_t g0p = pbase + p0;  // a multiple of 8
          const uint32_t pb = (g0p >> 3) & 1u;
#pragma unroll
          for (int k = 0; k < kTcBStages; ++k) {
            const uint32_t as = (uint32_t)k & 1u;
            ok = mbar_wait(&b_full[k], pb, abort_flag) &&
                 mbar_wait_short(&acc_empty[as], (((g0p + (uint32_t)k) >> 1) & 1u) ^ 1u, abort_flag);
            if (!ok) break;
            tc_fence_after();
            if (g0p + (uint32_t)k >= (uint32_t)kTcStages) mbar_arrive(&b_empty[(k + kTcBStages - kTcStages) % kTcBStages]);
            tc_mma(tmem + as * (uint32_t)kTcN, adesc, bdesc0 + (uint64_t)(k * (kTcN * 32 / 16)));
            tc_commit(&acc_full[as]);
            mbar_arrive(&acc_full[as]);
          }
        }
        if (ok && npairs) {  // the last MMA completes before the item's operands can change
          const uint32_t pl = pbase + npairs - 1;
          ok = mbar_wait(&acc_full[pl & 1u], (pl >> 1) & 1u, abort_flag);
        }
      }
      __syncwarp();
    } else if (warp < 4) {
      // ---------------------------------------------------------- B producers (per pair)
      for (uint32_t p = (uint32_t)(warp - 2); p < npairs && ok; p += 2) {
        const uint32_t pg = pbase + p;
        const uint32_t ja = jbase + 2 * p, jb = ja + 1;
        const uint32_t sa = ja & (uint32_t)(kTcParamSlots - 1), sb = jb & (uint32_t)(kTcParamSlots - 1);
        const uint32_t bs = pg & (uint32_t)(kTcBStages - 1);
        ok = mbar_wait(&p_full[sa], (ja >> 6) & 1u, abort_flag) && mbar_wait(&p_full[sb], (jb >> 6) & 1u, abort_flag);
        if (!ok) break;
        __half2 dg[8];
        float ra[4], rb[4];
        {
          const TcSlot& sl = slots[sa];
          float s5 = 0.f;
#pragma unroll
          for (int jb5 = 0; jb5 < 5; ++jb5)
            if ((lane >> jb5) & 1) s5 += sl.f[jb5];
          const float f5 = sl.f[5], f6 = sl.f[6], f7 = sl.f[7];
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            float cr = s5;
            if (r & 1) cr += f5;
            if (r & 2) cr += f6;
            if (r & 4) cr += f7;
            const float tq = rintf(cr);
            const float d1 = floorf(tq * (1.0f / 2048.0f));
            dg[r] = __floats2half2_rn(fmaf(-2048.0f, d1, tq), d1);
          }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const TcSlot& sl = slots[h ? sb : sa];
          float g5 = sl.et;
#pragma unroll
          for (int i = 0; i < 5; ++i)
            if ((lane >> i) & 1) g5 += sl.g[i];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            float v = g5;
            if (r & 1) v += sl.g[5];
            if (r & 2) v += sl.g[6];
            (h ? rb : ra)[r] = v + EY[lane + 32 * r];
          }
        }
        ok = mbar_wait(&b_empty[bs], ((pg >> 3) & 1u) ^ 1u, abort_flag);
        if (!ok) break;
        unsigned char* Bst = Bsm + bs * kTcN * 32;
#pragma unroll
        for (int r = 0; r < 8; ++r) *reinterpret_cast<__half2*>(Bst + kmaj_off(lane + 32 * r, 8)) = dg[r];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          Rs[bs * 128 + lane + 32 * r] = ra[r];
          Rs2[bs * 128 + lane + 32 * r] = rb[r];
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&b_full[bs]);
          mbar_arrive(&p_empty[sa]);
          mbar_arrive(&p_empty[sb]);
        }
      }
    } else {
      // ---------------------------------------------------------- epilogue (16-bit minima)
      const int q = warp & 3;
      const int cq = (warp - 4) >> 2;
      const int y = q * 32 + lane;
      const float inf = __int_as_float(0x7f800000);
      const uint32_t sp = (uint32_t)cq >> 1;  // pair parity = accumulator stage
      const uint32_t hh = (uint32_t)cq & 1u;  // column half: u bit 7
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + sp * (uint32_t)kTcN + hh * 128u;
      const uint32_t neg = (uint32_t)(((i_begin >> 1) + sp) & 1ull);
      uint32_t ct[8], cp[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        ct[c] = Tb.corr_t[neg][c];
        cp[c] = Tb.corr_p[neg][hh][c];
      }
      const float rbias = Tb.dmin - 8388608.0f;
      const float inv = I.inv_scale;
      float rmin = inf;
      auto pair_step = [&](uint32_t p) -> bool {
        const uint32_t pg = pbase + p;
        const uint32_t bs = pg & (uint32_t)(kTcBStages - 1);
        if (!mbar_wait(&acc_full[sp], (pg >> 1) & 1u, abort_flag)) return false;
        tc_fence_after();
        uint32_t r[4][16];
        QB_TC_LD16P(tbase, r[0]);
        QB_TC_LD16P(tbase + 32, r[1]);
        QB_TC_LD16P(tbase + 64, r[2]);
        QB_TC_LD16P(tbase + 96, r[3]);
        const float R1 = Rs[bs * 128 + y] + rbias;
        const float R2 = Rs2[bs * 128 + y] + rbias;
        tc_wait_ld();
#pragma unroll
        for (int c = 0; c < 4; ++c) reg_fence16(r[c]);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[sp]);
        uint32_t v1[8], v2[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const uint32_t* a = &r[c >> 1][(c & 1) * 8];
          v1[c] = uadd2(umin8(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]), ct[c]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
          v2[k] = uadd2(umin8(r[0][k], r[0][k + 8], r[1][k], r[1][k + 8], r[2][k], r[2][k + 8], r[3][k], r[3][k + 8]),
                        cp[k]);
        const uint32_t m1 = umin8(v1[0], v1[1], v1[2], v1[3], v1[4], v1[5], v1[6], v1[7]);
        const uint32_t m2 = umin8(v2[0], v2[1], v2[2], v2[3], v2[4], v2[5], v2[6], v2[7]);
        const float a1 = fminf(__uint_as_float(__byte_perm(m1, 0x4B000000u, 0x7610)),
                               __uint_as_float(__byte_perm(m1, 0x4B000000u, 0x7632)));
        const float a2 = fminf(__uint_as_float(__byte_perm(m2, 0x4B000000u, 0x7610)),
                               __uint_as_float(__byte_perm(m2, 0x4B000000u, 0x7632)));
        rmin = fmin3(rmin, a1 + R1, a2 + R2);
        return true;
      };
      uint32_t rec_left = 1u << (gl - 2);
      uint32_t Jrec = 0;
      for (uint32_t p = sp; p < npairs && ok; p += 4) {
        ok = pair_step(p) && pair_step(p + 2);
        if (!ok) break;
        rec_left -= 2;
        if (rec_left == 0) {
          const float wm = warp_min_f(rmin) * inv;
          if (lane == 0) {
            float* dst = rec + (((uint64_t)Jrec << 3) | ((uint64_t)hh << 2) | (uint64_t)q);
            if (wm >= 0.f)
              atomicMin(reinterpret_cast<int*>(dst), __float_as_int(wm));
            else
              atomicMax(reinterpret_cast<unsigned*>(dst), __float_as_uint(wm));
          }
          ++Jrec;
          rec_left = 1u << (gl - 2);
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
    tc_fence_after();
    jnext = jbase + (uint32_t)ntiles;
    if (*abort_flag) break;  // uniform: read after the barrier
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
  }
}

// the pair-form search kernel (one persistent CTA per SM); gamma = couplings of variable
// n-16 with u bits 0..7, in the units of the scaled W
inline int tc2_launch(const TcPlan& p, const float* gamma, float* rec, void* scratch, cudaStream_t st, int sms,
                      int* kernels) {
  unsigned* err = static_cast<unsigned*>(scratch);
  double* Wsc = reinterpret_cast<double*>(static_cast<char*>(scratch) + 16);
  const uint64_t groups = (p.tile_end - p.tile_begin) >> p.gl;
  if (!groups) return 0;
  uint64_t ctas = std::min<uint64_t>((uint64_t)sms, groups);
  uint64_t gpc = (groups + ctas - 1) / ctas;
  ctas = (groups + gpc - 1) / gpc;
  if ((gpc << p.gl) >> 32) return 1;
  Tc2Params Q{};
  TcParams& P = Q.P;
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
  P.stall = p.stall ? 1 : 0;
  for (int k = 0; k < 32; ++k) {
    float g = 0.f;
    for (int j = 0; j < 5; ++j)
      if ((k >> j) & 1) g += gamma[j];
    Q.g5[k] = g;
  }
  Q.whi[0] = gamma[5];
  Q.whi[1] = gamma[6];
  Q.whi[2] = gamma[7];
  if (p.u16) {
    P.dmin = p.dmin;
    tc2_u16_tables(gamma, p.dmin, &Q.tab);
  }
  const TcSmemLayout L = tc_layout(p.n);
  const size_t smem = std::max<size_t>(L.total + kTcBStages * 128 * 4, 120 * 1024) + 1024;
  auto* kern = p.u16 ? tc_pair_kernel<false> : tc_pair_fp32_kernel;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 4;
  kern<<<(unsigned)ctas, kTcThreads, smem, st>>>(Q);
  ++*kernels;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}
#endif

}  // namespace qb
