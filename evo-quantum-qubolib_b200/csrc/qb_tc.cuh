// qb_tc.cuh -- tensor-core (tcgen05) form of the exhaustive search.
//
// The state X splits into three groups of bits:
//   t = X >> 15          (n_T = n - 15 bits; one tile per value, visited in Gray order)
//   y = (X >> 8) & 127   (7 bits: the 128 rows of an MMA tile, one TMEM lane each)
//   u = X & 255          (8 bits: the 256 columns of an MMA tile)
// and the energy as
//   E(t, y, u) = R_t(y) + C_t(u) + y^T V u
//   R_t(y) = E_T(t) + E_Y(y) + (t^T W_TY) y       (per row, per tile: added after the row min)
//   C_t(u) = E_U(u) + (t^T W_TU) u                (per column, per tile: folded into the MMA)
//   V      = couplings between the y and u variables (fixed)
// One tcgen05.mma (kind::f16, M=128, N=256, K=16, fp32 accumulators in TMEM) computes
// D[y][u] = y^T V u + C_t(u) for all 32768 states of a tile:
//   A[y][2i+d] = y_i * s_d         B[u][2i+d] = digit_d((V u)_i)      i < 7, d in {0,1}
//   A[y][14+d] = s_d               B[u][14+d] = digit_d(C_t(u))
// with digits v = d0 + s_1 d1 (integer Q: s = (1, 2048), d0 in [0, 2048), exact in fp16;
// float Q: s = (1, 1), d0 + d1 = fp16 hi/lo split of v).  A is constant; per tile only
// the two C columns of B change.  The epilogue reads the accumulators (tcgen05.ld), takes
// row minima with 3-input fp32 min and adds R_t(y).
//
// Measured on B200 (sm_100a): back to back, an M=128 N=256 K=16 MMA takes 128 cycles; a
// one-way mbarrier signal between two warps (arrive -> try_wait returns) about 270 cycles.
// A tile's accumulator stage is busy for MMA + commit signal + epilogue loads + release
// signal + the MMA thread's reaction, so with the two 256-column stages the TMEM holds,
// throughput is set by that round trip; smaller N does not shorten it, so tiles use the
// largest N.  The fp32 min pipe (about 128 values per clock per SM, shared with fp32 adds)
// bounds the epilogue at half the MMA rate.
//
// Roles (one persistent CTA per SM, 640 threads):
//   warp 0      tile walk: 32 tiles per step, one per lane.  t = (t_hi, t_lo) with t_lo the
//               5 low bits: per-CTA tables give the t_lo parts, t_hi (constant over an
//               aligned run of 32 Gray tiles) is Gray-updated once per run; each lane
//               publishes E_T(t), t^T W_TY and t^T W_TU of its tile
//   warp 1      TMEM allocation and MMA issue (one elected thread)
//   warps 2-3   B producers, alternate tiles: C_t(u) digits into the B stage (generic
//               stores + proxy fence) and the 128 row terms R_t(y) beside it
//   warps 4-19  epilogue: warp w reads TMEM lanes 32*(w%4)..+31; warps 4-11 take the even
//               tiles, 12-19 the odd ones, each a 128-column half in two rounds; a warp
//               releases the accumulator stage as soon as its loads have landed, then
//               reduces (so the 4 warps of a scheduler alternate between the two stages)
// Pipelines on mbarriers: 64 tile-parameter slots (walk -> producers), 8 B stages
// (producers -> MMA and epilogue), 2 accumulator stages.  One tcgen05.commit per MMA
// (accumulator full); the MMA thread frees tile j-2's B stage when the epilogue's release
// of tile j-2 lets it issue MMA j.
// Every wait is bounded (%globaltimer): on timeout the waiting role raises an error flag,
// the CTA drains and frees TMEM, and the host reports QB_ETIMEOUT.
//
// Records: per block of 2^gl tiles (gl >= 5), 8 records of 32 rows x 128 columns x 2^gl
// tiles, each the atomic minimum of the two warps (even and odd tiles) that cover it.
//
// Integer Q with sum|Q| <= 2^22 is exact (all partial sums stay below 2^24 in fp32).
// Otherwise every value is within tc_error_bound() of the exact energy.
#pragma once
#include <cuda_fp16.h>

#include "qb_common.cuh"

namespace qb {

constexpr double kTcIntMaxAbsSum = 4194304.0;  // 2^22
constexpr int kTcThreads = 640;
constexpr int kTcStages = 2;                   // TMEM accumulator stages (2 x 256 columns)
constexpr int kTcEpiWarps = 16;
constexpr int kTcParamSlots = 64;
constexpr int kTcBStages = 8;
constexpr int kTcN = 256;                      // MMA N = tile columns
constexpr uint64_t kTcWaitLimitNs = 2000000000ull;  // 2 s per wait
static_assert(kTcStages == 2 && kTcParamSlots == 64 && kTcBStages == 8, "the roles' slot / stage / parity arithmetic");

struct TcPlan {
  int n = 0, nt = 0, gl = 0;
  bool is_int = false;
  bool exact = false;      // integer digits (exact arithmetic)
  double scale = 1.0;      // power of two applied to W on the device (float digits)
  double eps = 0.0;        // per-state error bound, unscaled units
  uint64_t tile_begin = 0, tile_end = 0;  // this shard's Gray tile indices
  uint64_t rec_begin = 0, rec_count = 0, states = 0;
  bool stall = false;      // test hook: the tile walk publishes nothing (waits expire)
  bool pair = false;       // two states per accumulator (tc_pair_kernel, qb_tc2.cuh)
  float gamma[8] = {0};    // pair form: scaled W[n-16][n-1-j], j < 8
  bool u16 = false;        // 16-bit epilogue (tc_u16_eligible)
  float dmin = 0.f;        // 16-bit epilogue: lower bound of every accumulator value D
};

// The 16-bit epilogue.  An accumulator holds D(y, u) = y^T V u + C_t(u), a sum of couplings
// W_ab with at least one of a, b among the u variables, so Dmin <= D <= Dmax with Dmin (Dmax)
// the sum of the negative (positive) such couplings.  When Dmax - Dmin < 2^16, every
// coupling row (V u)_i of a y variable stays within +-2048 (one exact fp16 digit) and integer
// Q is on the exact path, the MMA computes F = D + 2^23 - Dmin exactly (the column term
// carries the offset in three fp16 digits: 1, 2048 and 32768 times d0 < 2048, d1 < 16,
// d2 = 256 or 257): F is an integer in [2^23, 2^24), so the low 16 bits of its fp32 pattern
// are exactly D - Dmin.  The epilogue then loads the accumulators two per register
// (tcgen05.ld .pack::16b keeps the low 16 bits of each column) and takes unsigned 16-bit
// minima (min.u16x2, two states per full-rate ALU instruction, against one 3-input fp32 min
// per two states at half rate), and holds 128 columns in 64 registers, so each epilogue
// warp loads its whole half-stage at once and releases it before any arithmetic.
// W is the n x n FP64 matrix of the problem (unscaled: the exact path has scale 1).
// span (optional) receives Dmax - Dmin.
inline bool tc_u16_eligible(int n, const double* W, float* dmin, double* span = nullptr) {
  if (n < 20) return false;
  double lo = 0.0, hi = 0.0;
  auto add = [&](double w) {
    if (w < 0) lo += w;
    else hi += w;
  };
  for (int i = 0; i < 7; ++i) {  // y variable n-9-i: its coupling row with the u variables
    double rp = 0.0, rn = 0.0;
    for (int j = 0; j < 8; ++j) {
      const double w = W[(size_t)(n - 9 - i) * n + (n - 1 - j)];
      if (w < 0) rn -= w;
      else rp += w;
      add(w);
    }
    if (rp > 2048.0 || rn > 2048.0) return false;
  }
  for (int j = 0; j < 8; ++j) {
    const int a = n - 1 - j;
    add(W[(size_t)a * n + a]);                                          // u diagonal
    for (int j2 = 0; j2 < j; ++j2) add(W[(size_t)a * n + (n - 1 - j2)]);  // u-u couplings
    for (int t = 0; t < n - 15; ++t) add(W[(size_t)t * n + a]);          // t-u couplings
  }
  if (hi - lo > 65535.0) return false;
  *dmin = (float)lo;
  if (span) *span = hi - lo;
  return true;
}

// one CTA work item: a contiguous run of whole record blocks of one problem
struct TcItem {
  const double* W;     // scaled W of the problem, n*n
  float* rec;          // record 0 of the item's first block
  uint64_t i_begin;    // Gray index of the item's first tile (a multiple of 2^gl)
  uint64_t ntiles;     // tiles in the item (a multiple of 2^gl, below 2^31)
  int n, gl, exact;
  float inv_scale;     // 1 / scale of W
};

struct TcParams {
  int n, nt, gl;            // one problem (items == nullptr) ...
  int stall;
  int exact;
  float inv_scale;
  const double* W;          // scaled W, n*n
  uint64_t tile_begin;      // shard start (aligned to 2^gl)
  uint64_t groups;          // record blocks (2^gl tiles each) in this shard
  uint64_t groups_per_cta;  // contiguous blocks per CTA (last CTA may have fewer)
  float* rec;               // rec[0] = record (tile_begin >> gl) << 3
  const TcItem* items;      // ... or a list of work items: CTA b runs items
  const uint32_t* item_first;  //     [item_first[b], item_first[b + 1])
  int n_max;                // largest n among the items (shared-memory layout)
  unsigned* err;            // error word
  float dmin;               // 16-bit epilogue: lower bound of the accumulator values
  float k0;                 // 16-bit epilogue: 2^23 - dmin, added to the column term
};

inline bool tc_supported(int n) { return n >= 20 && n <= kMaxN; }

// per-state error bound of the float-digit path (unscaled units)
inline double tc_error_bound(double abs_sum) { return 256.0 * abs_sum * 5.9604644775390625e-08 + 1e-300; }

// default record granularity: runs of 32 tiles, at most 2^21 records (8 per block of 2^gl tiles)
// largest record block: 2^28 tiles, so that a record's gl + 12 free bits (2^gl tiles x 128
// rows x 256 columns of one block quarter and half) stay within the exact re-walk's 40
constexpr int kTcMaxGl = 28;
inline int tc_default_gl(int n) { return std::min(kTcMaxGl, std::max(5, n - 15 - 18)); }

// gl: log2 tiles per record block (0 = tc_default_gl); 5 <= gl <= min(n - 15, kTcMaxGl)
inline void tc_plan(int n, bool is_int, double abs_sum, int shard_idx, int shard_cnt, TcPlan* p, int gl = 0) {
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
  p->gl = gl >= 5 && gl <= std::min(p->nt, kTcMaxGl) ? gl : tc_default_gl(n);
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
// try_wait with a suspend-time hint of 40 ns: the MMA issuer's wait for a released
// accumulator stage, where waking promptly matters more than the few extra polls (measured on
// the pair kernel: 2.49 -> 2.40 ms per 2^36 states)
__device__ __forceinline__ bool mbar_try_wait_short(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity), "r"(40u)
      : "memory");
  return ok != 0;
}
// bounded wait with the short hint; the abort flag and the clock are read every 256 polls
__device__ __forceinline__ bool mbar_wait_short(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait_short(b, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait_short(b, parity)) return true;
    if ((it & 255u) == 0) {
      if (*abort_flag) return false;
      if (globaltimer_ns() - t0 > kTcWaitLimitNs) return false;
    }
  }
}
// bounded wait: false on timeout (or when another role already gave up).  try_wait suspends
// the warp in hardware until the phase completes or a system-dependent time limit runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    if (mbar_try_wait(b, parity)) return true;
    if (*abort_flag) return false;
    if (globaltimer_ns() - t0 > kTcWaitLimitNs) return false;
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
constexpr uint32_t kTcIdesc =
    (1u << 4) | (0u << 7) | (0u << 10) | (((uint32_t)kTcN >> 3) << 17) | ((128u >> 4) << 24);

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

// 32 columns as 16 registers, two columns per register (the low 16 bits of each)
#define QB_TC_LD16P(taddr, r)                                                                                  \
  asm volatile(                                                                                                \
      "tcgen05.ld.sync.aligned.32x32b.x16.pack::16b.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, " \
      "[%16];"                                                                                                 \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),        \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])   \
      : "r"(taddr))

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

// tcgen05.ld writes its registers asynchronously; only tcgen05.wait::ld makes them valid.
// Passing each register through an empty volatile asm after the wait gives every later use
// a data dependence on a statement ordered after the wait, so the compiler cannot hoist a
// use above it.
__device__ __forceinline__ void reg_fence32(uint32_t* r) {
#pragma unroll
  for (int i = 0; i < 32; ++i) asm volatile("" : "+r"(r[i]));
}

__device__ __forceinline__ void reg_fence16(uint32_t* r) {
#pragma unroll
  for (int i = 0; i < 16; ++i) asm volatile("" : "+r"(r[i]));
}

__device__ __forceinline__ uint32_t umin2(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// unsigned 16-bit minimum over 4 x 16 registers of packed pairs, as an int
__device__ __forceinline__ uint32_t umin64(uint32_t* a, uint32_t* b, uint32_t* c, uint32_t* d) {
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = umin2(umin2(a[i], b[i]), umin2(c[i], d[i]));
#pragma unroll
  for (int w = 8; w >= 1; w >>= 1)
#pragma unroll
    for (int i = 0; i < w; ++i) a[i] = umin2(a[i], a[i + w]);
  return min(a[0] & 0xffffu, a[0] >> 16);
}

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

// per-tile parameters published by the tile walk
struct TcSlot {
  float f[8];  // f_j = (t^T W_TU)_j: C_t(u) = E_U(u) + sum_j f_j u_j
  float g[8];  // g_i = (t^T W_TY)_i, i < 7
  float et;    // E_T(t)
  float pad[3];
};

struct TcSmemLayout {
  uint32_t a_off, b_off, bar_off, slot_off, eu_off, ey_off, rs_off, misc_off, lo_off, w_off, total;
};

__host__ __device__ inline TcSmemLayout tc_layout(int n) {
  TcSmemLayout L;
  uint32_t o = 0;
  L.a_off = o;
  o += 128 * 32;  // A: 128 rows x 16 f16
  L.b_off = o;
  o += kTcBStages * kTcN * 32;
  L.bar_off = o;
  o += (2 * kTcParamSlots + 2 * kTcBStages + 2 * kTcStages) * 8;
  L.slot_off = o;
  o += kTcParamSlots * sizeof(TcSlot);
  L.eu_off = o;
  o += kTcN * 4;
  L.ey_off = o;
  o += 128 * 4;  // E_Y(y) per row
  L.rs_off = o;
  o += kTcBStages * 128 * 4;  // R_t(y) per B stage and row, written with the stage
  L.misc_off = o;
  o += 64;
  L.lo_off = o;
  o += 32 * 16 * 8;  // per t_lo pattern: f (7), g (7), E_lo, pad -- fp64
  L.w_off = o;
  o += (uint32_t)n * n * 8;
  L.total = o;
  return L;
}

// kItems = false: one problem (one work item per CTA, compiled without the item loop's
// bookkeeping); kItems = true: the CTA's list of work items.  kU16 (one problem only): the
// 16-bit epilogue (tc_u16_eligible).
template <bool kItems, bool kU16 = false>
__global__ void __launch_bounds__(kTcThreads, 1) tc_pass1_kernel(TcParams P) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
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
  float* Rs = reinterpret_cast<float*>(tc_smem + L.rs_off);
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

  // ---------------------------------------------------------------- one-time set-up
  if (tid == 0) {
    for (int s = 0; s < kTcParamSlots; ++s) {
      mbar_init(&p_full[s], 1);
      mbar_init(&p_empty[s], 1);  // the tile's producer warp (the only reader of the slot)
    }
    for (int s = 0; s < kTcBStages; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
    }
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&acc_full[s], 2);  // the MMA's commit and the MMA thread (after it saw the B stage full)
      mbar_init(&acc_empty[s], kTcEpiWarps / 2);  // the 8 warps that read this stage
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // Every role walks the CTA's tiles in the same order; barrier slots, stages and phases
  // follow the CTA-wide tile counter jbase + local index across items.  Between items all
  // roles meet at a CTA barrier with the pipelines empty (the MMA thread waits for its last
  // MMA), so the per-item tables and B operand columns can be rewritten.
  uint32_t jbase = 0;
  for (uint32_t it = it_lo; it < (kItems ? it_hi : 1u); ++it) {
    const TcItem I = kItems ? P.items[it] : one;
    const int n = I.n, nt = n - 15, gl = I.gl, exact = I.exact;
    const float inv_scale = I.inv_scale;
    const uint64_t i_begin = I.i_begin, ntiles = I.ntiles;
    float* rec = I.rec;
    const uint64_t t0 = gray64(i_begin);
    const float s1 = exact ? 2048.0f : 1.0f;
    // variables: t bit k <-> n-16-k, y bit i <-> n-9-i, u bit j <-> n-1-j

    // ------------------------------------------------------------ per-item set-up
    if (kItems && tid == 0) {  // read by the epilogue at record flushes (keeps them out of registers)
      *reinterpret_cast<float**>(tc_smem + L.misc_off + 16) = rec;
      *reinterpret_cast<float*>(tc_smem + L.misc_off + 24) = inv_scale;
    }
    for (int i = tid; i < n * n; i += kTcThreads) Ws[i] = I.W[i];
    // the item's records start at +inf (the epilogue folds into them with atomic minima)
    for (uint64_t r = (uint64_t)tid; r < ((ntiles >> gl) << 3); r += kTcThreads) rec[r] = __int_as_float(0x7f800000);
    __syncthreads();
    // A operand (constant)
    for (int e = tid; e < 128 * 16; e += kTcThreads) {
      int y = e >> 4, k = e & 15;
      float v;
      if (kU16)  // A[y][i] = y_i (i < 7); the column term's digit weights 1, 2048, 32768
        v = k < 7 ? (float)((y >> k) & 1) : (k == 7 ? 1.0f : (k == 8 ? 2048.0f : (k == 9 ? 32768.0f : 0.0f)));
      else if (k < 14)
        v = ((y >> (k >> 1)) & 1) ? ((k & 1) ? s1 : 1.0f) : 0.0f;
      else
        v = (k & 1) ? s1 : 1.0f;
      *reinterpret_cast<__half*>(Asm + kmaj_off(y, k)) = __float2half_rn(v);
    }
    // B operand, coupling columns (same in every stage)
    if (kU16) {
      // one exact fp16 value per coupling row (|(V u)_i| <= 2048), zeros in the unused K slots
      for (int e = tid; e < kTcN * 16; e += kTcThreads) {
        const int u = e >> 4, k = e & 15;
        if (k >= 7 && k < 10) continue;  // the column term's digits, written per tile
        double v = 0.0;
        if (k < 7) {
          const double* row = Ws + (n - 9 - k) * n;
          for (int j = 0; j < 8; ++j)
            if ((u >> j) & 1) v += row[n - 1 - j];
        }
        const __half hv = __float2half_rn((float)v);
        for (int s = 0; s < kTcBStages; ++s) *reinterpret_cast<__half*>(Bsm + s * kTcN * 32 + kmaj_off(u, k)) = hv;
      }
    } else {
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
    }
    // E_U(u)
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
    // E_Y(y)
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
    // t_lo tables: LO[p*16 + j] = (p^T W_TlU)_j (j < 8), LO[p*16 + 8 + i] = (p^T W_TlY)_i
    // (i < 7), LO[p*16 + 15] = energy of the t_lo bits p
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
    fence_proxy_async();  // A / B stores (generic proxy) -> visible to tcgen05.mma
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    bool ok = true;
    if (warp == 0 && P.stall) {
      // test hook (QB_FLAG_TEST_STALL): no tile parameters are published, so every other
      // role's bounded wait runs out; the CTA drains and the host reports QB_ETIMEOUT
    } else if (warp == 0) {
      // ---------------------------------------------------------- tile walk
      // Every lane keeps the t_hi state (fp64, lane-redundant): fh = t_hi^T W_ThU, gh =
      // t_hi^T W_ThY, eh = E(t_hi), c_k = coupling of t_lo bit k with t_hi; lane l also
      // keeps the fields of t_hi bits l and l + 32 from the other t_hi bits.
      const int nh = nt - 5;  // t_hi bits: t bit 5 + m <-> variable n-21-m
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
        if (j0 > 0) {  // t_hi changes by one bit between aligned runs of 32 Gray tiles
          const int kb = __ffsll((long long)i0) - 1;  // >= 5
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
        // this lane's tile
        const uint64_t j = j0 + (uint64_t)lane;
        const int tl = (int)(gray64(i0 + (uint64_t)lane) & 31ull);
        const double* lo = LO + tl * 16;
        double et = eh + lo[15];
#pragma unroll
        for (int k = 0; k < 5; ++k)
          if ((tl >> k) & 1) et += c[k];
        const uint64_t jg = jbase + j;
        const int s = (int)(jg % kTcParamSlots);
        ok = mbar_wait(&p_empty[s], (uint32_t)(((jg / kTcParamSlots) & 1) ^ 1), abort_flag);
        ok = __all_sync(0xffffffffu, ok);  // keep the warp converged for the next shuffle
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
      // ---------------------------------------------------------- MMA issue
      // Unrolled over the 8 B stages: the CTA-wide tile counter starts every item at a
      // multiple of 8 and an item has a multiple of 32 tiles, so the stage of each unrolled
      // step and its accumulator-barrier parity are constants.  The issuing thread shares its
      // scheduler with four epilogue warps; a short per-tile instruction chain keeps MMA j + 2
      // close behind the release of tile j.
      if (lane == 0) {
        const uint64_t adesc = umma_desc(smem_u32(Asm), 128, 256);
        const uint64_t bdesc0 = umma_desc(smem_u32(Bsm), 128, 256);
        const uint32_t nt32 = (uint32_t)ntiles;
        for (uint32_t jl0 = 0; jl0 < nt32 && ok; jl0 += kTcBStages) {
          const uint32_t j0 = jbase + jl0;
          const uint32_t pb = (j0 >> 3) & 1u;  // b_full parity of the 8 tiles
#pragma unroll
          for (int k = 0; k < kTcBStages; ++k) {
            const uint32_t as = (uint32_t)k & 1u;
            // tile j0 + k: its B stage is full and tile j0 + k - 2 has left accumulator stage as
            ok = mbar_wait(&b_full[k], pb, abort_flag) &&
                 mbar_wait_short(&acc_empty[as], (((uint32_t)k >> 1) & 1u) ^ 1u, abort_flag);
            if (!ok) break;
            tc_fence_after();
            // every epilogue warp has released tile j-2 (it read that tile's row terms before its
            // release, and MMA j-2 completed before the tile could be read): its B stage is free
            if (j0 + (uint32_t)k >= (uint32_t)kTcStages) mbar_arrive(&b_empty[(k + kTcBStages - kTcStages) % kTcBStages]);
            // B stage k starts k * 8 KB after stage 0 (descriptor address field in 16-byte units)
            tc_mma(tmem + as * (uint32_t)kTcN, adesc, bdesc0 + (uint64_t)(k * (kTcN * 32 / 16)));
            tc_commit(&acc_full[as]);  // one commit per MMA
            // the second arrival on acc_full: this thread has seen the B stage full, so the
            // epilogue's acquire of acc_full also orders the row terms written with the stage
            mbar_arrive(&acc_full[as]);
          }
        }
        if (ok && nt32) {  // the last MMA completes before the item's operands can change
          const uint32_t j = jbase + nt32 - 1;
          mbar_wait(&acc_full[j & 1u], (j >> 1) & 1u, abort_flag);
        }
      }
      __syncwarp();
    } else if (warp < 4) {
      // ---------------------------------------------------------- B producers (C_t columns)
      // warp 2 + (j & 1) fills tile j: rows u = lane + 32 r, r < 8 (u bits 5..7 = r)
      // and the row terms R_t(y) = E_T(t) + E_Y(y) + (t^T W_TY) y of rows y = lane + 32 r, r < 4
      const uint32_t nt32 = (uint32_t)ntiles;
      for (uint32_t jl = (uint32_t)(warp - 2); jl < nt32 && ok; jl += 2) {
        const uint32_t j = jbase + jl;  // CTA-wide tile counter: slots, stages and phases
        const uint32_t s = j & (uint32_t)(kTcParamSlots - 1);
        const uint32_t bs = j & (uint32_t)(kTcBStages - 1);
        ok = mbar_wait(&p_full[s], (j >> 6) & 1u, abort_flag);
        if (!ok) break;
        __half2 dg[8];
        __half dl[8];  // 16-bit epilogue: the column term's lowest digit
        float rr[4];
        {
          const TcSlot& sl = slots[s];
          float s5 = 0.f;
#pragma unroll
          for (int jb = 0; jb < 5; ++jb)
            if ((lane >> jb) & 1) s5 += sl.f[jb];
          const float f5 = sl.f[5], f6 = sl.f[6], f7 = sl.f[7];
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            float cr = s5;
            if (r & 1) cr += f5;
            if (r & 2) cr += f6;
            if (r & 4) cr += f7;
            if (kU16) {
              // C + 2^23 - Dmin, an integer in [2^23, 2^24): digits d0 < 2048, d1 < 16, d2
              const float c = EU[lane + 32 * r] + cr + P.k0;
              const float d2 = floorf(c * (1.0f / 32768.0f));
              const float rem = c - 32768.0f * d2;
              const float d1 = floorf(rem * (1.0f / 2048.0f));
              dl[r] = __float2half_rn(rem - 2048.0f * d1);
              dg[r] = __halves2half2(__float2half_rn(d1), __float2half_rn(d2));
            } else {
              dg[r] = digits(EU[lane + 32 * r] + cr, exact);
            }
          }
          float g5 = sl.et;
#pragma unroll
          for (int i = 0; i < 5; ++i)
            if ((lane >> i) & 1) g5 += sl.g[i];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            float v = g5;
            if (r & 1) v += sl.g[5];
            if (r & 2) v += sl.g[6];
            rr[r] = v + EY[lane + 32 * r];
          }
        }
        ok = mbar_wait(&b_empty[bs], ((j >> 3) & 1u) ^ 1u, abort_flag);
        if (!ok) break;
        unsigned char* Bst = Bsm + bs * kTcN * 32;
        if (kU16) {
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            *reinterpret_cast<__half*>(Bst + kmaj_off(lane + 32 * r, 7)) = dl[r];
            *reinterpret_cast<__half2*>(Bst + kmaj_off(lane + 32 * r, 8)) = dg[r];
          }
        } else {
#pragma unroll
          for (int r = 0; r < 8; ++r) *reinterpret_cast<__half2*>(Bst + kmaj_off(lane + 32 * r, 14)) = dg[r];
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) Rs[bs * 128 + lane + 32 * r] = rr[r];
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&b_full[bs]);
          mbar_arrive(&p_empty[s]);
        }
      }
    } else {
      // ---------------------------------------------------------- epilogue
      const int q = warp & 3;           // TMEM lane quarter (warp id % 4)
      const int cq = (warp - 4) >> 2;   // 0..3: (tile parity, column half) below
      const int y = q * 32 + lane;
      const float inv = inv_scale;
      const float inf = __int_as_float(0x7f800000);
      float rmin = inf;
      // warps 4-11 take the even tiles (accumulator stage 0), warps 12-19 the odd ones (stage 1),
      // so the four warps sharing a scheduler work on different tiles and one stage's waits
      // overlap the other stage's minima; each reads 128 columns (column half hh) in two
      // 64-column rounds and releases the stage once the second round has landed
      const uint32_t sp = (uint32_t)cq >> 1;   // tile parity = accumulator stage
      const uint32_t hh = (uint32_t)cq & 1u;   // column half
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + sp * (uint32_t)kTcN + hh * 128u;
      // 32-bit loop state (a CTA walks fewer than 2^32 tiles); records every 2^gl tiles (2^(gl-1)
      // of this warp's parity), counted down from the CTA's first block (aligned to 2^gl)
      const uint32_t nt32 = (uint32_t)ntiles;
      uint32_t rec_left = 1u << (gl - 1);
      uint32_t Jrec = 0;  // records of this item (fewer than 2^31)
      for (uint32_t jl = sp; jl < nt32 && ok; jl += 2) {
        const uint32_t j = jbase + jl;  // CTA-wide tile counter (jbase is even)
        const uint32_t bs = j & (uint32_t)(kTcBStages - 1);
        // acc_full completes after the MMA thread saw tile j's B stage full, so its row terms
        // are visible; they stay until this warp has released tile j (the producer rewrites the
        // stage for tile j + 8 only after MMA j + 2, which waits for that release)
        ok = mbar_wait(&acc_full[sp], (j >> 1) & 1u, abort_flag);
        if (!ok) break;
        const float R = Rs[bs * 128 + y];
        tc_fence_after();
        if (kU16) {
          // the warp's 128 columns at once, two per register; released before the minima
          uint32_t r0[16], r1[16], r2[16], r3[16];
          QB_TC_LD16P(tbase, r0);
          QB_TC_LD16P(tbase + 32, r1);
          QB_TC_LD16P(tbase + 64, r2);
          QB_TC_LD16P(tbase + 96, r3);
          tc_wait_ld();
          reg_fence16(r0);
          reg_fence16(r1);
          reg_fence16(r2);
          reg_fence16(r3);
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[sp]);
          // min over the row of D - Dmin, then E = that + Dmin + R (all exact integers in fp32)
          rmin = fminf(rmin, (float)umin64(r0, r1, r2, r3) + (R + P.dmin));
        } else {
        uint32_t ra[32], rb[32];
        QB_TC_LD32(tbase, ra);
        QB_TC_LD32(tbase + 32, rb);
        tc_wait_ld();
        reg_fence32(ra);
        reg_fence32(rb);
        const float m1 = fminf(min32(ra), min32(rb));
        QB_TC_LD32(tbase + 64, ra);
        QB_TC_LD32(tbase + 96, rb);
        tc_wait_ld();
        reg_fence32(ra);
        reg_fence32(rb);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[sp]);  // the stage is free once the data is in registers
        const float m = fminf(m1, fminf(min32(ra), min32(rb)));
        rmin = fminf(rmin, m + R);
        }
        if (--rec_left == 0) {
          // both parities' warps of (column half, lane quarter) fold into one record
          // the multi-item kernel re-reads the item's record base and scale from shared memory
          const float sc = kItems ? *reinterpret_cast<volatile float*>(tc_smem + L.misc_off + 24) : inv;
          float* rb0 = kItems ? *reinterpret_cast<float* volatile*>(tc_smem + L.misc_off + 16) : rec;
          const float wm = warp_min_f(rmin) * sc;
          if (lane == 0) {
            float* dst = rb0 + (((uint64_t)Jrec << 3) | ((uint64_t)hh << 2) | (uint64_t)q);
            if (wm >= 0.f)
              atomicMin(reinterpret_cast<int*>(dst), __float_as_int(wm));
            else
              atomicMax(reinterpret_cast<unsigned*>(dst), __float_as_uint(wm));
          }
          ++Jrec;
          rec_left = 1u << (gl - 1);
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
    if (!kItems) break;
    jbase += (uint32_t)ntiles;
    if (*abort_flag) break;  // uniform: read after the barrier
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

// clears the error word and writes the scaled W into the scratch buffer
inline int tc_prepare(const TcPlan& p, ProblemDev pd, void* scratch, cudaStream_t st, int* kernels) {
  unsigned* err = static_cast<unsigned*>(scratch);
  double* Wsc = reinterpret_cast<double*>(static_cast<char*>(scratch) + 16);
  if (cudaMemsetAsync(err, 0, 16, st) != cudaSuccess) return 4;
  tc_scale_w_kernel<<<8, 256, 0, st>>>(pd.W, Wsc, p.n * p.n, p.scale);
  ++*kernels;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

// the search kernel itself (one persistent CTA per SM)
inline int tc_launch(const TcPlan& p, float* rec, void* scratch, cudaStream_t st, int sms, int* kernels) {
  unsigned* err = static_cast<unsigned*>(scratch);
  double* Wsc = reinterpret_cast<double*>(static_cast<char*>(scratch) + 16);
  const uint64_t groups = (p.tile_end - p.tile_begin) >> p.gl;
  if (!groups) return 0;
  uint64_t ctas = std::min<uint64_t>((uint64_t)sms, groups);
  uint64_t gpc = (groups + ctas - 1) / ctas;
  ctas = (groups + gpc - 1) / gpc;
  if ((gpc << p.gl) >> 32) return 1;  // a CTA's tile count must fit 32 bits (n <= 54 on 148 SMs)
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
  P.stall = p.stall ? 1 : 0;
  P.dmin = p.dmin;
  P.k0 = 8388608.0f - p.dmin;
  const TcSmemLayout L = tc_layout(p.n);
  // at least 120 KB so that one CTA (and one 512-column TMEM allocation) runs per SM
  const size_t smem = std::max<size_t>(L.total, 120 * 1024) + 1024;
  auto kern = p.u16 ? tc_pass1_kernel<false, true> : tc_pass1_kernel<false, false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 4;
  kern<<<(unsigned)ctas, kTcThreads, smem, st>>>(P);
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
