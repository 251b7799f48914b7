// qb_qbf1.cuh -- QB_F1 with the reference's int16 arithmetic (opt-in).
//
// The reference's QB_F1 (src/qubo_lib/solvers/qbf1.py:86-133, 179-249, 253-289) keeps every
// energy in int16: the suffix table BB, the Gray-permuted prefix table AA, the cross table
// ABBA = (Q_0B + Q_1A^T) X_B^T and the running suffix sums all wrap modulo 2^16.  Where the
// partial sums of Q leave the int16 range its answer is not the true minimum.  This form
// reproduces that answer: because every int16 operation is exact modulo 2^16, each value the
// reference holds equals the exact integer quantity reduced modulo 2^16 to [-32768, 32767],
// so the tables are built from exact integers and the search repeats the reference's
// per-thread order (256 x 64 threads, 16 suffix columns each: column = block * 1024 +
// 64 * c + thread; Gray prefix steps; strict < keeps the earliest step; lowest thread wins;
// the suffix is then the first minimum of that prefix's int16 row).
//
// B = 18 suffix bits, A = n - 18 prefix bits (19 <= n <= 46).
#pragma once
#include "qb_common.cuh"

namespace qb {

constexpr int kQbf1B = 18;
constexpr int kQbf1Threads = 16384;  // the reference's grid: 256 blocks x 64 threads
constexpr int kQbf1MaxN = 46;

__device__ __forceinline__ int wrap16(int v) { return (int)(short)v; }

// BB[s] and ABBA[k][s] (k < A) for every 18-bit suffix s (MSB-first: bit 17 - j of s is
// variable A + j).  Q: n x n int32 copy of the int16 matrix.
__global__ void qbf1w_tables_kernel(const int* __restrict__ Q, int n, int A, short* __restrict__ BB,
                                    short* __restrict__ ABBA) {
  extern __shared__ int q1_smem[];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) q1_smem[i] = Q[i];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= (1 << kQbf1B)) return;
  int e = 0;
  for (int j = 0; j < kQbf1B; ++j) {
    if (!((s >> (kQbf1B - 1 - j)) & 1)) continue;
    for (int l = 0; l < kQbf1B; ++l)
      if ((s >> (kQbf1B - 1 - l)) & 1) e += q1_smem[(A + j) * n + (A + l)];
  }
  BB[s] = (short)wrap16(e);
  for (int k = 0; k < A; ++k) {
    int c = 0;
    for (int j = 0; j < kQbf1B; ++j)
      if ((s >> (kQbf1B - 1 - j)) & 1) c += q1_smem[k * n + (A + j)] + q1_smem[(A + j) * n + k];
    ABBA[(size_t)k * (1 << kQbf1B) + s] = (short)wrap16(c);
  }
}

// AA[i] = int16 of E_pre(gray(i)) (prefix bit A-1-k is variable k)
__global__ void qbf1w_prefix_kernel(const int* __restrict__ Q, int n, int A, short* __restrict__ AA) {
  extern __shared__ int q1p_smem[];
  for (int i = threadIdx.x; i < A * A; i += blockDim.x) q1p_smem[i] = Q[(i / A) * n + (i % A)];
  __syncthreads();
  const uint64_t steps = 1ull << A;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < steps; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = gray64(i);
    int e = 0;
    for (int k = 0; k < A; ++k) {
      if (!((p >> (A - 1 - k)) & 1)) continue;
      for (int l = 0; l < A; ++l)
        if ((p >> (A - 1 - l)) & 1) e += q1p_smem[k * A + l];
    }
    AA[i] = (short)wrap16(e);
  }
}

// packed int16 pairs: per-halfword add (wraps modulo 2^16) and signed minimum
__device__ __forceinline__ uint32_t add16x2(uint32_t x, uint32_t y) {
  uint32_t r;
  asm("add.u16x2 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(y));
  return r;
}
__device__ __forceinline__ uint32_t min16x2(uint32_t x, uint32_t y) {
  uint32_t r;
  asm("min.s16x2 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(y));
  return r;
}
__device__ __forceinline__ uint32_t pack16(int lo, int hi) { return (uint32_t)(uint16_t)lo | ((uint32_t)(uint16_t)hi << 16); }

// shared memory of the search kernel: +ABBA and -ABBA rows of the block's 1024 columns,
// two columns per 32-bit word
inline size_t qbf1w_search_smem(int A) { return (size_t)2 * A * 512 * sizeof(uint32_t); }

// The search.  blockIdx.x = the reference block (64 threads, 1024 columns), blockIdx.y picks
// 4 consecutive chunks of Gray steps; thread = (chunk lane, reference thread t).  Thread t's
// 16 columns 64 c + t are held as 8 int16 pairs (c = 2 c2, 2 c2 + 1), so one step costs 8
// packed adds and 7 packed minima; a step that turns a prefix variable off adds the negated
// row.  Each thread reports (best int16 value, its step) of its chunk into key[tid] by a
// 64-bit atomic min, which keeps the smallest value and, among equal values, the earliest
// step.  Chunks of at least 32 steps are walked in aligned groups of 32 unrolled steps, in
// which the flipped prefix bit and its direction are constants.
__global__ void __launch_bounds__(256) qbf1w_search_kernel(int A, const short* __restrict__ BB,
                                                           const short* __restrict__ ABBA,
                                                           const short* __restrict__ AA, uint64_t chunk_len,
                                                           unsigned long long* __restrict__ key) {
  extern __shared__ uint32_t q1w_smem[];  // [2][A][8][64]: word (row k, pair c2, thread t)
  const int blk = blockIdx.x;
  for (int i = threadIdx.x; i < A * 512; i += blockDim.x) {
    const int k = i >> 9, c2 = (i >> 6) & 7, tt = i & 63;
    const size_t base = (size_t)k * (1 << kQbf1B) + (size_t)blk * 1024 + tt;
    const int lo = ABBA[base + 64 * (2 * c2)], hi = ABBA[base + 64 * (2 * c2 + 1)];
    q1w_smem[i] = pack16(lo, hi);
    q1w_smem[A * 512 + i] = pack16(-lo, -hi);
  }
  __syncthreads();
  const int t = threadIdx.x & 63;
  const uint64_t chunk = (uint64_t)blockIdx.y * 4 + (threadIdx.x >> 6);
  const uint64_t steps = 1ull << A;
  const uint64_t i0 = chunk * chunk_len;
  if (i0 >= steps) return;
  const uint64_t i1 = min(steps, i0 + chunk_len);
  const uint32_t* pos = q1w_smem + t;            // + row * 512 + c2 * 64
  const uint32_t* neg = q1w_smem + A * 512 + t;
  uint32_t E2[8];
  {
    const uint64_t p0 = gray64(i0);
    int E[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      int v = BB[blk * 1024 + 64 * c + t];
      for (int k = 0; k < A; ++k)
        if ((p0 >> (A - 1 - k)) & 1) v += ABBA[(size_t)k * (1 << kQbf1B) + (size_t)blk * 1024 + 64 * c + t];
      E[c] = v;
    }
#pragma unroll
    for (int c2 = 0; c2 < 8; ++c2) E2[c2] = pack16(E[2 * c2], E[2 * c2 + 1]);
  }
  // one step: E += the (signed) row, then int16 minimum of the 16 energies
  auto step_min = [&](const uint32_t* r) -> int {
#pragma unroll
    for (int c2 = 0; c2 < 8; ++c2) E2[c2] = add16x2(E2[c2], r[c2 * 64]);
    const uint32_t m2 = min16x2(min16x2(min16x2(E2[0], E2[1]), min16x2(E2[2], E2[3])),
                                min16x2(min16x2(E2[4], E2[5]), min16x2(E2[6], E2[7])));
    return min((int)(short)(m2 & 0xffffu), (int)m2 >> 16);
  };
  int m0;
  {
    const uint32_t m2 = min16x2(min16x2(min16x2(E2[0], E2[1]), min16x2(E2[2], E2[3])),
                                min16x2(min16x2(E2[4], E2[5]), min16x2(E2[6], E2[7])));
    m0 = min((int)(short)(m2 & 0xffffu), (int)m2 >> 16);
  }
  int best = wrap16((int)AA[i0] + m0);
  uint64_t bi = i0;
  if ((chunk_len & 31) == 0) {
    // aligned groups of 32 steps; the chunk's first step i0 is the initial state above
    for (uint64_t ig = i0; ig < i1; ig += 32) {
      uint32_t aa[16];  // AA[ig .. ig + 31], two per word
      {
        const uint4* src = reinterpret_cast<const uint4*>(AA + ig);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint4 w = __ldg(src + q);
          aa[4 * q] = w.x;
          aa[4 * q + 1] = w.y;
          aa[4 * q + 2] = w.z;
          aa[4 * q + 3] = w.w;
        }
      }
      const bool odd = (ig >> 5) & 1;  // bit 5 of the step index: direction of prefix bit 4
#pragma unroll
      for (int l = 0; l < 32; ++l) {
        const uint32_t* r;
        if (l == 0) {
          if (ig == i0) continue;
          const int kb = __ffsll((long long)ig) - 1;  // >= 5
          const bool on = (gray64(ig) >> kb) & 1;
          r = (on ? pos : neg) + (A - 1 - kb) * 512;
        } else {
          const int kb = ctz5(l);
          const bool on = kb < 4 ? !((l >> (kb + 1)) & 1) : !odd;
          r = (on ? pos : neg) + (A - 1 - kb) * 512;
        }
        const int m = step_min(r);
        const int a16 = (l & 1) ? (int)aa[l >> 1] >> 16 : (int)(short)(aa[l >> 1] & 0xffffu);
        const int tt = wrap16(a16 + m);
        if (tt < best) {  // strict: the earliest step keeps a tie
          best = tt;
          bi = ig + (uint64_t)l;
        }
      }
    }
  } else {
    for (uint64_t i = i0 + 1; i < i1; ++i) {
      const int kb = __ffsll((long long)i) - 1;
      const bool on = (gray64(i) >> kb) & 1;
      const int m = step_min((on ? pos : neg) + (A - 1 - kb) * 512);
      const int tt = wrap16((int)AA[i] + m);
      if (tt < best) {
        best = tt;
        bi = i;
      }
    }
  }
  const int tid = blk * 64 + t;
  atomicMin(key + tid, ((unsigned long long)(best + 32768) << 40) | (unsigned long long)bi);
}

// int16 row of prefix p: first s with the smallest wrap16(BB[s] + sum of ABBA rows of p)
__global__ void qbf1w_row_kernel(int A, const short* __restrict__ BB, const short* __restrict__ ABBA, uint64_t p,
                                 unsigned long long* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= (1 << kQbf1B)) return;
  int v = BB[s];
  for (int k = 0; k < A; ++k)
    if ((p >> (A - 1 - k)) & 1) v += ABBA[(size_t)k * (1 << kQbf1B) + s];
  v = wrap16(v);
  atomicMin(out, ((unsigned long long)(v + 32768) << 32) | (unsigned long long)s);
}

}  // namespace qb
