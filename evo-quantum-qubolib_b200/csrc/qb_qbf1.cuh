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

// The search.  blockIdx.x = the reference block (64 threads, 1024 columns), blockIdx.y picks
// 4 consecutive chunks of Gray steps; thread = (chunk lane, reference thread t).  Each thread
// reports (best int16 value, its step) of its chunk into key[tid] by a 64-bit atomic min,
// which keeps the smallest value and, among equal values, the earliest step.
__global__ void __launch_bounds__(256) qbf1w_search_kernel(int A, const short* __restrict__ BB,
                                                           const short* __restrict__ ABBA,
                                                           const short* __restrict__ AA, uint64_t chunk_len,
                                                           unsigned long long* __restrict__ key) {
  extern __shared__ short q1s_smem[];  // [A][1024]: this block's columns of ABBA
  const int blk = blockIdx.x;
  for (int i = threadIdx.x; i < A * 1024; i += blockDim.x)
    q1s_smem[i] = ABBA[(size_t)(i >> 10) * (1 << kQbf1B) + (size_t)blk * 1024 + (i & 1023)];
  __syncthreads();
  const int t = threadIdx.x & 63;
  const uint64_t chunk = (uint64_t)blockIdx.y * 4 + (threadIdx.x >> 6);
  const uint64_t steps = 1ull << A;
  const uint64_t i0 = chunk * chunk_len;
  if (i0 >= steps) return;
  const uint64_t i1 = min(steps, i0 + chunk_len);
  int E[16];
  const uint64_t p0 = gray64(i0);
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    int v = BB[blk * 1024 + 64 * c + t];
    for (int k = 0; k < A; ++k)
      if ((p0 >> (A - 1 - k)) & 1) v += q1s_smem[k * 1024 + 64 * c + t];
    E[c] = wrap16(v);
  }
  int m = E[0];
#pragma unroll
  for (int c = 1; c < 16; ++c) m = min(m, E[c]);
  int best = wrap16((int)AA[i0] + m);
  uint64_t bi = i0;
  for (uint64_t i = i0 + 1; i < i1; ++i) {
    const int kb = __ffsll((long long)i) - 1;
    const int row = A - 1 - kb;
    const bool add = (gray64(i) >> kb) & 1;
    const short* r = q1s_smem + row * 1024 + t;
    m = 32767;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int d = r[64 * c];
      E[c] = wrap16(add ? E[c] + d : E[c] - d);
      m = min(m, E[c]);
    }
    const int tt = wrap16((int)AA[i] + m);
    if (tt < best) {  // strict: the earliest step keeps a tie
      best = tt;
      bi = i;
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
