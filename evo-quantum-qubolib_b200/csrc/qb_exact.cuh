// qb_exact.cuh -- exact enumeration of state records (the "pass 2" kernel).
//
// One CTA per record.  A record is a set of 2^f states: a base state with f free bits
// (record_states in qb_common.cuh).  Threads split the free bits: the top bits select a
// thread, the low L bits are walked in Gray order with an incremental energy update
//   flip v:  E += (1 - 2 x_v) * (W_vv + h_v),   h_u += (1 - 2 x_v) * W_uv  (u free, u != v)
// in FP64, which is exact for integer Q with sum|Q| < 2^53.  Each thread keeps the
// lexicographic minimum of (E, tie key); the CTA reduces and writes one ExactOut per
// record.  The winner's energy is re-evaluated from scratch so the reported value does not
// carry the walk's rounding.
#pragma once
#include "qb_common.cuh"

namespace qb {

struct ExactOut {
  double e;
  uint64_t key;
  uint64_t x;
};

constexpr int kExactThreads = 256;
constexpr int kExactMaxFree = 40;
constexpr int kExactTableMaxL = 12;  // walks of up to 12 bits use the table form below

__device__ __forceinline__ double energy_from_scratch(const double* __restrict__ Ws, int n, uint64_t X) {
  double e = 0.0;
  uint64_t rem = X & mask64(n);
  while (rem) {
    int p = 63 - __clzll(rem);  // highest set bit = lowest variable index
    rem &= ~(1ull << p);
    int i = n - 1 - p;
    const double* row = Ws + i * n;
    e += row[i];
    uint64_t r2 = rem;  // variables after i
    while (r2) {
      int q = 63 - __clzll(r2);
      r2 &= ~(1ull << q);
      e += row[n - 1 - q];
    }
  }
  return e;
}

__device__ __forceinline__ bool lex_less(double e1, uint64_t k1, double e2, uint64_t k2) {
  return e1 < e2 || (e1 == e2 && k1 < k2);
}

// One CTA (kExactThreads threads) evaluates record rid exactly -- or, with split_bits > 0,
// part `part` of it: the record's top split_bits free bits fixed to the bits of part (at
// most f - 8 of them) -- and thread 0 writes the lexicographic minimum to *out_slot.
// smem_d: exact_smem_bytes(n, f) of dynamic shared memory.
__device__ __forceinline__ void exact_record_body(const ProblemDev& P, const TieRule& R, const RecGeom& G,
                                                  uint64_t rid, ExactOut* __restrict__ out_slot, double* smem_d,
                                                  int part = 0, int split_bits = 0) {
  const int n = P.n;
  double* Ws = smem_d;                       // n*n
  double* Wl = Ws + n * n;                   // L*L couplings among low free variables
  __shared__ int pos[kExactMaxFree];         // free bit positions, ascending
  __shared__ int nfree;
  __shared__ double red_e[kExactThreads / 32];
  __shared__ uint64_t red_k[kExactThreads / 32], red_x[kExactThreads / 32];

  for (int i = threadIdx.x; i < n * n; i += blockDim.x) Ws[i] = P.W[i];
  uint64_t base, fm;
  record_states(G, rid, &base, &fm);
  if (threadIdx.x == 0) {
    int c = 0;
    uint64_t m = fm & mask64(n);
    while (m && c < kExactMaxFree) {
      int b = __ffsll((long long)m) - 1;
      pos[c++] = b;
      m &= m - 1;
    }
    nfree = c;
  }
  __syncthreads();
  const int sb = split_bits < nfree - 8 ? split_bits : (nfree > 8 ? nfree - 8 : 0);
  const int f = nfree - sb;  // the top sb free bits are fixed by part
  for (int j = 0; j < sb; ++j)
    if ((part >> j) & 1) base |= 1ull << pos[f + j];
  const int tb = f < 8 ? f : 8;  // thread-selecting bits
  const int L = f - tb;          // bits walked per thread
  for (int i = threadIdx.x; i < L * L; i += blockDim.x) {
    int a = i / L, c = i % L;
    Wl[i] = Ws[(n - 1 - pos[a]) * n + (n - 1 - pos[c])];
  }
  __syncthreads();
  // Table form (walks of at most kExactTableMaxL bits, when the record's smem holds the
  // tables): with the thread's other bits fixed in X0, the energy of X0 with the walked
  // pattern g is E(X0) + a . g + q(g), where a_u is the field of walked variable u from X0
  // (per thread, in smem) and q(g) the energy of the pattern alone (shared by all threads).
  // A Gray walk then costs one field add, one table read and one add per state.
  const bool table = L <= kExactTableMaxL && nfree - 8 <= kExactTableMaxL;
  double* qt = Wl + L * L;                    // q(g), 2^L entries
  double* at = qt + (table ? (1 << L) : 0);   // a_u of thread t at [u * blockDim.x + t]
  if (table) {
    for (int g = threadIdx.x; g < (1 << L); g += blockDim.x) {
      double q = 0.0;
      for (int u = 0; u < L; ++u) {
        if (!((g >> u) & 1)) continue;
        q += Wl[u * L + u];
        for (int w = 0; w < u; ++w)
          if ((g >> w) & 1) q += Wl[u * L + w];
      }
      qt[g] = q;
    }
    __syncthreads();
  }

  double best_e = __longlong_as_double(0x7ff0000000000000ll);  // +inf
  uint64_t best_k = ~0ull, best_x = 0;
  const int t = threadIdx.x;
  if (table && t < (1 << tb)) {
    uint64_t X0 = base;
    for (int j = 0; j < tb; ++j)
      if ((t >> j) & 1) X0 |= 1ull << pos[L + j];
    const double c0 = energy_from_scratch(Ws, n, X0);
    for (int j = 0; j < L; ++j) {
      const int v = n - 1 - pos[j];
      double s = 0.0;
      uint64_t rem = X0 & mask64(n);
      while (rem) {
        const int q = __ffsll((long long)rem) - 1;
        rem &= rem - 1;
        s += Ws[v * n + (n - 1 - q)];  // the walked bits are 0 in X0: no self term
      }
      at[j * blockDim.x + t] = s;
    }
    best_e = c0;
    best_k = tie_key(R, X0);
    best_x = X0;
    double A = 0.0;
    const uint32_t steps = 1u << L;
    for (uint32_t st = 1; st < steps; ++st) {
      const int j = __ffs(st) - 1;
      const uint32_t g = st ^ (st >> 1);
      const double aj = at[j * blockDim.x + t];
      A = ((g >> j) & 1) ? A + aj : A - aj;
      const double e = c0 + A + qt[g];
      if (e <= best_e) {
        uint64_t X = X0;
        for (int u = 0; u < L; ++u)
          if ((g >> u) & 1) X |= 1ull << pos[u];
        const uint64_t k = tie_key(R, X);
        if (lex_less(e, k, best_e, best_k)) {
          best_e = e;
          best_k = k;
          best_x = X;
        }
      }
    }
    best_e = energy_from_scratch(Ws, n, best_x);
  } else if (t < (1 << tb)) {
    uint64_t X = base;
    for (int j = 0; j < tb; ++j)
      if ((t >> j) & 1) X |= 1ull << pos[L + j];
    double e = energy_from_scratch(Ws, n, X);
    double h[kExactMaxFree];
    for (int j = 0; j < L; ++j) {
      int v = n - 1 - pos[j];
      double s = 0.0;
      uint64_t rem = X & mask64(n);
      while (rem) {
        int q = __ffsll((long long)rem) - 1;
        rem &= rem - 1;
        int u = n - 1 - q;
        if (u != v) s += Ws[v * n + u];
      }
      h[j] = s;
    }
    best_e = e;
    best_k = tie_key(R, X);
    best_x = X;
    const uint64_t steps = 1ull << L;
    for (uint64_t s = 1; s < steps; ++s) {
      int j = __ffsll((long long)s) - 1;
      uint64_t bit = 1ull << pos[j];
      bool on = !(X & bit);
      int v = n - 1 - pos[j];
      double d = Ws[v * n + v] + h[j];
      e = on ? e + d : e - d;
      X ^= bit;
      const double* wl = Wl + j * L;
      for (int u = 0; u < L; ++u) {
        if (u == j) continue;
        h[u] = on ? h[u] + wl[u] : h[u] - wl[u];
      }
      if (e <= best_e) {
        uint64_t k = tie_key(R, X);
        if (lex_less(e, k, best_e, best_k)) {
          best_e = e;
          best_k = k;
          best_x = X;
        }
      }
    }
    best_e = energy_from_scratch(Ws, n, best_x);
  }
  // CTA reduction of (e, key, x)
  for (int off = 16; off; off >>= 1) {
    double oe = __shfl_down_sync(0xffffffffu, best_e, off);
    uint64_t ok = __shfl_down_sync(0xffffffffu, best_k, off);
    uint64_t ox = __shfl_down_sync(0xffffffffu, best_x, off);
    if (lex_less(oe, ok, best_e, best_k)) {
      best_e = oe;
      best_k = ok;
      best_x = ox;
    }
  }
  if ((t & 31) == 0) {
    red_e[t >> 5] = best_e;
    red_k[t >> 5] = best_k;
    red_x[t >> 5] = best_x;
  }
  __syncthreads();
  if (t == 0) {
    for (int w = 1; w < kExactThreads / 32; ++w)
      if (lex_less(red_e[w], red_k[w], best_e, best_k)) {
        best_e = red_e[w];
        best_k = red_k[w];
        best_x = red_x[w];
      }
    *out_slot = ExactOut{best_e, best_k, best_x};
  }
}

// rec_ids: candidate record indices (nullptr: record = rec_offset + block).
// count_ptr: number of valid entries (nullptr: count_static).
// split_bits: 2^split_bits CTAs per record (block = blockIdx.x >> split_bits); outputs are
// indexed (slot << split_bits) | part.
__global__ void __launch_bounds__(kExactThreads)
exact_records_kernel(ProblemDev P, TieRule R, RecGeom G, const uint64_t* __restrict__ rec_ids,
                     const int* __restrict__ count_ptr, int64_t count_static, int64_t rec_offset,
                     ExactOut* __restrict__ out, int split_bits) {
  extern __shared__ double smem_d[];
  const int64_t blk = (int64_t)(blockIdx.x >> split_bits);
  const int part = (int)(blockIdx.x & ((1u << split_bits) - 1u));
  const int64_t slot = blk + (rec_ids ? rec_offset : 0);
  const int64_t count = count_ptr ? (int64_t)(*count_ptr) : count_static;
  if (slot >= count) return;
  const uint64_t rid = rec_ids ? rec_ids[slot] : (uint64_t)(rec_offset + blk);
  exact_record_body(P, R, G, rid, out + ((slot << split_bits) | part), smem_d, part, split_bits);
}

// The candidate records listed in rec_ids[0 .. min(*count_ptr, cap)), each split into
// 2^split_bits parts, as a grid-stride loop over (record, part) items: the host launches it
// before it knows the count.  Outputs at (slot << split_bits) | part.
__global__ void __launch_bounds__(kExactThreads)
exact_candidates_kernel(ProblemDev P, TieRule R, RecGeom G, const uint64_t* __restrict__ rec_ids,
                        const int* __restrict__ count_ptr, int cap, int split_bits, ExactOut* __restrict__ out) {
  extern __shared__ double smem_d[];
  const int count = min(*count_ptr, cap);
  const int64_t items = (int64_t)count << split_bits;
  for (int64_t w = blockIdx.x; w < items; w += gridDim.x) {
    __syncthreads();  // the previous item's shared-memory readers are done
    const int64_t slot = w >> split_bits;
    const int part = (int)(w & ((1 << split_bits) - 1));
    exact_record_body(P, R, G, rec_ids[slot], out + w, smem_d, part, split_bits);
  }
}

// One CTA: the lexicographic minimum of the first min(*count_ptr, cap) << split_bits
// outputs into *best (x = 0 with energy 0 and key 0 when *zero_flag is set).
__global__ void exact_final_kernel(const ExactOut* __restrict__ out, const int* __restrict__ count_ptr, int cap,
                                   int split_bits, const int* __restrict__ zero_flag, ExactOut* __restrict__ best) {
  __shared__ double se[32];
  __shared__ uint64_t sk[32], sx[32];
  const int64_t items = (int64_t)min(*count_ptr, cap) << split_bits;
  double be = __longlong_as_double(0x7ff0000000000000ll);
  uint64_t bk = ~0ull, bx = 0;
  for (int64_t i = threadIdx.x; i < items; i += blockDim.x)
    if (lex_less(out[i].e, out[i].key, be, bk)) {
      be = out[i].e;
      bk = out[i].key;
      bx = out[i].x;
    }
  for (int off = 16; off; off >>= 1) {
    const double oe = __shfl_down_sync(0xffffffffu, be, off);
    const uint64_t ok = __shfl_down_sync(0xffffffffu, bk, off);
    const uint64_t ox = __shfl_down_sync(0xffffffffu, bx, off);
    if (lex_less(oe, ok, be, bk)) {
      be = oe;
      bk = ok;
      bx = ox;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    se[threadIdx.x >> 5] = be;
    sk[threadIdx.x >> 5] = bk;
    sx[threadIdx.x >> 5] = bx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (lex_less(se[w], sk[w], be, bk)) {
        be = se[w];
        bk = sk[w];
        bx = sx[w];
      }
    *best = *zero_flag ? ExactOut{0.0, 0ull, 0ull} : ExactOut{be, bk, bx};
  }
}

inline size_t exact_smem_bytes(int n, int f) {
  int L = f > 8 ? f - 8 : 0;
  size_t d = (size_t)(n * n + L * L);
  if (L <= kExactTableMaxL) d += ((size_t)1 << L) + (size_t)kExactThreads * L;  // q table, per-thread fields
  return d * sizeof(double);
}

}  // namespace qb
