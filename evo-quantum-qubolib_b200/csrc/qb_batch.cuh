// qb_batch.cuh -- many independent problems in one launch sequence.
//
// A batch of small problems (1 <= n <= 36) runs as six launches in total, whatever the
// number of problems, with no host round trip in between:
//   1. batch_gtab_kernel    G tables of every Gray-form problem (20 <= n < 24)
//   2. batch_gray_kernel    pass 1 of every Gray-form problem: one CTA per (problem, unit)
//   2'. tc_pass1_kernel     pass 1 of every tensor-core problem (n >= 24): each persistent
//                           CTA runs a list of (problem, run of record blocks) items
//   3. batch_select_kernel  per problem: smallest record, threshold, candidate records
//   4. batch_exact_kernel   exact FP64 re-evaluation of every candidate record -- and, for
//                           problems with n < 20, of all their records (the whole search)
//   5. batch_key_kernel     per problem: smallest order key among the states of minimal E
// Per-problem minima are combined with 64-bit atomics on an order-preserving encoding of
// the FP64 energy, then on the tie-rule key, which maps one-to-one to the state.
#pragma once
#include "qb_common.cuh"
#include "qb_exact.cuh"
#include "qb_gray.cuh"

namespace qb {

constexpr int kBatchGray = 1;   // Gray form + exact pass 2
constexpr int kBatchTC = 2;     // tensor-core form + exact pass 2
constexpr int kBatchExact = 3;  // exact enumeration of every record (small n)

struct BatchInst {
  int n, kind;
  int a, b, cbbits, sbits, gubits;  // Gray plan
  int fbits;                        // exact plan: states per record = 2^fbits
  int gl;                           // tensor-core plan: log2 tiles per record block
  int exact_digits;                 // tensor-core plan: integer digits (exact)
  double scale;                     // tensor-core plan: power of two applied to W
  int A, B;                         // QBF tie rule split (A inverse-Gray ranked prefix bits)
  int natural;                      // 1: natural order (smallest X) among ties
  int is_int;
  int tc_kernel;                    // tensor-core plan: qb_result.tc_kernel (1 fp32, 4 16-bit pair)
  uint64_t w_off;     // doubles into the packed W array
  uint64_t gtab_off;  // floats into the packed G tables
  uint64_t rec_off;   // floats into the packed record minima
  uint64_t nrec;      // Gray records
  double eps;         // pass-1 error bound (0: exact fp32 arithmetic)
};

struct BatchItem {  // one CTA's work: (problem, first, last)
  uint32_t inst, pad;
  uint64_t lo, hi;
};

struct BatchCand {  // a record to evaluate exactly
  uint32_t inst, pad;
  uint64_t rid;
};

__host__ __device__ __forceinline__ uint64_t ord_f64(double e) {
#ifdef __CUDA_ARCH__
  uint64_t u = (uint64_t)__double_as_longlong(e);
#else
  uint64_t u;
  memcpy(&u, &e, 8);
#endif
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__host__ __device__ __forceinline__ double unord_f64(uint64_t k) {
  uint64_t u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double e;
  memcpy(&e, &u, 8);
  return e;
#endif
}

__device__ __forceinline__ ProblemDev batch_problem(const BatchInst& I, const double* W) {
  return ProblemDev{I.n, W + I.w_off};
}

__device__ __forceinline__ TieRule batch_rule(const BatchInst& I) {
  return I.natural ? TieRule{kTieNatural, I.n, 0, 0, 0} : TieRule{kTieQBF, I.n, 0, I.A, I.B};
}

__device__ __forceinline__ RecGeom batch_geom(const BatchInst& I) {
  RecGeom g{};
  g.n = I.n;
  if (I.kind == kBatchTC) {
    g.kind = kGeomTC;
    g.gl = I.gl;
  } else if (I.kind == kBatchGray) {
    g.kind = kGeomGray;
    g.a = I.a;
    g.b = I.b;
    g.sbits = I.sbits;
    g.cbbits = I.cbbits;
    g.gubits = I.gubits;
  } else {
    g.kind = kGeomBlock;
    g.fbits = I.fbits;
  }
  return g;
}

// 1. G tables: one CTA per item = (Gray problem, steps [lo, hi))
__global__ void batch_gtab_kernel(const BatchInst* __restrict__ insts, const BatchItem* __restrict__ items,
                                  const double* __restrict__ W, float* __restrict__ gtab) {
  extern __shared__ double bgt_smem[];
  const BatchItem it = items[blockIdx.x];
  const BatchInst I = insts[it.inst];
  gray_gtab_body(batch_problem(I, W), I.a, gtab + I.gtab_off, it.lo, it.hi, bgt_smem);
}

// 2. pass 1: one CTA per item = (Gray problem, unit lo)
__global__ void __launch_bounds__(kGrayThreads, 2)
batch_gray_kernel(const BatchInst* __restrict__ insts, const BatchItem* __restrict__ items,
                  const double* __restrict__ W, const float* __restrict__ gtab, float* __restrict__ rec) {
  extern __shared__ __align__(16) unsigned char bgr_smem[];
  const BatchItem it = items[blockIdx.x];
  const BatchInst I = insts[it.inst];
  GrayParams g{};
  g.P = batch_problem(I, W);
  g.a = I.a;
  g.b = I.b;
  g.cbbits = I.cbbits;
  g.sbits = I.sbits;
  g.gubits = I.gubits;
  g.unit_begin = 0;
  g.gtab = gtab + I.gtab_off;
  g.rec = rec + I.rec_off;
  gray_unit_body(g, it.lo, bgr_smem);
}

// 3. per Gray or tensor-core problem (one CTA each): pass-1 minimum, threshold, candidate records
__global__ void batch_select_kernel(const BatchInst* __restrict__ insts, const uint32_t* __restrict__ gray_ids,
                                    const float* __restrict__ rec, BatchCand* __restrict__ cand,
                                    int* __restrict__ cand_count, int cap, float* __restrict__ pass1_min,
                                    uint64_t* __restrict__ emin, uint64_t* __restrict__ kmin) {
  __shared__ uint32_t red[32];
  const uint32_t id = gray_ids[blockIdx.x];
  const BatchInst I = insts[id];
  const float* r = rec + I.rec_off;
  uint32_t k = 0xffffffffu;
  for (uint64_t i = threadIdx.x; i < I.nrec; i += blockDim.x) {
    const uint32_t v = f2key(r[i]);
    k = v < k ? v : k;
  }
  k = __reduce_min_sync(0xffffffffu, k);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0xffffffffu;
    v = __reduce_min_sync(0xffffffffu, v);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  const double m = (double)key2f(red[0]);
  if (threadIdx.x == 0) pass1_min[id] = (float)m;
  if (I.is_int && I.eps == 0.0 && m >= 0.0) {  // E(0) = 0 is minimal and X = 0 has key 0
    if (threadIdx.x == 0) {
      emin[id] = ord_f64(0.0);
      kmin[id] = 0ull;
    }
    return;
  }
  double thr = m + 2.0 * I.eps;
  if (I.eps > 0.0) thr += fabs(thr) * 1e-12;
  for (uint64_t i = threadIdx.x; i < I.nrec; i += blockDim.x) {
    if ((double)r[i] <= thr) {
      const int s = atomicAdd(cand_count, 1);
      if (s < cap) cand[s] = BatchCand{id, 0u, i};
    }
  }
}

// 4. exact evaluation of candidate s = blockIdx.x (s < min(count, cap))
__global__ void __launch_bounds__(kExactThreads)
batch_exact_kernel(const BatchInst* __restrict__ insts, const double* __restrict__ W,
                   const BatchCand* __restrict__ cand, const int* __restrict__ cand_count, int cap,
                   ExactOut* __restrict__ out, uint64_t* __restrict__ emin) {
  extern __shared__ double bex_smem[];
  const int count = min(*cand_count, cap);
  if ((int)blockIdx.x >= count) return;
  const BatchCand c = cand[blockIdx.x];
  const BatchInst I = insts[c.inst];
  exact_record_body(batch_problem(I, W), batch_rule(I), batch_geom(I), c.rid, out + blockIdx.x, bex_smem);
  if (threadIdx.x == 0) atomicMin(reinterpret_cast<unsigned long long*>(emin + c.inst),
                                  (unsigned long long)ord_f64(out[blockIdx.x].e));
}

// 5. smallest key among each problem's minimal-energy candidates
__global__ void batch_key_kernel(const BatchCand* __restrict__ cand, const int* __restrict__ cand_count, int cap,
                                 const ExactOut* __restrict__ out, const uint64_t* __restrict__ emin,
                                 uint64_t* __restrict__ kmin) {
  const int count = min(*cand_count, cap);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
    const uint32_t id = cand[s].inst;
    if (ord_f64(out[s].e) == emin[id])
      atomicMin(reinterpret_cast<unsigned long long*>(kmin + id), (unsigned long long)out[s].key);
  }
}

}  // namespace qb
