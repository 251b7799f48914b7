// qb_reduce.cuh -- reduction of pass-1 record minima and selection of candidate records.
//
// Pass 1 writes one float per record: the minimum pass-1 energy over the record's states.
// rec_min_kernel finds the smallest record value (order-preserving uint32 keys, atomicMin).
// rec_select_kernel lists every record whose value is <= global_min + slack, where slack is
// twice the per-state error bound of pass-1 arithmetic (0 for the exact integer path), so
// every record that can hold an exact minimiser is re-evaluated in pass 2.
#pragma once
#include "qb_common.cuh"

namespace qb {

__global__ void rec_min_kernel(const float* __restrict__ rec, int64_t count, uint32_t* __restrict__ min_key) {
  uint32_t k = 0xffffffffu;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    uint32_t v = f2key(rec[i]);
    k = v < k ? v : k;
  }
  k = __reduce_min_sync(0xffffffffu, k);
  if ((threadIdx.x & 31) == 0 && k != 0xffffffffu) atomicMin(min_key, k);
}

// Candidate indices are rec_index_offset + i for the selected positions i.
__global__ void rec_select_kernel(const float* __restrict__ rec, int64_t count, int64_t rec_index_offset,
                                  double threshold, uint64_t* __restrict__ cand, int* __restrict__ cand_count,
                                  int cap) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    if ((double)rec[i] <= threshold) {
      int s = atomicAdd(cand_count, 1);
      if (s < cap) cand[s] = (uint64_t)(rec_index_offset + i);
    }
  }
}

// threshold of the candidate selection from the pass-1 minimum (on the device, so the
// selection can follow without a host round trip): min + 2 eps (+ 1e-12 relative when eps >
// 0); *zero_flag = 1 when the arithmetic is exact, the problem integer and the minimum >= 0
// (then E(0) = 0 is minimal and X = 0 wins every tie rule)
// (*zero_flag is also set, skipping the selection, when the search kernel reported an
// error in *err: its records are incomplete and the host reports the error)
__global__ void rec_threshold_kernel(const uint32_t* __restrict__ min_key, double eps, int exact_int,
                                     const unsigned* __restrict__ err, double* __restrict__ thr,
                                     int* __restrict__ zero_flag, int* __restrict__ cand_count) {
  const double m = (*min_key == 0xffffffffu) ? __longlong_as_double(0x7ff0000000000000ll) : (double)key2f(*min_key);
  double t = m + 2.0 * eps;
  if (eps > 0.0) t += fabs(t) * 1e-12;
  *thr = t;
  *zero_flag = ((exact_int && eps == 0.0 && m >= 0.0) || (err && *err)) ? 1 : 0;
  *cand_count = 0;
}

// rec_select_kernel with the threshold (and the zero shortcut) read from the device
__global__ void rec_select_dev_kernel(const float* __restrict__ rec, int64_t count, int64_t rec_index_offset,
                                      const double* __restrict__ thr, const int* __restrict__ zero_flag,
                                      uint64_t* __restrict__ cand, int* __restrict__ cand_count, int cap) {
  if (*zero_flag) return;
  const double t = *thr;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    if ((double)rec[i] <= t) {
      const int s = atomicAdd(cand_count, 1);
      if (s < cap) cand[s] = (uint64_t)(rec_index_offset + i);
    }
  }
}

}  // namespace qb
