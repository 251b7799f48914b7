/*
 * qubo_b200.h -- C ABI of libqubo_b200.so, the B200 (sm_100a) exhaustive QUBO search.
 *
 * The reference (cloud-ru-tech/evo-quantum-qubolib) has no native library: its solvers are
 * Python classes whose hot loops call numpy/cupy.  Each entry point below replaces one of
 * those Python call sites; the citation beside it names the reference code it stands in for.
 * A binding adds nothing but pointers and sizes: no torch, numpy or CUDA-runtime types
 * cross this boundary (streams are passed as void*).
 *
 * Problem: minimise E(x) = sum_ij Q_ij x_i x_j over x in {0,1}^n, Q the full (possibly
 * asymmetric) n x n matrix.  States are reported as the MSB-first integer X of the state
 * vector: variable i is bit (n-1-i), the convention of the reference's best_X printout.
 *
 * Ties between minimal states follow the reference's search order (tie_rule):
 *   QB_TIE_QBF   : with fixed_bits = k and prefix_bits = A, the smallest
 *                  (first k bits as an integer, inverse-Gray rank of the next A bits,
 *                   remaining bits as an integer) -- QBF's prefix loop
 *                  (src/qubo_lib/solvers/qbf.py:188-230, 395-412) under Parallel's bit
 *                  fixing (src/qubo_lib/solvers/parallel.py:145-157, lowest task first).
 *   QB_TIE_QB_F1 : QB_F1's kernel order (src/qubo_lib/solvers/qbf1.py:179-249, 253-264):
 *                  lowest thread of the 256x64 grid, then earliest Gray prefix, then the
 *                  smallest 18-bit suffix of that prefix.
 *   QB_TIE_NATURAL: smallest X.
 * Float Q: the answer is the FP64 argmin (energies re-evaluated in FP64 on the GPU).
 *
 * Errors are returned as int status codes; no exceptions or exits cross the ABI.
 * Thread-compatible per handle: one handle per host thread / stream.
 */
#ifndef QUBO_B200_H
#define QUBO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define QB_OK 0
#define QB_EINVAL 1      /* bad argument (n, dtype, split, pointer) */
#define QB_ERANGE 2      /* |Q| too large for exact evaluation (see qb_solve) */
#define QB_ENOMEM 3      /* device allocation failed */
#define QB_ECUDA 4       /* CUDA runtime error */
#define QB_ETIMEOUT 5    /* a bounded wait inside a kernel gave up */
#define QB_ENODEV 6      /* no CUDA device / bad device index */
#define QB_EOVERFLOW 7   /* too many candidate records (raise QB_MAX_CANDIDATES) */
#define QB_ETOOBIG 8     /* qb_solve_noalloc: n outside the fixed scratch (20 <= n <= 36) */

/* element types of Q */
#define QB_F32 1
#define QB_F64 2
#define QB_I8 3
#define QB_I16 4
#define QB_I32 5
#define QB_I64 6

/* search forms */
#define QB_FORM_AUTO 0   /* tensor-core form when it applies, else Gray form, else exact */
#define QB_FORM_GRAY 1   /* plain Gray-code SIMT kernel (fp32 or int32 arithmetic) */
#define QB_FORM_TC 2     /* tcgen05 contraction form (f16 digits, fp32 accumulate) */
#define QB_FORM_EXACT 3  /* FP64 / integer-exact enumeration (small n) */
#define QB_FORM_QBF1_INT16 4  /* (reported only) QB_F1 in the reference's int16 arithmetic */

/* qb_options.flags */
#define QB_FLAG_INT16_WRAP 1  /* QB_TIE_QB_F1, int16 Q, 19 <= n <= 46: reproduce the reference
                                 QB_F1's int16 arithmetic (its tables and running sums wrap
                                 modulo 2^16), so that the state and the reported best_e_int
                                 are the reference's even where its sums overflow; best_e is
                                 the exact energy of that state (qbf1.py:86-133, 179-289) */
#define QB_FLAG_GRAPH 4       /* qb_solve_batch: run the batch's device work (uploads, the six
                                 launches, the result copy) as one CUDA graph launch.  The graph
                                 is captured on the first call and replayed by later calls whose
                                 batch has the same shape (sizes, dtype classes, options); any
                                 other batch is captured anew.  pass1_ms then holds the whole
                                 graph's device time and pass2_ms is 0 */
#define QB_FLAG_TC_PAIR 8      /* QB_FORM_TC, qb_solve / qb_solve_begin: run the tensor-core pair
                                 form, which derives a second state from every accumulator (each
                                 MMA tile also yields the tile that differs in one variable)
                                 instead of reading one state per accumulator; the answers are
                                 the same (qb_autotune may also choose it) */
#define QB_FLAG_TC_ONE 32      /* QB_FORM_TC, qb_solve / qb_solve_begin: run one state per
                                 accumulator where the pair form would be the default (the
                                 16-bit pair form is the default wherever it applies and no
                                 tuned entry names the kernel); QB_EINVAL together with
                                 QB_FLAG_TC_PAIR; the answers are the same */
#define QB_FLAG_TC_NO16 16     /* QB_FORM_TC: keep the fp32 minima where the 16-bit epilogue
                                 would apply (tc_kernel 1 instead of 3, 2 instead of 4); the
                                 answers are the same */
#define QB_FLAG_TEST_STALL 2  /* tests only, QB_FORM_TC: the search kernel's tile walk
                                 publishes nothing, so the kernel's bounded waits run out
                                 (about 2 s); the call returns QB_ETIMEOUT and the handle
                                 and CUDA context stay usable */

/* tie rules */
#define QB_TIE_QBF 0
#define QB_TIE_QB_F1 1
#define QB_TIE_NATURAL 2

typedef struct qb_handle_s qb_handle;

typedef struct qb_problem {
  int32_t n;            /* variables, 1..62; one call's search must fit one launch: the
                           tensor-core form below 2^32 tiles per CTA (n <= 54 on 148 SMs),
                           the Gray form below 2^31 work units (n <= 59), else QB_EINVAL /
                           QB_ECUDA -- split larger searches with shard_index/shard_count */
  int32_t dtype;        /* QB_F32 .. QB_I64 */
  const void* q;        /* n x n, row-major, leading dimension ldq elements */
  int64_t ldq;
  int32_t q_on_device;  /* 0: host memory; 1: device memory of the handle's device */
  int32_t reserved;
} qb_problem;

typedef struct qb_options {
  int32_t form;         /* QB_FORM_* */
  int32_t tie_rule;     /* QB_TIE_* */
  int32_t fixed_bits;   /* QB_TIE_QBF: k leading task bits (Parallel splits_cnt = 2^k) */
  int32_t prefix_bits;  /* QB_TIE_QBF: A inverse-Gray ranked bits after them; -1 = QBF default */
  int32_t shard_index;  /* multi-GPU: this rank's share of the search space ... */
  int32_t shard_count;  /* ... out of shard_count equal shares (1 = everything) */
  int32_t max_candidates; /* cap on candidate records re-scored per pass-2 launch (0 = default) */
  int32_t flags;        /* QB_FLAG_*, 0 = none */
  void* stream;         /* cudaStream_t to run on; NULL = the handle's own stream */
} qb_options;

typedef struct qb_result {
  uint64_t best_x;        /* MSB-first state integer */
  double best_e;          /* E(best_x) in FP64 (exact for integer Q) */
  int64_t best_e_int;     /* exact energy for integer Q */
  uint64_t order_key;     /* tie-rule key of best_x (smaller wins among equal energies) */
  double pass1_min;       /* minimum seen by the pass-1 kernel (fp32 arithmetic) */
  double err_bound;       /* bound on |pass-1 value - exact value| per state */
  int64_t states;         /* states whose energy entered the minimum in this call */
  int64_t candidate_records; /* records re-evaluated exactly in pass 2 */
  int32_t form_used;      /* QB_FORM_* actually run */
  int32_t is_integer;     /* Q had an integer dtype */
  int32_t found;          /* 1 if this call's share holds a minimal state */
  int32_t status;
  float pass1_ms;         /* device time of pass 1 (CUDA events) */
  float pass2_ms;         /* device time of reduction + candidate re-evaluation */
  int32_t kernels;        /* kernel launches issued by this call */
  float kernel_ms;        /* device time of the main pass-1 search kernel alone */
  int64_t h2d_bytes;      /* bytes copied host -> device by this call */
  int64_t d2h_bytes;      /* bytes copied device -> host by this call */
  int32_t rec_log2;       /* record granularity: log2 tiles per record block (QB_FORM_TC),
                             log2 prefix steps per record (QB_FORM_GRAY), log2 states per
                             record (QB_FORM_EXACT) */
  int32_t suffix_bits;    /* QB_FORM_GRAY: suffix bits b of the prefix/suffix split;
                             QB_FORM_TC: 15 (the 128 x 256 states of a tile); else 0 */
  int32_t unit_log2;      /* QB_FORM_GRAY: log2 prefix steps per work unit; else 0 */
  int32_t tuned;          /* 1 when qb_autotune's choice for (n, dtype class) was applied */
  int32_t tc_kernel;      /* QB_FORM_TC: 1 one state per accumulator, fp32 minima; 2 pair form,
                             fp32 minima; 3 one state per accumulator, exact 16-bit minima
                             (integer Q whose accumulator values span fewer than 2^16
                             integers); 4 pair form, exact 16-bit minima (the same, with room
                             for the pair's per-chunk shifts); 0 other forms */
} qb_result;

/* Library version (major * 10000 + minor * 100 + patch). */
int qb_version(void);

/* Human-readable text of a status code. */
const char* qb_strerror(int status);

/* Open a handle on CUDA device `device`.  The handle owns a stream and its device scratch
 * (per-record minima, candidate lists), grown on demand and freed by qb_handle_destroy.
 * Replaces SolverABC.init_gpu / parse_device_arg (src/qubo_lib/abc/solver_abc.py:62-84). */
int qb_handle_create(int device, qb_handle** out);
int qb_handle_destroy(qb_handle* h);

/* Exhaustive minimum of one problem: pass 1 (GPU kernel over all states, per-record
 * minima), pass 2 (exact re-evaluation of the records that can hold the minimum), tie rule.
 * Replaces QBF.prepare + iterate_prefix_interval + pack_results
 * (src/qubo_lib/solvers/qbf.py:72-103, 188-230, 328-360) and QB_F1.prepare + QB_F1_kernel +
 * pack_results (src/qubo_lib/solvers/qbf1.py:86-133, 179-249, 253-289).  Blocks until the
 * result is on the host.  Integer Q needs sum|Q_ij| < 2^53 (else QB_ERANGE). */
int qb_solve(qb_handle* h, const qb_problem* p, const qb_options* o, qb_result* r);

/* Two-phase form of qb_solve for sharded (multi-GPU) searches: qb_solve_begin runs pass 1
 * over this shard and returns its minimum in *local_min; the caller reduces the minima over
 * all shards (min) and passes the global value to qb_solve_finish, which re-evaluates this
 * shard's candidate records and fills *r (r->found = 0 when the shard holds no minimiser).
 * Replaces devices_scheduler + merge_bruteforcer_partial_solutions
 * (src/qubo_lib/solvers/scheduler.py:5-45, src/qubo_lib/solvers/parallel.py:225-320). */
int qb_solve_begin(qb_handle* h, const qb_problem* p, const qb_options* o, double* local_min);
int qb_solve_finish(qb_handle* h, double global_min, qb_result* r);

/* Many independent problems in one launch sequence (persistent kernel over all
 * (problem, tile) work items).  Results in r[0..count).  Replaces a host loop of
 * QBF().solve calls (src/qubo_lib/solvers/qbf.py:48-70). */
int qb_solve_batch(qb_handle* h, const qb_problem* problems, int32_t count, const qb_options* o,
                   qb_result* r);

/* Minimum energy of every A-bit prefix, in the order QBF's prefix loop visits them:
 * out[i] = min over the last n - A variables of E(x) with the first A variables equal to
 * the MSB-first bits of gray(i) = i ^ (i >> 1).  out holds 2^A doubles (host memory).
 * prefix_bits = A (-1 = QBF default n - min(n, 20)); A <= 26 and n - A <= 40.  Energies
 * are exact FP64 sums (integer Q exact).  Replaces the energy_arr metric that QBF records
 * per prefix in update_global_minima (src/qubo_lib/solvers/qbf.py:395-412, 342-351). */
int qb_prefix_minima(qb_handle* h, const qb_problem* p, int32_t prefix_bits, double* out);

/* Tune the search for problems of n variables and dtype: times, on a seeded synthetic problem
 * of the dtype's class (integer or float) on the handle's device, pass 1 + re-evaluation of
 * one shard of at most 2^36 states for the Gray-code form over its prefix/suffix split and
 * record granularity, and for the tensor-core form over its record granularity (the
 * defaults among the candidates), and keeps the fastest (form, parameters) in the handle per
 * (dtype class, n).  QB_FORM_AUTO then runs that form, and every solve of that class and n
 * uses the tuned parameters of its form, in qb_solve and in qb_solve_batch; qb_result reports
 * the parameters used (rec_log2, suffix_bits, unit_log2, tuned).  n < 20 always gives
 * QB_FORM_EXACT.  *form_out receives the chosen QB_FORM_*.  Generalises
 * QBF.define_chunk_size (src/qubo_lib/solvers/qbf.py:429-466), which picks a split from
 * memory size alone. */
int qb_autotune(qb_handle* h, int32_t n, int32_t dtype, int32_t* form_out);

/* Result written by qb_solve_noalloc into device memory. */
typedef struct qb_noalloc_result {
  double best_e;        /* E(best_x) in FP64 (exact for integer Q) */
  uint64_t best_x;      /* MSB-first state integer */
  uint64_t order_key;   /* QB_TIE_QBF key of best_x */
  int32_t status;       /* QB_OK; QB_EOVERFLOW when more candidate records than fit;
                           QB_EINVAL when Q holds a NaN or infinity, or a fractional entry
                           with is_integer set; QB_ERANGE (see below) */
  int32_t candidates;   /* candidate records found by the selection */
} qb_noalloc_result;

/* Exhaustive minimum and argmin (QB_TIE_QBF with prefix_bits, -1 = QBF default) of one
 * problem, for callers that cannot allocate: an application that hands out all of its
 * device memory from its own pool up front, a real-time loop that must not stall on the
 * allocator (cudaMalloc / cudaFree synchronise the device), or code with a device-memory
 * budget fixed at start-up.  No counterpart in the reference, whose solvers allocate
 * (numpy / cupy) on every call.
 *
 * q_dev: n x n float64 Q on `device` (row-major); is_integer: Q holds integers (exact
 * search); out_dev: device pointer receiving the result; stream: cudaStream_t (NULL =
 * default stream).  Queues the Gray-code form on `stream` and returns without waiting.
 * All scratch lives in one fixed device array of 16.9 MB (16,924,928 bytes) inside the library, held
 * by every GPU that loads the library until the process exits: no cudaMalloc, cudaFree or
 * allocating library routine is called.  Limit: 20 <= n <= 36 (QB_ETOOBIG otherwise);
 * up to 4096 candidate records (out_dev->status = QB_EOVERFLOW beyond); integer Q needs
 * sum |Q_ij| < 2^53 (out_dev->status = QB_ERANGE otherwise).
 * The first call on a device resolves the array's address (cudaGetSymbolAddress with that
 * device current): make it before any stream capture, and make it a complete, valid solve
 * (20 <= n <= 36, finite Q), not an early error return, so that it also launches every kernel
 * the entry point uses once (with CUDA's lazy module loading a kernel's first launch can load
 * code and take device memory) before capture begins or a memory budget is fixed.  Every
 * call reuses the same array, so calls that overlap on the GPU race; serialise them. */
int qb_solve_noalloc(int device, const double* q_dev, int32_t n, int32_t is_integer, int32_t prefix_bits,
                     qb_noalloc_result* out_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QUBO_B200_H */
