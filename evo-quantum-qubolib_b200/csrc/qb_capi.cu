// qb_capi.cu -- the C ABI of libqubo_b200.so (declared in include/qubo_b200.h) and the
// host orchestration of one exhaustive search:
//
//   pass 1   a search-form kernel (tensor-core, Gray or exact) visits every state and
//            writes one minimum per record of states;
//   reduce   smallest record value (the pass-1 minimum);
//   select   every record whose value is within 2 * err_bound of the global minimum;
//   pass 2   exact (FP64 / integer) re-evaluation of the selected records with the tie
//            rule's order key; the host takes the lexicographic minimum of (E, key).
//
// Only pass 1 touches all 2^n states.  For integer Q inside the fp32-exact range the
// selection keeps exactly the records that hold a minimal state.
#include "../../include/qubo_b200.h"
#include "qb_batch.cuh"
#include "qb_common.cuh"
#include "qb_exact.cuh"
#include "qb_gray.cuh"
#include "qb_qbf1.cuh"
#include "qb_reduce.cuh"
#include "qb_tc.cuh"
#include "qb_tc2.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 4096);
    cudaError_t e = cudaMallocHost(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

constexpr double kTwo24 = 16777216.0;
constexpr double kTwo53 = 9007199254740992.0;
constexpr int kPrefixMinimaMaxA = 26;  // qb_prefix_minima: at most 2^26 prefixes (512 MiB of results)
constexpr int kDefaultCap = 1 << 16;

// Gray-form split: suffix bits b (>= 13), prefix a = n - b, 2^sbits prefix steps per record,
// 2^ubits prefix steps per work unit
struct GrayShape {
  int a, b, cbbits, sbits, ubits;
};

// the default shape for n, or the one with suffix bits b / record steps 2^sbits when those are
// given (0 = default) and valid: 13 <= b, 7 <= a <= 24, 5 <= sbits <= a
inline GrayShape gray_shape(int n, int b_want = 0, int sbits_want = 0) {
  GrayShape g;
  g.b = std::max(13, n - 16);
  if (b_want >= 13 && n - b_want >= 7 && n - b_want <= 24) g.b = b_want;
  g.a = n - g.b;
  g.cbbits = g.b - 13;
  g.sbits = std::min(g.a, std::max(5, n - 34));
  if (sbits_want >= 5 && sbits_want <= g.a) g.sbits = sbits_want;
  g.ubits = std::min(g.a, std::max(7, std::max(g.sbits, std::min(g.a, g.a + g.cbbits - 11))));
  return g;
}

struct Plan {
  int n = 0;
  bool is_int = false;
  double abs_sum = 0.0;
  int form = QB_FORM_EXACT;
  qb::RecGeom geom{};
  qb::TieRule rule{};
  double eps = 0.0;       // per-state error bound of pass-1 values
  uint64_t rec_begin = 0; // this shard's records [rec_begin, rec_begin + rec_count)
  uint64_t rec_count = 0;
  uint64_t states = 0;
  // Gray form
  int a = 0, b = 0, ubits = 0;
  uint64_t unit_begin = 0, unit_end = 0;
  // TC form
  qb::TcPlan tc{};
};

}  // namespace

struct qb_handle_s {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t st = nullptr;
  DevBuf W, gtab, rec, cand, misc, exout, tcscratch;
  DevBuf bat[15];  // qb_solve_batch: W, insts, gtab items, unit items, selection ids, cands, out, G tables,
                   // records, minima, scaled W, tensor-core items, item ranges, error word
  HostBuf hW, hmisc, hout, hbat;  // hbat: qb_solve_batch's packed W matrices (pinned)
  HostBuf hstage;                  // qb_solve_batch: descriptors and work lists (pinned)
  // qb_solve_batch with QB_FLAG_GRAPH: the captured launch sequence of the last batch and
  // the fingerprint (shapes, options, buffer addresses) it is valid for
  cudaGraphExec_t batch_graph = nullptr;
  std::vector<uint64_t> batch_graph_key;
  int batch_graph_kernels = 0;
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // 4, 5: main kernel
  int64_t h2d = 0, d2h = 0;  // bytes copied by the current call
  float kernel_ms = 0.f;
  int sm_count = 0;
  // state between qb_solve_begin and qb_solve_finish
  bool pending = false;
  Plan plan;
  int kernels = 0;
  float pass1_ms = 0.f;
  double local_min = 0.0;
  int64_t exact_count = 0;  // EXACT form: records evaluated in pass 1
  int cap = kDefaultCap;
  // qb_autotune's choices per (dtype class: 0 float, 1 integer; n); 0 fields = defaults
  struct Tuned {
    int form = 0;
    int tc_gl = 0;
    int tc_pair = 0;  // tensor-core pair form (two states per accumulator)
    int gray_b = 0, gray_sbits = 0;
  };
  Tuned tuned[2][qb::kMaxN + 1];
};

namespace {

int cuda_fail(cudaError_t e) {
  if (e == cudaErrorMemoryAllocation) return QB_ENOMEM;
  return e == cudaSuccess ? QB_OK : QB_ECUDA;
}

#define QB_CUDA(expr)                          \
  do {                                         \
    cudaError_t _e = (expr);                   \
    if (_e != cudaSuccess) return cuda_fail(_e); \
  } while (0)

int dtype_size(int dt) {
  switch (dt) {
    case QB_F32: return 4;
    case QB_F64: return 8;
    case QB_I8: return 1;
    case QB_I16: return 2;
    case QB_I32: return 4;
    case QB_I64: return 8;
    default: return 0;
  }
}

double load_elem(const unsigned char* p, int dt) {
  switch (dt) {
    case QB_F32: { float v; memcpy(&v, p, 4); return v; }
    case QB_F64: { double v; memcpy(&v, p, 8); return v; }
    case QB_I8: { int8_t v; memcpy(&v, p, 1); return v; }
    case QB_I16: { int16_t v; memcpy(&v, p, 2); return v; }
    case QB_I32: { int32_t v; memcpy(&v, p, 4); return v; }
    default: { int64_t v; memcpy(&v, p, 8); return (double)v; }
  }
}

template <class T>
int host_problem_typed(const qb_problem* p, double* Wout, double* abs_sum) {
  const int n = p->n;
  const T* src = static_cast<const T*>(p->q);
  const size_t ld = (size_t)p->ldq;
  double s = 0.0;
  bool bad = false;
  for (int i = 0; i < n; ++i) {
    const T* row = src + i * ld;
    const double d = (double)row[i];
    bad |= !std::isfinite(d);
    s += std::fabs(d);
    Wout[(size_t)i * n + i] = d;
    for (int j = i + 1; j < n; ++j) {
      const double a = (double)row[j], b = (double)src[j * ld + i];
      bad |= !std::isfinite(a) || !std::isfinite(b);
      s += std::fabs(a) + std::fabs(b);
      Wout[(size_t)i * n + j] = Wout[(size_t)j * n + i] = a + b;
    }
  }
  if (bad) return QB_EINVAL;
  *abs_sum = s;
  return QB_OK;
}

// Q in host memory (any dtype) -> W (n x n doubles, written to Wout) and sum |Q_ij|, without
// intermediate copies (the batched search packs thousands of these).
int load_host_problem_into(const qb_problem* p, double* Wout, double* abs_sum, bool* is_int) {
  *is_int = p->dtype >= QB_I8;
  switch (p->dtype) {
    case QB_F32: return host_problem_typed<float>(p, Wout, abs_sum);
    case QB_F64: return host_problem_typed<double>(p, Wout, abs_sum);
    case QB_I8: return host_problem_typed<int8_t>(p, Wout, abs_sum);
    case QB_I16: return host_problem_typed<int16_t>(p, Wout, abs_sum);
    case QB_I32: return host_problem_typed<int32_t>(p, Wout, abs_sum);
    case QB_I64: return host_problem_typed<int64_t>(p, Wout, abs_sum);
    default: return QB_EINVAL;
  }
}

// Q (any dtype, host or device) -> W (n x n doubles) and sum |Q_ij|.
int load_problem(qb_handle* h, const qb_problem* p, std::vector<double>& W, double* abs_sum, bool* is_int) {
  const int n = p->n;
  const int es = dtype_size(p->dtype);
  std::vector<unsigned char> raw((size_t)n * n * es);
  if (p->q_on_device) {
    QB_CUDA(cudaMemcpy2DAsync(raw.data(), (size_t)n * es, p->q, (size_t)p->ldq * es, (size_t)n * es, n,
                              cudaMemcpyDeviceToHost, h->st));
    QB_CUDA(cudaStreamSynchronize(h->st));
    h->d2h += (int64_t)n * n * es;
  } else {
    const unsigned char* src = static_cast<const unsigned char*>(p->q);
    for (int i = 0; i < n; ++i) memcpy(raw.data() + (size_t)i * n * es, src + (size_t)i * p->ldq * es, (size_t)n * es);
  }
  *is_int = p->dtype >= QB_I8;
  W.assign((size_t)n * n, 0.0);
  double s = 0.0;
  std::vector<double> Q((size_t)n * n);
  for (size_t i = 0; i < Q.size(); ++i) {
    double v = load_elem(raw.data() + i * es, p->dtype);
    if (!std::isfinite(v)) return QB_EINVAL;
    Q[i] = v;
    s += std::fabs(v);
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) W[(size_t)i * n + j] = (i == j) ? Q[(size_t)i * n + i] : Q[(size_t)i * n + j] + Q[(size_t)j * n + i];
  *abs_sum = s;
  return QB_OK;
}

int make_rule(const qb_options* o, int n, qb::TieRule* r) {
  r->n = n;
  r->kind = o->tie_rule;
  r->k = r->A = r->B = 0;
  if (o->tie_rule == QB_TIE_QBF) {
    int k = o->fixed_bits;
    if (k < 0 || k >= n + (n == 0)) return QB_EINVAL;
    int m = n - k;
    int A = o->prefix_bits;
    if (A < 0) A = m - std::min(m, 20);
    if (A > m) return QB_EINVAL;
    r->k = k;
    r->A = A;
    r->B = m - A;
  } else if (o->tie_rule == QB_TIE_QB_F1) {
    int k = o->fixed_bits;
    if (k < 0 || n - k < 19) return QB_EINVAL;
    r->k = k;
    r->A = n - k - 18;
    r->B = 18;
  } else if (o->tie_rule != QB_TIE_NATURAL) {
    return QB_EINVAL;
  }
  return QB_OK;
}

void shard_range(uint64_t total, int idx, int cnt, uint64_t* b, uint64_t* e) {
  // contiguous, as even as integer division allows
  unsigned __int128 t = total;
  *b = (uint64_t)(t * (unsigned)idx / (unsigned)cnt);
  *e = (uint64_t)(t * (unsigned)(idx + 1) / (unsigned)cnt);
}

int choose_form(qb_handle* h, const Plan& P, int requested) {
  if (requested == QB_FORM_EXACT) return QB_FORM_EXACT;
  const bool tc_ok = qb::tc_supported(P.n);
  if (requested == QB_FORM_TC) return tc_ok ? QB_FORM_TC : -1;
  if (requested == QB_FORM_GRAY) return P.n >= 20 ? QB_FORM_GRAY : -1;
  // auto
  if (h->tuned[P.is_int ? 1 : 0][P.n].form) return h->tuned[P.is_int ? 1 : 0][P.n].form;
  if (tc_ok) return QB_FORM_TC;
  if (P.n >= 20) return QB_FORM_GRAY;
  return QB_FORM_EXACT;
}

int plan_problem(qb_handle* h, const qb_options* o, Plan& P) {
  const int n = P.n;
  const int shard_idx = o->shard_count > 1 ? o->shard_index : 0;
  const int shard_cnt = o->shard_count > 1 ? o->shard_count : 1;
  int form = choose_form(h, P, o->form);
  if (form < 0) return QB_EINVAL;
  P.form = form;
  P.geom = qb::RecGeom{};
  P.geom.n = n;
  if (form == QB_FORM_EXACT) {
    int f = std::min(n, 16);
    P.geom.kind = qb::kGeomBlock;
    P.geom.fbits = f;
    uint64_t total = 1ull << (n - f);
    uint64_t rb, re;
    shard_range(total, shard_idx, shard_cnt, &rb, &re);
    P.rec_begin = rb;
    P.rec_count = re - rb;
    P.states = P.rec_count << f;
    P.eps = 0.0;
    return QB_OK;
  }
  const qb_handle::Tuned& T = h->tuned[P.is_int ? 1 : 0][n];
  if (form == QB_FORM_GRAY) {
    const GrayShape gs = gray_shape(n, T.gray_b, T.gray_sbits);
    const int a = gs.a, b = gs.b, cbbits = gs.cbbits, sbits = gs.sbits, ubits = gs.ubits;
    P.a = a;
    P.b = b;
    P.ubits = ubits;
    P.geom.kind = qb::kGeomGray;
    P.geom.a = a;
    P.geom.b = b;
    P.geom.sbits = sbits;
    P.geom.cbbits = cbbits;
    P.geom.gubits = ubits - sbits;
    uint64_t units = 1ull << (a - ubits + cbbits);
    shard_range(units, shard_idx, shard_cnt, &P.unit_begin, &P.unit_end);
    P.rec_begin = P.unit_begin << (P.geom.gubits + 3);
    P.rec_count = (P.unit_end - P.unit_begin) << (P.geom.gubits + 3);
    P.states = (P.unit_end - P.unit_begin) << (ubits + 13);
    P.eps = (P.is_int && P.abs_sum < kTwo24) ? 0.0 : qb::gray_error_bound(P.abs_sum);
    return QB_OK;
  }
  // tensor-core form
  qb::tc_plan(n, P.is_int, P.abs_sum, shard_idx, shard_cnt, &P.tc, T.tc_gl);
  P.tc.stall = (o->flags & QB_FLAG_TEST_STALL) != 0;
  if ((o->flags & QB_FLAG_TC_PAIR) && (o->flags & QB_FLAG_TC_ONE)) return QB_EINVAL;
  P.tc.pair = (o->flags & QB_FLAG_TC_PAIR) != 0 || (!(o->flags & QB_FLAG_TC_ONE) && T.tc_pair);
  if (P.tc.pair && !P.tc.exact) P.tc.eps = qb::tc2_error_bound(P.abs_sum);
  P.geom.kind = qb::kGeomTC;
  P.geom.gl = P.tc.gl;
  P.rec_begin = P.tc.rec_begin;
  P.rec_count = P.tc.rec_count;
  P.states = P.tc.states;
  P.eps = P.tc.eps;
  return QB_OK;
}

// the plan parameters a result reports
void fill_plan_fields(const qb_handle* h, const Plan& P, qb_result* r) {
  const qb_handle::Tuned& T = h->tuned[P.is_int ? 1 : 0][P.n];
  if (P.form == QB_FORM_GRAY) {
    r->rec_log2 = P.geom.sbits;
    r->suffix_bits = P.b;
    r->unit_log2 = P.ubits;
    r->tuned = (T.gray_b || T.gray_sbits) ? 1 : 0;
  } else if (P.form == QB_FORM_TC) {
    r->rec_log2 = P.tc.gl;
    r->suffix_bits = 15;
    r->unit_log2 = 0;
    r->tuned = T.tc_gl ? 1 : 0;
  } else {
    r->rec_log2 = P.geom.fbits;
    r->suffix_bits = 0;
    r->unit_log2 = 0;
    r->tuned = 0;
  }
  if (T.form && T.form == P.form) r->tuned = 1;
  r->tc_kernel = P.form != QB_FORM_TC ? 0 : (P.tc.pair ? (P.tc.u16 ? 4 : 2) : (P.tc.u16 ? 3 : 1));
}

int upload_W(qb_handle* h, const std::vector<double>& W) {
  size_t bytes = W.size() * sizeof(double);
  QB_CUDA(h->hW.ensure(bytes));
  QB_CUDA(h->W.ensure(bytes));
  memcpy(h->hW.p, W.data(), bytes);
  QB_CUDA(cudaMemcpyAsync(h->W.p, h->hW.p, bytes, cudaMemcpyHostToDevice, h->st));
  h->h2d += (int64_t)bytes;
  return QB_OK;
}

int run_pass1(qb_handle* h, Plan& P) {
  const qb::ProblemDev pd{P.n, static_cast<const double*>(h->W.p)};
  if (P.form == QB_FORM_EXACT) {
    QB_CUDA(h->exout.ensure(std::max<uint64_t>(P.rec_count, 1) * sizeof(qb::ExactOut)));
    size_t sm = qb::exact_smem_bytes(P.n, P.geom.fbits);
    QB_CUDA(cudaFuncSetAttribute(qb::exact_records_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    // chunked over the grid limit
    const uint64_t maxg = 1u << 30;
    QB_CUDA(cudaEventRecord(h->ev[4], h->st));
    for (uint64_t off = 0; off < P.rec_count; off += maxg) {
      uint64_t g = std::min<uint64_t>(maxg, P.rec_count - off);
      qb::exact_records_kernel<<<(unsigned)g, qb::kExactThreads, sm, h->st>>>(
          pd, P.rule, P.geom, nullptr, nullptr, (int64_t)(P.rec_begin + P.rec_count), (int64_t)(P.rec_begin + off),
          static_cast<qb::ExactOut*>(h->exout.p) + off, 0);
      ++h->kernels;
    }
    QB_CUDA(cudaEventRecord(h->ev[5], h->st));
    QB_CUDA(cudaGetLastError());
    return QB_OK;
  }
  QB_CUDA(h->rec.ensure(std::max<uint64_t>(P.rec_count, 1) * sizeof(float)));
  if (P.form == QB_FORM_GRAY) {
    QB_CUDA(h->gtab.ensure(((size_t)1 << P.a) * 32 * sizeof(float)));
    size_t sm0 = qb::gray_gtab_smem(P.n, P.a);
    QB_CUDA(cudaFuncSetAttribute(qb::gray_gtab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm0));
    unsigned gblocks = (unsigned)std::min<uint64_t>((1ull << P.a) / 8 + 1, (uint64_t)h->sm_count * 4);
    qb::gray_gtab_kernel<<<gblocks, 256, sm0, h->st>>>(pd, P.a, P.b, static_cast<float*>(h->gtab.p));
    ++h->kernels;
    qb::GrayParams gp{};
    gp.P = pd;
    gp.a = P.a;
    gp.b = P.b;
    gp.cbbits = P.geom.cbbits;
    gp.sbits = P.geom.sbits;
    gp.gubits = P.geom.gubits;
    gp.unit_begin = P.unit_begin;
    gp.gtab = static_cast<const float*>(h->gtab.p);
    gp.rec = static_cast<float*>(h->rec.p);
    size_t sm = qb::gray_pass1_smem(P.n, P.a);
    QB_CUDA(cudaFuncSetAttribute(qb::gray_pass1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    uint64_t units = P.unit_end - P.unit_begin;
    QB_CUDA(cudaEventRecord(h->ev[4], h->st));
    if (units) {
      qb::gray_pass1_kernel<<<(unsigned)units, qb::kGrayThreads, sm, h->st>>>(gp);
      ++h->kernels;
    }
    QB_CUDA(cudaEventRecord(h->ev[5], h->st));
    QB_CUDA(cudaGetLastError());
    return QB_OK;
  }
  QB_CUDA(h->tcscratch.ensure(qb::tc_scratch_bytes(P.tc)));
  int rc = qb::tc_prepare(P.tc, pd, h->tcscratch.p, h->st, &h->kernels);
  if (rc) return rc;
  QB_CUDA(cudaEventRecord(h->ev[4], h->st));
  rc = P.tc.pair ? qb::tc2_launch(P.tc, P.tc.gamma, static_cast<float*>(h->rec.p), h->tcscratch.p, h->st,
                                  h->sm_count, &h->kernels)
                 : qb::tc_launch(P.tc, static_cast<float*>(h->rec.p), h->tcscratch.p, h->st, h->sm_count, &h->kernels);
  if (rc) return rc;
  QB_CUDA(cudaEventRecord(h->ev[5], h->st));
  return QB_OK;
}

}  // namespace

extern "C" {

int qb_version(void) { return 100; }

const char* qb_strerror(int s) {
  switch (s) {
    case QB_OK: return "ok";
    case QB_EINVAL: return "invalid argument";
    case QB_ERANGE: return "Q magnitude out of the exact range (sum |Q| must be < 2^53)";
    case QB_ENOMEM: return "device memory allocation failed";
    case QB_ECUDA: return "CUDA runtime error";
    case QB_ETIMEOUT: return "a bounded wait inside a kernel timed out";
    case QB_ENODEV: return "no such CUDA device";
    case QB_EOVERFLOW: return "too many candidate records";
    case QB_ETOOBIG: return "problem larger than the fixed no-allocation scratch (qb_solve_noalloc: 20 <= n <= 36)";
    default: return "unknown status";
  }
}

int qb_handle_create(int device, qb_handle** out) {
  if (!out) return QB_EINVAL;
  *out = nullptr;
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt <= 0) {
    cudaGetLastError();
    return QB_ENODEV;
  }
  if (device < 0 || device >= cnt) return QB_ENODEV;
  QB_CUDA(cudaSetDevice(device));
  qb_handle* h = new qb_handle_s();
  h->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking);
  for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&h->ev[i]);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    qb_handle_destroy(h);
    return cuda_fail(e);
  }
  h->st = h->own;
  *out = h;
  return QB_OK;
}

int qb_handle_destroy(qb_handle* h) {
  if (!h) return QB_EINVAL;
  cudaSetDevice(h->device);
  if (h->own) cudaStreamSynchronize(h->own);
  h->W.release();
  h->gtab.release();
  h->rec.release();
  h->cand.release();
  h->misc.release();
  h->exout.release();
  h->tcscratch.release();
  for (auto& b : h->bat) b.release();
  h->hW.release();
  h->hmisc.release();
  h->hout.release();
  h->hbat.release();
  h->hstage.release();
  if (h->batch_graph) cudaGraphExecDestroy(h->batch_graph);
  for (auto& ev : h->ev)
    if (ev) cudaEventDestroy(ev);
  if (h->own) cudaStreamDestroy(h->own);
  delete h;
  return QB_OK;
}

}  // extern "C"

namespace {

// validation, problem upload and the pass-1 launch of qb_solve_begin
int begin_launch(qb_handle* h, const qb_problem* p, const qb_options* o, Plan& P) {
  if (p->n < 1 || p->n > qb::kMaxN || !p->q || p->ldq < p->n || dtype_size(p->dtype) == 0) return QB_EINVAL;
  if (o->shard_count > 1 && (o->shard_index < 0 || o->shard_index >= o->shard_count)) return QB_EINVAL;
  QB_CUDA(cudaSetDevice(h->device));
  h->st = o->stream ? static_cast<cudaStream_t>(o->stream) : h->own;
  h->pending = false;
  h->kernels = 0;
  h->h2d = h->d2h = 0;
  h->cap = o->max_candidates > 0 ? o->max_candidates : kDefaultCap;
  P.n = p->n;
  std::vector<double> W;
  int rc = load_problem(h, p, W, &P.abs_sum, &P.is_int);
  if (rc) return rc;
  if (P.abs_sum >= kTwo53) return QB_ERANGE;
  rc = make_rule(o, P.n, &P.rule);
  if (rc) return rc;
  rc = plan_problem(h, o, P);
  if (rc) return rc;
  if (P.form == QB_FORM_TC) {  // pair form: couplings of variable n-16 with the u variables
    for (int j = 0; j < 8; ++j) P.tc.gamma[j] = (float)(W[(size_t)(P.n - 16) * P.n + (P.n - 1 - j)] * P.tc.scale);
    const bool no16 = (o->flags & QB_FLAG_TC_NO16) != 0;
    // default kernel where neither a flag nor the tuned entry names one: the 16-bit pair form
    // wherever it applies (the fastest measured), else one state per accumulator
    const qb_handle::Tuned& T = h->tuned[P.is_int ? 1 : 0][P.n];
    // off the exact path (float Q, or integer Q beyond 2^22): the 16-bit pair form on values
    // rounded to integers in units of 1/sigma, with its error bound, where it applies and the
    // pair form is the default, requested or tuned
    double sg = 0.0, qeps = 0.0;
    float qdmin = 0.f;
    const bool want_pair = P.tc.pair || (!(o->flags & QB_FLAG_TC_ONE) && T.form != QB_FORM_TC);
    if (!P.tc.exact && !no16 && want_pair && qb::tc2_u16_quantized(P.n, W.data(), P.abs_sum, &sg, &qdmin, &qeps)) {
      P.tc.pair = P.tc.u16 = true;
      P.tc.scale = sg;
      P.tc.dmin = qdmin;
      P.tc.eps = P.eps = qeps;
      for (int j = 0; j < 8; ++j) P.tc.gamma[j] = (float)(W[(size_t)(P.n - 16) * P.n + (P.n - 1 - j)] * sg);
    } else {
      if (!P.tc.pair && P.tc.exact && !no16 && !(o->flags & QB_FLAG_TC_ONE) && T.form != QB_FORM_TC)
        P.tc.pair = qb::tc2_u16_eligible(P.n, W.data(), &P.tc.dmin);
      P.tc.u16 = P.tc.exact && !no16 &&
                 (P.tc.pair ? qb::tc2_u16_eligible(P.n, W.data(), &P.tc.dmin) : qb::tc_u16_eligible(P.n, W.data(), &P.tc.dmin));
    }
  }
  rc = upload_W(h, W);
  if (rc) return rc;
  QB_CUDA(h->misc.ensure(64));
  QB_CUDA(h->hmisc.ensure(64));
  QB_CUDA(cudaEventRecord(h->ev[0], h->st));
  return run_pass1(h, P);
}

// the rest of qb_solve_begin: the pass-1 minimum on the host
int begin_finish_pass1(qb_handle* h, Plan& P, double* local_min) {
  double lmin = INFINITY;
  if (P.form == QB_FORM_EXACT) {
    QB_CUDA(cudaEventRecord(h->ev[1], h->st));
    size_t bytes = P.rec_count * sizeof(qb::ExactOut);
    QB_CUDA(h->hout.ensure(std::max<size_t>(bytes, 64)));
    if (bytes) QB_CUDA(cudaMemcpyAsync(h->hout.p, h->exout.p, bytes, cudaMemcpyDeviceToHost, h->st));
    h->d2h += (int64_t)bytes;
    QB_CUDA(cudaStreamSynchronize(h->st));
    const qb::ExactOut* eo = static_cast<const qb::ExactOut*>(h->hout.p);
    for (uint64_t i = 0; i < P.rec_count; ++i) lmin = std::min(lmin, eo[i].e);
    h->exact_count = (int64_t)P.rec_count;
  } else {
    uint32_t* mk = static_cast<uint32_t*>(h->misc.p);
    QB_CUDA(cudaMemsetAsync(mk, 0xff, sizeof(uint32_t), h->st));
    if (P.rec_count) {
      unsigned blocks = (unsigned)std::min<uint64_t>((P.rec_count + 255) / 256, (uint64_t)h->sm_count * 8);
      qb::rec_min_kernel<<<blocks, 256, 0, h->st>>>(static_cast<const float*>(h->rec.p), (int64_t)P.rec_count, mk);
      ++h->kernels;
      QB_CUDA(cudaGetLastError());
    }
    QB_CUDA(cudaEventRecord(h->ev[1], h->st));
    QB_CUDA(cudaMemcpyAsync(h->hmisc.p, mk, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st));
    h->d2h += (int64_t)sizeof(uint32_t);
    QB_CUDA(cudaStreamSynchronize(h->st));
    if (P.form == QB_FORM_TC) {
      int trc = qb::tc_check_error(h->tcscratch.p, h->st);
      h->d2h += (int64_t)sizeof(unsigned);
      if (trc) return trc;
    }
    uint32_t key = *static_cast<uint32_t*>(h->hmisc.p);
    lmin = (P.rec_count && key != 0xffffffffu) ? (double)qb::key2f(key) : INFINITY;
  }
  QB_CUDA(cudaEventElapsedTime(&h->pass1_ms, h->ev[0], h->ev[1]));
  QB_CUDA(cudaEventElapsedTime(&h->kernel_ms, h->ev[4], h->ev[5]));
  h->plan = P;
  h->local_min = lmin;
  h->pending = true;
  *local_min = lmin;
  return QB_OK;
}

// qb_solve of one whole problem (Gray or tensor-core form, QB_TIE_QBF / QB_TIE_NATURAL):
// minimum, threshold, selection, exact re-evaluation and the final pick all on the device,
// then one copy of the answer to the host.  Returns -1 when the candidates overflow the cap
// (the caller then takes the two-phase path with a larger cap).
int solve_fused(qb_handle* h, const Plan& P, qb_result* r) {
  char* m = static_cast<char*>(h->misc.p);  // [0] min key, [8] thr, [16] flag, [20] count, [24] best
  uint32_t* mk = reinterpret_cast<uint32_t*>(m);
  double* thr = reinterpret_cast<double*>(m + 8);
  int* flag = reinterpret_cast<int*>(m + 16);
  int* count = reinterpret_cast<int*>(m + 20);
  qb::ExactOut* best = reinterpret_cast<qb::ExactOut*>(m + 24);
  const unsigned* err = P.form == QB_FORM_TC ? static_cast<const unsigned*>(h->tcscratch.p) : nullptr;
  QB_CUDA(cudaMemsetAsync(mk, 0xff, sizeof(uint32_t), h->st));
  if (P.rec_count) {
    const unsigned blocks = (unsigned)std::min<uint64_t>((P.rec_count + 255) / 256, (uint64_t)h->sm_count * 8);
    qb::rec_min_kernel<<<blocks, 256, 0, h->st>>>(static_cast<const float*>(h->rec.p), (int64_t)P.rec_count, mk);
    ++h->kernels;
  }
  QB_CUDA(cudaEventRecord(h->ev[1], h->st));
  QB_CUDA(cudaEventRecord(h->ev[2], h->st));
  qb::rec_threshold_kernel<<<1, 1, 0, h->st>>>(mk, P.eps, P.is_int ? 1 : 0, err, thr, flag, count);
  QB_CUDA(h->cand.ensure((size_t)h->cap * sizeof(uint64_t)));
  if (P.rec_count) {
    const unsigned blocks = (unsigned)std::min<uint64_t>((P.rec_count + 255) / 256, (uint64_t)h->sm_count * 8);
    qb::rec_select_dev_kernel<<<blocks, 256, 0, h->st>>>(static_cast<const float*>(h->rec.p), (int64_t)P.rec_count,
                                                         (int64_t)P.rec_begin, thr, flag,
                                                         static_cast<uint64_t*>(h->cand.p), count, h->cap);
  }
  int maxf = 0;
  {
    uint64_t b, f;
    qb::record_states(P.geom, 0, &b, &f);
    maxf = __builtin_popcountll(f & qb::mask64(P.n));
  }
  if (maxf > qb::kExactMaxFree) return QB_EINVAL;
  const int sb = std::max(0, std::min(4, maxf - 12));
  QB_CUDA(h->exout.ensure(((size_t)h->cap << sb) * sizeof(qb::ExactOut)));
  const qb::ProblemDev pd{P.n, static_cast<const double*>(h->W.p)};
  const size_t sm = qb::exact_smem_bytes(P.n, maxf);
  QB_CUDA(cudaFuncSetAttribute(qb::exact_candidates_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  qb::exact_candidates_kernel<<<(unsigned)(2 * h->sm_count), qb::kExactThreads, sm, h->st>>>(
      pd, P.rule, P.geom, static_cast<const uint64_t*>(h->cand.p), count, h->cap, sb,
      static_cast<qb::ExactOut*>(h->exout.p));
  qb::exact_final_kernel<<<1, 256, 0, h->st>>>(static_cast<const qb::ExactOut*>(h->exout.p), count, h->cap, sb, flag,
                                               best);
  h->kernels += 4;
  QB_CUDA(cudaGetLastError());
  QB_CUDA(cudaEventRecord(h->ev[3], h->st));
  QB_CUDA(cudaMemcpyAsync(h->hmisc.p, m, 48, cudaMemcpyDeviceToHost, h->st));
  h->d2h += 48;
  unsigned herr = 0;
  if (err) {
    QB_CUDA(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, h->st));
    h->d2h += (int64_t)sizeof(unsigned);
  }
  QB_CUDA(cudaStreamSynchronize(h->st));
  if (herr & qb::kErrTimeout) return QB_ETIMEOUT;
  const char* hm = static_cast<const char*>(h->hmisc.p);
  const uint32_t key = *reinterpret_cast<const uint32_t*>(hm);
  const int zero = *reinterpret_cast<const int*>(hm + 16);
  const int cnt = *reinterpret_cast<const int*>(hm + 20);
  if (!zero && cnt > h->cap) return -1;
  const qb::ExactOut b = *reinterpret_cast<const qb::ExactOut*>(hm + 24);
  const bool found = zero ? (P.rec_begin == 0 && P.rec_count > 0) : cnt > 0;
  memset(r, 0, sizeof(*r));
  r->form_used = P.form;
  r->is_integer = P.is_int ? 1 : 0;
  r->pass1_min = (P.rec_count && key != 0xffffffffu) ? (double)qb::key2f(key) : INFINITY;
  r->err_bound = P.eps;
  r->states = (int64_t)P.states;
  r->candidate_records = zero ? 0 : cnt;
  QB_CUDA(cudaEventElapsedTime(&r->pass1_ms, h->ev[0], h->ev[1]));
  QB_CUDA(cudaEventElapsedTime(&r->pass2_ms, h->ev[2], h->ev[3]));
  QB_CUDA(cudaEventElapsedTime(&r->kernel_ms, h->ev[4], h->ev[5]));
  r->found = found ? 1 : 0;
  r->best_x = b.x;
  r->best_e = found ? b.e : INFINITY;
  r->best_e_int = (found && P.is_int) ? (int64_t)llround(b.e) : 0;
  r->order_key = b.key;
  r->kernels = h->kernels;
  r->h2d_bytes = h->h2d;
  r->d2h_bytes = h->d2h;
  fill_plan_fields(h, P, r);
  r->status = QB_OK;
  return QB_OK;
}

}  // namespace

extern "C" {

int qb_solve_begin(qb_handle* h, const qb_problem* p, const qb_options* o, double* local_min) {
  if (!h || !p || !o || !local_min) return QB_EINVAL;
  Plan P;
  int rc = begin_launch(h, p, o, P);
  if (rc) return rc;
  return begin_finish_pass1(h, P, local_min);
}

namespace {

// Exact re-evaluation of `count` candidate records listed in h->cand (device).
int rescore(qb_handle* h, const Plan& P, const qb::TieRule& rule, const qb::RecGeom& geom, int count,
            std::vector<qb::ExactOut>& out) {
  out.clear();
  if (count <= 0) return QB_OK;
  int maxf = 0;
  {
    uint64_t b, f;
    qb::record_states(geom, 0, &b, &f);
    maxf = __builtin_popcountll(f & qb::mask64(P.n));
  }
  if (maxf > qb::kExactMaxFree) return QB_EINVAL;
  const qb::ProblemDev pd{P.n, static_cast<const double*>(h->W.p)};
  // few candidate records: split each over several CTAs (at least 2^12 states per CTA)
  int sb = 0;
  while (sb < maxf - 12 && ((int64_t)count << (sb + 1)) <= 2 * (int64_t)h->sm_count) ++sb;
  const size_t nout = (size_t)count << sb;
  QB_CUDA(h->exout.ensure(nout * sizeof(qb::ExactOut)));
  size_t sm = qb::exact_smem_bytes(P.n, maxf);
  QB_CUDA(cudaFuncSetAttribute(qb::exact_records_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  qb::exact_records_kernel<<<(unsigned)nout, qb::kExactThreads, sm, h->st>>>(
      pd, rule, geom, static_cast<const uint64_t*>(h->cand.p), nullptr, count, 0,
      static_cast<qb::ExactOut*>(h->exout.p), sb);
  ++h->kernels;
  QB_CUDA(cudaGetLastError());
  QB_CUDA(h->hout.ensure(nout * sizeof(qb::ExactOut)));
  QB_CUDA(cudaMemcpyAsync(h->hout.p, h->exout.p, nout * sizeof(qb::ExactOut), cudaMemcpyDeviceToHost, h->st));
  h->d2h += (int64_t)(nout * sizeof(qb::ExactOut));
  QB_CUDA(cudaStreamSynchronize(h->st));
  const qb::ExactOut* eo = static_cast<const qb::ExactOut*>(h->hout.p);
  // the lexicographic minimum over each record's parts
  out.resize(count);
  for (int c = 0; c < count; ++c) {
    qb::ExactOut b = eo[(size_t)c << sb];
    for (int q = 1; q < (1 << sb); ++q) {
      const qb::ExactOut& o = eo[((size_t)c << sb) + q];
      if (o.e < b.e || (o.e == b.e && o.key < b.key)) b = o;
    }
    out[c] = b;
  }
  return QB_OK;
}

bool lex_less_h(const qb::ExactOut& a, const qb::ExactOut& b) {
  return a.e < b.e || (a.e == b.e && a.key < b.key);
}

// QB_F1 rule, final step: smallest 18-bit suffix of the winning prefix with E == e_star.
int qbf1_row(qb_handle* h, const Plan& P, uint64_t X, double e_star, uint64_t* Xout) {
  qb::RecGeom g{};
  g.kind = qb::kGeomBlock;
  g.n = P.n;
  g.fbits = 18;
  qb::TieRule nat{qb::kTieNatural, P.n, 0, 0, 0};
  uint64_t rid = X >> 18;
  QB_CUDA(h->cand.ensure(sizeof(uint64_t)));
  QB_CUDA(cudaMemcpyAsync(h->cand.p, &rid, sizeof(uint64_t), cudaMemcpyHostToDevice, h->st));
  h->h2d += (int64_t)sizeof(uint64_t);
  std::vector<qb::ExactOut> o;
  int rc = rescore(h, P, nat, g, 1, o);
  if (rc) return rc;
  if (o.empty() || o[0].e != e_star) return QB_ECUDA;
  *Xout = o[0].x;
  return QB_OK;
}

}  // namespace

int qb_solve_finish(qb_handle* h, double global_min, qb_result* r) {
  if (!h || !r) return QB_EINVAL;
  if (!h->pending) return QB_EINVAL;
  h->pending = false;
  Plan& P = h->plan;
  memset(r, 0, sizeof(*r));
  r->form_used = P.form;
  r->is_integer = P.is_int ? 1 : 0;
  r->pass1_min = h->local_min;
  r->err_bound = P.eps;
  r->states = (int64_t)P.states;
  r->pass1_ms = h->pass1_ms;
  QB_CUDA(cudaSetDevice(h->device));
  QB_CUDA(cudaEventRecord(h->ev[2], h->st));
  qb::ExactOut best{INFINITY, ~0ull, 0};
  bool found = false;
  if (P.form == QB_FORM_EXACT) {
    const qb::ExactOut* eo = static_cast<const qb::ExactOut*>(h->hout.p);
    for (int64_t i = 0; i < h->exact_count; ++i)
      if (lex_less_h(eo[i], best)) best = eo[i];
    found = h->exact_count > 0 && best.e == global_min;
    r->candidate_records = 0;
  } else if (P.is_int && P.eps == 0.0 && global_min >= 0.0) {
    // E(0) = 0 is minimal and X = 0 has the smallest key under every rule
    found = P.rec_begin == 0 && P.rec_count > 0;
    best = qb::ExactOut{0.0, 0ull, 0ull};
  } else {
    double thr = global_min + 2.0 * P.eps;
    if (P.eps > 0.0) thr += std::fabs(thr) * 1e-12;
    int* cnt = reinterpret_cast<int*>(static_cast<char*>(h->misc.p) + 16);
    int count = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      QB_CUDA(h->cand.ensure((size_t)h->cap * sizeof(uint64_t)));
      QB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), h->st));
      if (P.rec_count) {
        unsigned blocks = (unsigned)std::min<uint64_t>((P.rec_count + 255) / 256, (uint64_t)h->sm_count * 8);
        qb::rec_select_kernel<<<blocks, 256, 0, h->st>>>(static_cast<const float*>(h->rec.p), (int64_t)P.rec_count,
                                                          (int64_t)P.rec_begin, thr, static_cast<uint64_t*>(h->cand.p),
                                                          cnt, h->cap);
        ++h->kernels;
        QB_CUDA(cudaGetLastError());
      }
      QB_CUDA(cudaMemcpyAsync(h->hmisc.p, cnt, sizeof(int), cudaMemcpyDeviceToHost, h->st));
      h->d2h += (int64_t)sizeof(int);
      QB_CUDA(cudaStreamSynchronize(h->st));
      count = *static_cast<int*>(h->hmisc.p);
      if (count <= h->cap) break;
      if (count > (1 << 24)) return QB_EOVERFLOW;
      h->cap = count;
    }
    if (count > h->cap) return QB_EOVERFLOW;
    std::vector<qb::ExactOut> outs;
    int rc = rescore(h, P, P.rule, P.geom, count, outs);
    if (rc) return rc;
    for (auto& e : outs)
      if (lex_less_h(e, best)) best = e;
    found = count > 0;
    r->candidate_records = count;
  }
  if (found && P.rule.kind == qb::kTieQBF1 && best.x != 0) {
    uint64_t X;
    int rc = qbf1_row(h, P, best.x, best.e, &X);
    if (rc) return rc;
    best.x = X;
  }
  QB_CUDA(cudaEventRecord(h->ev[3], h->st));
  QB_CUDA(cudaEventSynchronize(h->ev[3]));
  float ms2 = 0.f;
  QB_CUDA(cudaEventElapsedTime(&ms2, h->ev[2], h->ev[3]));
  r->pass2_ms = ms2;
  r->found = found ? 1 : 0;
  r->best_x = best.x;
  r->best_e = found ? best.e : INFINITY;
  r->best_e_int = (found && P.is_int) ? (int64_t)llround(best.e) : 0;
  r->order_key = best.key;
  r->kernels = h->kernels;
  r->kernel_ms = h->kernel_ms;
  r->h2d_bytes = h->h2d;
  r->d2h_bytes = h->d2h;
  fill_plan_fields(h, P, r);
  r->status = QB_OK;
  return QB_OK;
}

}  // extern "C"

namespace {

// QB_F1 with the reference's int16 arithmetic (QB_FLAG_INT16_WRAP; qb_qbf1.cuh).
int qbf1_wrap_solve(qb_handle* h, const qb_problem* p, const qb_options* o, qb_result* r) {
  memset(r, 0, sizeof(*r));
  const int n = p->n;
  if (p->dtype != QB_I16 || n < 19 || n > qb::kQbf1MaxN || o->fixed_bits != 0 || o->shard_count > 1 ||
      p->ldq < n || !p->q)
    return QB_EINVAL;
  QB_CUDA(cudaSetDevice(h->device));
  h->st = o->stream ? static_cast<cudaStream_t>(o->stream) : h->own;
  h->pending = false;
  h->kernels = 0;
  h->h2d = h->d2h = 0;
  // the int16 matrix, as int32
  std::vector<int16_t> raw((size_t)n * n);
  if (p->q_on_device) {
    QB_CUDA(cudaMemcpy2DAsync(raw.data(), (size_t)n * 2, p->q, (size_t)p->ldq * 2, (size_t)n * 2, n,
                              cudaMemcpyDeviceToHost, h->st));
    QB_CUDA(cudaStreamSynchronize(h->st));
    h->d2h += (int64_t)n * n * 2;
  } else {
    const int16_t* src = static_cast<const int16_t*>(p->q);
    for (int i = 0; i < n; ++i) memcpy(raw.data() + (size_t)i * n, src + (size_t)i * p->ldq, (size_t)n * 2);
  }
  std::vector<int> Qi(raw.begin(), raw.end());
  const int A = n - qb::kQbf1B;
  const uint64_t steps = 1ull << A;
  const size_t cols = (size_t)1 << qb::kQbf1B;
  DevBuf* B = h->bat;
  QB_CUDA(B[0].ensure(Qi.size() * sizeof(int)));
  QB_CUDA(B[6].ensure(cols * sizeof(short)));
  QB_CUDA(B[7].ensure((size_t)A * cols * sizeof(short)));
  QB_CUDA(B[8].ensure(steps * sizeof(short)));
  QB_CUDA(B[9].ensure((qb::kQbf1Threads + 1) * sizeof(unsigned long long)));
  QB_CUDA(cudaMemcpyAsync(B[0].p, Qi.data(), Qi.size() * sizeof(int), cudaMemcpyHostToDevice, h->st));
  h->h2d += (int64_t)(Qi.size() * sizeof(int));
  const int* dQ = static_cast<const int*>(B[0].p);
  short* BB = static_cast<short*>(B[6].p);
  short* ABBA = static_cast<short*>(B[7].p);
  short* AA = static_cast<short*>(B[8].p);
  unsigned long long* key = static_cast<unsigned long long*>(B[9].p);
  QB_CUDA(cudaMemsetAsync(key, 0xff, (qb::kQbf1Threads + 1) * sizeof(unsigned long long), h->st));
  QB_CUDA(cudaEventRecord(h->ev[0], h->st));
  qb::qbf1w_tables_kernel<<<(unsigned)(cols / 256), 256, (size_t)n * n * sizeof(int), h->st>>>(dQ, n, A, BB, ABBA);
  qb::qbf1w_prefix_kernel<<<(unsigned)std::min<uint64_t>((steps + 255) / 256, (uint64_t)h->sm_count * 8), 256,
                            (size_t)A * A * sizeof(int), h->st>>>(dQ, n, A, AA);
  const uint64_t nchunks = std::min<uint64_t>(64, std::max<uint64_t>(4, steps));
  const uint64_t chunk_len = (steps + nchunks - 1) / nchunks;
  const size_t sm = qb::qbf1w_search_smem(A);
  QB_CUDA(cudaFuncSetAttribute(qb::qbf1w_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  QB_CUDA(cudaEventRecord(h->ev[4], h->st));
  qb::qbf1w_search_kernel<<<dim3(qb::kQbf1Threads / 64, (unsigned)(nchunks / 4)), 256, sm, h->st>>>(
      A, BB, ABBA, AA, chunk_len, key);
  QB_CUDA(cudaEventRecord(h->ev[5], h->st));
  h->kernels += 3;
  QB_CUDA(cudaGetLastError());
  QB_CUDA(h->hout.ensure(qb::kQbf1Threads * sizeof(unsigned long long)));
  QB_CUDA(cudaMemcpyAsync(h->hout.p, key, qb::kQbf1Threads * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          h->st));
  h->d2h += (int64_t)qb::kQbf1Threads * 8;
  QB_CUDA(cudaStreamSynchronize(h->st));
  // the host's argmin over the threads' best values: the lowest thread among equals
  const unsigned long long* hk = static_cast<const unsigned long long*>(h->hout.p);
  int tid = 0;
  for (int i = 1; i < qb::kQbf1Threads; ++i)
    if ((hk[i] >> 40) < (hk[tid] >> 40)) tid = i;
  if (hk[tid] == ~0ull) return QB_ECUDA;
  const int best16 = (int)(hk[tid] >> 40) - 32768;
  const uint64_t step = hk[tid] & ((1ull << 40) - 1);
  const uint64_t prefix = qb::gray64(step);
  qb::qbf1w_row_kernel<<<(unsigned)(cols / 256), 256, 0, h->st>>>(A, BB, ABBA, prefix, key + qb::kQbf1Threads);
  ++h->kernels;
  QB_CUDA(cudaGetLastError());
  QB_CUDA(cudaEventRecord(h->ev[1], h->st));
  QB_CUDA(cudaMemcpyAsync(h->hmisc.p, key + qb::kQbf1Threads, 8, cudaMemcpyDeviceToHost, h->st));
  h->d2h += 8;
  QB_CUDA(cudaStreamSynchronize(h->st));
  const uint64_t sfx = *static_cast<const unsigned long long*>(h->hmisc.p) & 0xffffffffull;
  const uint64_t X = (prefix << qb::kQbf1B) | sfx;
  double e = 0.0;  // exact energy of the reported state
  for (int i = 0; i < n; ++i) {
    if (!((X >> (n - 1 - i)) & 1)) continue;
    for (int j = 0; j < n; ++j)
      if ((X >> (n - 1 - j)) & 1) e += Qi[(size_t)i * n + j];
  }
  float p1 = 0.f, km = 0.f;
  QB_CUDA(cudaEventElapsedTime(&p1, h->ev[0], h->ev[1]));
  QB_CUDA(cudaEventElapsedTime(&km, h->ev[4], h->ev[5]));
  r->best_x = X;
  r->best_e = e;
  r->best_e_int = best16;  // the value the reference reports (its int16 running sum)
  r->order_key = ((uint64_t)tid << 40) | step;
  r->pass1_min = (double)best16;
  r->states = (int64_t)1 << n;
  r->form_used = QB_FORM_QBF1_INT16;
  r->is_integer = 1;
  r->found = 1;
  r->status = QB_OK;
  r->pass1_ms = p1;
  r->kernels = h->kernels;
  r->kernel_ms = km;
  r->h2d_bytes = h->h2d;
  r->d2h_bytes = h->d2h;
  return QB_OK;
}

}  // namespace

extern "C" {

int qb_solve(qb_handle* h, const qb_problem* p, const qb_options* o, qb_result* r) {
  if (!r) return QB_EINVAL;
  if (h && p && o && (o->flags & QB_FLAG_INT16_WRAP)) {
    if (o->tie_rule != QB_TIE_QB_F1) return QB_EINVAL;
    QB_CUDA(h->hmisc.ensure(64));
    const int rc = qbf1_wrap_solve(h, p, o, r);
    if (rc) r->status = rc;
    return rc;
  }
  if (!h || !p || !o) {
    memset(r, 0, sizeof(*r));
    r->status = QB_EINVAL;
    return QB_EINVAL;
  }
  Plan P;
  int rc = begin_launch(h, p, o, P);
  if (rc) {
    memset(r, 0, sizeof(*r));
    r->status = rc;
    return rc;
  }
  if (o->shard_count <= 1 && P.form != QB_FORM_EXACT && P.rule.kind != qb::kTieQBF1) {
    rc = solve_fused(h, P, r);
    if (rc >= 0) {
      if (rc) {
        memset(r, 0, sizeof(*r));
        r->status = rc;
      }
      return rc;
    }
    // too many candidate records for the cap: the two-phase path grows it
  }
  double lmin = 0.0;
  rc = begin_finish_pass1(h, P, &lmin);
  if (rc) {
    memset(r, 0, sizeof(*r));
    r->status = rc;
    return rc;
  }
  rc = qb_solve_finish(h, lmin, r);
  if (rc) r->status = rc;
  return rc;
}

}  // extern "C"

namespace {

static_assert(qb::kTcMaxGl + 12 <= qb::kExactMaxFree, "a tensor-core record must fit the exact re-walk");
constexpr int kBatchMaxN = 36;            // larger problems are solved one by one
constexpr int kBatchTcMinN = 24;          // from here on the tensor-core form (>= 512 tiles)
constexpr uint64_t kBatchGtabChunk = 1024;  // G-table steps per CTA

// fn(lo, hi) over [0, count) split into contiguous ranges on up to 16 threads (one thread for
// small counts)
template <class F>
void parallel_ranges(int count, F fn) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::max(1, std::min({16, hw, count / 64}));
  if (nt <= 1) {
    fn(0, count);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    const int lo = (int)((int64_t)count * t / nt), hi = (int)((int64_t)count * (t + 1) / nt);
    th.emplace_back([=]() { fn(lo, hi); });
  }
  for (auto& x : th) x.join();
}

// Host -> device copies of qb_solve_batch's small arrays, staged in one pinned buffer so that
// every copy reads from a stable address (a captured graph replays the same copies)
struct Stage {
  struct Copy {
    void* dst;
    size_t off, bytes;
  };
  std::vector<unsigned char> bytes;  // assembled here, then copied into the pinned buffer once
  std::vector<Copy> copies;
  template <class T>
  void add(void* dst, const std::vector<T>& v) {
    const size_t off = (bytes.size() + 15) & ~(size_t)15;
    bytes.resize(off + v.size() * sizeof(T));
    if (!v.empty()) memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
    if (!v.empty()) copies.push_back(Copy{dst, off, v.size() * sizeof(T)});
  }
};

template <class T>
int ensure_for(DevBuf& d, const std::vector<T>& v) {
  QB_CUDA(d.ensure(std::max<size_t>(v.size() * sizeof(T), 16)));
  return QB_OK;
}

int batch_loop(qb_handle* h, const qb_problem* problems, const std::vector<int32_t>& ids, const qb_options* o,
               qb_result* r) {
  for (int32_t i : ids) {
    int rc = qb_solve(h, &problems[i], o, &r[i]);
    if (rc) return rc;
  }
  return QB_OK;
}

// The batched search of problems[ids] (all 1 <= n <= kBatchMaxN), QB_TIE_QBF with no task
// bits or QB_TIE_NATURAL.
int batch_run(qb_handle* h, const qb_problem* problems, const std::vector<int32_t>& ids, const qb_options* o,
              qb_result* r, bool* overflow) {
  *overflow = false;
  const int m = (int)ids.size();
  if (!m) return QB_OK;
  std::vector<qb::BatchInst> insts(m);
  // every problem's W, then the tensor-core problems' scaled W, packed in pinned memory
  uint64_t w_total = 0;
  for (int j = 0; j < m; ++j) w_total += (uint64_t)problems[ids[j]].n * problems[ids[j]].n;
  QB_CUDA(h->hbat.ensure(2 * w_total * sizeof(double) + 64));
  double* Wall = static_cast<double*>(h->hbat.p);
  double* Wtc = Wall + w_total;
  uint64_t w_used = 0, wtc_used = 0;
  std::vector<qb::BatchItem> gitems, uitems;
  std::vector<uint32_t> gray_ids;  // problems with a selection step (Gray and tensor-core forms)
  std::vector<qb::BatchCand> pre;
  std::vector<std::pair<int, uint64_t>> tcs;  // (problem, offset in Wtc)
  uint64_t gtab_total = 0, rec_total = 0;
  size_t sm_gtab = 0, sm_gray = 0, sm_exact = 0;
  int n_tc_max = 0;
  bool any_gray = false;
  const bool tc_allowed = o->form == QB_FORM_AUTO || o->form == QB_FORM_TC;
  // every problem's W and sum |Q| (host matrices converted on several threads; a device
  // matrix is copied back on the handle's stream first)
  std::vector<uint64_t> w_offs(m);
  std::vector<double> sums(m, 0.0);
  std::vector<char> ints(m, 0);
  std::vector<int> rcs(m, QB_OK);
  {
    uint64_t off = 0;
    for (int j = 0; j < m; ++j) {
      w_offs[j] = off;
      off += (uint64_t)problems[ids[j]].n * problems[ids[j]].n;
    }
    for (int j = 0; j < m; ++j) {
      const qb_problem* p = &problems[ids[j]];
      if (!p->q_on_device) continue;
      std::vector<double> Wv;
      bool ii = false;
      rcs[j] = load_problem(h, p, Wv, &sums[j], &ii);
      ints[j] = ii;
      if (!rcs[j]) memcpy(Wall + w_offs[j], Wv.data(), Wv.size() * sizeof(double));
    }
    auto convert = [&](int j0, int j1) {
      for (int j = j0; j < j1; ++j) {
        const qb_problem* p = &problems[ids[j]];
        if (p->q_on_device) continue;
        bool ii = false;
        rcs[j] = load_host_problem_into(p, Wall + w_offs[j], &sums[j], &ii);
        ints[j] = ii;
      }
    };
    parallel_ranges(m, convert);
  }
  std::vector<std::pair<int, double>> tc_scale;  // (problem, scale) of the tensor-core problems
  for (int j = 0; j < m; ++j) {
    const qb_problem* p = &problems[ids[j]];
    const int n = p->n;
    const double abs_sum = sums[j];
    const bool is_int = ints[j] != 0;
    if (rcs[j]) return rcs[j];
    if (abs_sum >= kTwo53) return QB_ERANGE;
    qb::BatchInst& I = insts[j];
    memset(&I, 0, sizeof(I));
    I.n = n;
    I.is_int = is_int ? 1 : 0;
    I.natural = o->tie_rule == QB_TIE_NATURAL ? 1 : 0;
    I.A = o->prefix_bits < 0 ? n - std::min(n, 20) : o->prefix_bits;
    if (I.A > n) return QB_EINVAL;
    I.B = n - I.A;
    I.w_off = w_offs[j];
    w_used += (uint64_t)n * n;
    int free_bits;
    const qb_handle::Tuned& T = h->tuned[is_int ? 1 : 0][n];
    // the tuned form of (dtype class, n) when qb_autotune chose one, else tensor-core from 24
    const bool use_tc = tc_allowed && qb::tc_supported(n) &&
                        (T.form ? T.form == QB_FORM_TC : n >= kBatchTcMinN);
    if (use_tc) {
      qb::TcPlan tp;
      qb::tc_plan(n, is_int, abs_sum, 0, 1, &tp, T.tc_gl);
      I.kind = qb::kBatchTC;
      I.gl = tp.gl;
      I.exact_digits = tp.exact ? 1 : 0;
      I.scale = tp.scale;
      I.nrec = tp.rec_count;
      I.eps = tp.eps;
      I.rec_off = rec_total;
      rec_total += I.nrec;
      tcs.emplace_back(j, wtc_used);
      tc_scale.emplace_back(j, tp.scale);
      wtc_used += (uint64_t)n * n;
      gray_ids.push_back((uint32_t)j);
      n_tc_max = std::max(n_tc_max, n);
      free_bits = I.gl + 12;
    } else if (n >= 20) {
      any_gray = true;
      I.kind = qb::kBatchGray;
      const GrayShape gs = gray_shape(n, T.gray_b, T.gray_sbits);
      I.b = gs.b;
      I.a = gs.a;
      I.cbbits = gs.cbbits;
      I.sbits = gs.sbits;
      const int ubits = gs.ubits;
      I.gubits = ubits - I.sbits;
      const uint64_t units = 1ull << (I.a - ubits + I.cbbits);
      I.nrec = units << (I.gubits + 3);
      I.eps = (is_int && abs_sum < kTwo24) ? 0.0 : qb::gray_error_bound(abs_sum);
      I.gtab_off = gtab_total;
      gtab_total += (1ull << I.a) * 32;
      I.rec_off = rec_total;
      rec_total += I.nrec;
      for (uint64_t lo = 0; lo < (1ull << I.a); lo += kBatchGtabChunk)
        gitems.push_back(qb::BatchItem{(uint32_t)j, 0u, lo, std::min<uint64_t>(lo + kBatchGtabChunk, 1ull << I.a)});
      for (uint64_t u = 0; u < units; ++u) uitems.push_back(qb::BatchItem{(uint32_t)j, 0u, u, u + 1});
      gray_ids.push_back((uint32_t)j);
      sm_gtab = std::max(sm_gtab, qb::gray_gtab_smem(n, I.a));
      sm_gray = std::max(sm_gray, qb::gray_pass1_smem(n, I.a));
      free_bits = I.sbits + 10;
    } else {
      I.kind = qb::kBatchExact;
      I.fbits = std::min(n, 16);
      for (uint64_t rid = 0; rid < (1ull << (n - I.fbits)); ++rid) pre.push_back(qb::BatchCand{(uint32_t)j, 0u, rid});
      free_bits = I.fbits;
    }
    sm_exact = std::max(sm_exact, qb::exact_smem_bytes(n, free_bits));
  }
  // The 16-bit pair kernel for the tensor-core problems when every one of them takes it: exact
  // integer digits with 16-bit room, else values rounded to a power-of-two unit with an error
  // bound (tc2_u16_quantized).  Its unit replaces the problem's W scale and its bound the
  // problem's eps; each problem gets a table of its 16-bit constants.
  std::vector<qb::Tc2Tab> tc_tabs;
  bool tc_pair = !tcs.empty() && !(o->flags & (QB_FLAG_TC_ONE | QB_FLAG_TC_NO16));
  if (tc_pair) {
    tc_tabs.resize(tcs.size());
    std::vector<double> sg(tcs.size(), 1.0), ep(tcs.size(), 0.0);
    for (size_t k = 0; k < tcs.size() && tc_pair; ++k) {
      const int j = tcs[k].first;
      const int n = insts[j].n;
      const double* W = Wall + w_offs[j];
      float dm = 0.f;
      const bool fits = (insts[j].exact_digits && qb::tc2_u16_eligible(n, W, &dm)) ||
                        qb::tc2_u16_quantized(n, W, sums[j], &sg[k], &dm, &ep[k]);
      if (!fits) {
        tc_pair = false;
        break;
      }
      float gamma[8];
      for (int b = 0; b < 8; ++b) gamma[b] = (float)(W[(size_t)(n - 16) * n + (n - 1 - b)] * sg[k]);
      qb::tc2_u16_tables(gamma, dm, &tc_tabs[k]);
    }
    if (tc_pair) {  // every member fits: only now change the members' plans
      for (size_t k = 0; k < tcs.size(); ++k) {
        qb::BatchInst& I = insts[tcs[k].first];
        if (ep[k] > 0.0) I.exact_digits = 0;  // rounded values (the digits flag is unused by this kernel)
        I.scale = sg[k];
        I.eps = ep[k];
        I.tc_kernel = 4;
        tc_scale[k].second = sg[k];
      }
    } else {
      tc_tabs.clear();
    }
  }
  for (auto& t : tcs)
    if (!insts[t.first].tc_kernel) insts[t.first].tc_kernel = 1;
  // the tensor-core problems' W scaled into their own block (several threads)
  parallel_ranges((int)tcs.size(), [&](int k0, int k1) {
    for (int k = k0; k < k1; ++k) {
      const int j = tcs[k].first;
      const uint64_t nn = (uint64_t)insts[j].n * insts[j].n;
      const double sc = tc_scale[k].second;
      const double* W = Wall + w_offs[j];
      double* dst = Wtc + tcs[k].second;
      for (uint64_t e = 0; e < nn; ++e) dst[e] = W[e] * sc;
    }
  });
  // candidate list: the small problems' records first, then room for the Gray problems'
  const int prefilled = (int)pre.size();
  const int cap = prefilled + std::max(4096, 8 * (int)gray_ids.size());
  DevBuf* B = h->bat;
  int rc;
  // the tensor-core problems' record blocks, dealt out as contiguous runs to one persistent
  // CTA per SM (a run may span problems: one item per problem piece)
  std::vector<qb::TcItem> items;
  std::vector<qb::Tc2Tab> item_tabs;                 // the 16-bit pair kernel: per item
  std::vector<std::pair<uint64_t, uint64_t>> offs;  // (scaled-W offset, record offset) per item
  std::vector<uint32_t> first(1, 0);
  if (!tcs.empty()) {
    uint64_t total = 0;
    for (auto& t : tcs) total += 1ull << (insts[t.first].n - 15 - insts[t.first].gl);
    const uint64_t ctas = std::min<uint64_t>((uint64_t)h->sm_count, total);
    const uint64_t per = (total + ctas - 1) / ctas;
    uint64_t left = per;
    for (size_t k = 0; k < tcs.size(); ++k) {
      const auto& t = tcs[k];
      const qb::BatchInst& I = insts[t.first];
      const uint64_t groups = 1ull << (I.n - 15 - I.gl);
      uint64_t g = 0;
      while (g < groups) {
        const uint64_t take = std::min(left, groups - g);
        qb::TcItem it{};
        offs.emplace_back(t.second, I.rec_off + (g << 3));
        it.i_begin = g << I.gl;
        it.ntiles = take << I.gl;
        it.n = I.n;
        it.gl = I.gl;
        it.exact = I.exact_digits;
        it.inv_scale = (float)(1.0 / I.scale);
        items.push_back(it);
        if (tc_pair) item_tabs.push_back(tc_tabs[k]);
        g += take;
        left -= take;
        if (left == 0) {
          first.push_back((uint32_t)items.size());
          left = per;
        }
      }
    }
    if (first.back() != (uint32_t)items.size()) first.push_back((uint32_t)items.size());
  }
  // every device and pinned host allocation happens here, before any copy or launch is issued
  QB_CUDA(B[0].ensure(std::max<uint64_t>(w_used, 2) * sizeof(double)));
  if ((rc = ensure_for(B[1], insts))) return rc;
  if ((rc = ensure_for(B[2], gitems))) return rc;
  if ((rc = ensure_for(B[3], uitems))) return rc;
  if ((rc = ensure_for(B[4], gray_ids))) return rc;
  QB_CUDA(B[5].ensure((size_t)cap * sizeof(qb::BatchCand)));
  QB_CUDA(B[6].ensure((size_t)cap * sizeof(qb::ExactOut)));
  QB_CUDA(B[7].ensure(std::max<uint64_t>(gtab_total, 4) * sizeof(float)));
  QB_CUDA(B[8].ensure(std::max<uint64_t>(rec_total, 4) * sizeof(float)));
  // minima: emin[m], kmin[m] (uint64), pass1_min[m] (float), cand_count (int)
  const size_t mb = (size_t)m * 8;
  const size_t res_bytes = 2 * mb + (size_t)m * 4 + sizeof(int);
  QB_CUDA(B[9].ensure(res_bytes + 16));
  if (!tcs.empty()) {
    QB_CUDA(B[10].ensure(std::max<uint64_t>(wtc_used, 2) * sizeof(double)));
    if ((rc = ensure_for(B[11], items))) return rc;
    if ((rc = ensure_for(B[12], first))) return rc;
    QB_CUDA(B[13].ensure(16));
    if (tc_pair && (rc = ensure_for(B[14], item_tabs))) return rc;
  }
  QB_CUDA(h->hout.ensure(res_bytes + 16));
  uint64_t* emin = static_cast<uint64_t*>(B[9].p);
  uint64_t* kmin = emin + m;
  float* p1min = reinterpret_cast<float*>(kmin + m);
  int* ccount = reinterpret_cast<int*>(static_cast<char*>(B[9].p) + 2 * mb + (size_t)m * 4);
  for (size_t k = 0; k < items.size(); ++k) {  // device addresses of the items' W and records
    items[k].W = static_cast<const double*>(B[10].p) + offs[k].first;
    items[k].rec = static_cast<float*>(B[8].p) + offs[k].second;
  }
  Stage stg;
  stg.add(B[1].p, insts);
  stg.add(B[2].p, gitems);
  stg.add(B[3].p, uitems);
  stg.add(B[4].p, gray_ids);
  stg.add(B[5].p, pre);
  stg.add(ccount, std::vector<int>(1, prefilled));
  if (!tcs.empty()) {
    stg.add(B[11].p, items);
    stg.add(B[12].p, first);
    if (tc_pair) stg.add(B[14].p, item_tabs);
  }
  QB_CUDA(h->hstage.ensure(std::max<size_t>(stg.bytes.size(), 16)));
  memcpy(h->hstage.p, stg.bytes.data(), stg.bytes.size());
  int64_t h2d_bytes = (int64_t)(w_used * sizeof(double)) + (int64_t)(wtc_used * sizeof(double));
  for (auto& c : stg.copies) h2d_bytes += (int64_t)c.bytes;
  unsigned* tc_err = tcs.empty() ? nullptr : static_cast<unsigned*>(B[13].p);
  const int64_t d2h_bytes = (int64_t)res_bytes + (tc_err ? (int64_t)sizeof(unsigned) : 0);
  const double* dW = static_cast<const double*>(B[0].p);
  const qb::BatchInst* dI = static_cast<const qb::BatchInst*>(B[1].p);
  qb::BatchCand* dC = static_cast<qb::BatchCand*>(B[5].p);
  qb::ExactOut* dO = static_cast<qb::ExactOut*>(B[6].p);
  qb::TcParams P{};
  size_t sm_tc = 0;
  if (!tcs.empty()) {
    P.items = static_cast<const qb::TcItem*>(B[11].p);
    P.item_first = static_cast<const uint32_t*>(B[12].p);
    P.n_max = n_tc_max;
    P.err = tc_err;
    const qb::TcSmemLayout L = qb::tc_layout(n_tc_max);
    if (tc_pair) {  // plus the second tile's row terms of each B stage
      sm_tc = std::max<size_t>(L.total + qb::kTcBStages * 128 * 4, 120 * 1024) + 1024;
      QB_CUDA(cudaFuncSetAttribute(qb::tc_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_tc));
    } else {
      sm_tc = std::max<size_t>(L.total, 120 * 1024) + 1024;
      QB_CUDA(cudaFuncSetAttribute(qb::tc_pass1_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_tc));
    }
  }
  if (any_gray) {
    QB_CUDA(cudaFuncSetAttribute(qb::batch_gtab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_gtab));
    QB_CUDA(cudaFuncSetAttribute(qb::batch_gray_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_gray));
  }
  QB_CUDA(cudaFuncSetAttribute(qb::batch_exact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_exact));
  const unsigned key_blocks = (unsigned)std::min<int>((cap + 255) / 256, h->sm_count * 4);

  // the whole device side of the batch: uploads, the six launches, the result copy
  auto issue = [&](cudaStream_t st, bool timed) -> int {
    QB_CUDA(cudaMemcpyAsync(B[0].p, Wall, w_used * sizeof(double), cudaMemcpyHostToDevice, st));
    for (auto& c : stg.copies)
      QB_CUDA(cudaMemcpyAsync(c.dst, static_cast<unsigned char*>(h->hstage.p) + c.off, c.bytes,
                              cudaMemcpyHostToDevice, st));
    QB_CUDA(cudaMemsetAsync(B[9].p, 0xff, 2 * mb, st));
    if (timed) {
      QB_CUDA(cudaEventRecord(h->ev[0], st));
      QB_CUDA(cudaEventRecord(h->ev[4], st));
    }
    if (any_gray) {
      qb::batch_gtab_kernel<<<(unsigned)gitems.size(), 256, sm_gtab, st>>>(
          dI, static_cast<const qb::BatchItem*>(B[2].p), dW, static_cast<float*>(B[7].p));
      qb::batch_gray_kernel<<<(unsigned)uitems.size(), qb::kGrayThreads, sm_gray, st>>>(
          dI, static_cast<const qb::BatchItem*>(B[3].p), dW, static_cast<const float*>(B[7].p),
          static_cast<float*>(B[8].p));
      h->kernels += 2;
    }
    if (!tcs.empty()) {
      QB_CUDA(cudaMemcpyAsync(B[10].p, Wtc, wtc_used * sizeof(double), cudaMemcpyHostToDevice, st));
      QB_CUDA(cudaMemsetAsync(tc_err, 0, 16, st));
      if (tc_pair) {
        qb::Tc2Params Q2{};
        Q2.P = P;
        Q2.tabs = static_cast<const qb::Tc2Tab*>(B[14].p);
        qb::tc_pair_kernel<true><<<(unsigned)(first.size() - 1), qb::kTcThreads, sm_tc, st>>>(Q2);
      } else
        qb::tc_pass1_kernel<true><<<(unsigned)(first.size() - 1), qb::kTcThreads, sm_tc, st>>>(P);
      ++h->kernels;
    }
    if (timed) {
      QB_CUDA(cudaEventRecord(h->ev[5], st));
      QB_CUDA(cudaEventRecord(h->ev[1], st));
      QB_CUDA(cudaEventRecord(h->ev[2], st));
    }
    if (!gray_ids.empty()) {
      qb::batch_select_kernel<<<(unsigned)gray_ids.size(), 256, 0, st>>>(
          dI, static_cast<const uint32_t*>(B[4].p), static_cast<const float*>(B[8].p), dC, ccount, cap, p1min,
          emin, kmin);
      ++h->kernels;
    }
    qb::batch_exact_kernel<<<(unsigned)cap, qb::kExactThreads, sm_exact, st>>>(dI, dW, dC, ccount, cap, dO, emin);
    qb::batch_key_kernel<<<key_blocks, 256, 0, st>>>(dC, ccount, cap, dO, emin, kmin);
    h->kernels += 2;
    QB_CUDA(cudaGetLastError());
    if (timed) QB_CUDA(cudaEventRecord(h->ev[3], st));
    QB_CUDA(cudaMemcpyAsync(h->hout.p, B[9].p, res_bytes, cudaMemcpyDeviceToHost, st));
    if (tc_err)
      QB_CUDA(cudaMemcpyAsync(static_cast<char*>(h->hout.p) + res_bytes, tc_err, sizeof(unsigned),
                              cudaMemcpyDeviceToHost, st));
    return QB_OK;
  };

  const bool graph = (o->flags & QB_FLAG_GRAPH) != 0;
  if (graph) {
    // one graph launch per batch; the graph is captured again whenever the batch's shape, the
    // options or any buffer address differ from the captured one
    std::vector<uint64_t> key = {(uint64_t)m, (uint64_t)w_used, (uint64_t)wtc_used, (uint64_t)cap,
                                 (uint64_t)gitems.size(), (uint64_t)uitems.size(), (uint64_t)gray_ids.size(),
                                 (uint64_t)first.size(), (uint64_t)sm_gtab, (uint64_t)sm_gray, (uint64_t)sm_exact,
                                 (uint64_t)sm_tc, (uint64_t)any_gray, (uint64_t)tc_pair, (uint64_t)(uintptr_t)Wall,
                                 (uint64_t)(uintptr_t)h->hstage.p, (uint64_t)(uintptr_t)h->hout.p,
                                 (uint64_t)(uintptr_t)h->own};
    for (int k = 0; k < 14; ++k) key.push_back((uint64_t)(uintptr_t)B[k].p);
    for (auto& c : stg.copies) {
      key.push_back((uint64_t)(uintptr_t)c.dst);
      key.push_back((uint64_t)c.off);
      key.push_back((uint64_t)c.bytes);
    }
    if (!h->batch_graph || key != h->batch_graph_key) {
      if (h->batch_graph) {
        cudaGraphExecDestroy(h->batch_graph);
        h->batch_graph = nullptr;
        h->batch_graph_key.clear();
      }
      cudaGraph_t g = nullptr;
      QB_CUDA(cudaStreamBeginCapture(h->own, cudaStreamCaptureModeThreadLocal));
      const int k0 = h->kernels;
      const int irc = issue(h->own, false);
      const cudaError_t ce = cudaStreamEndCapture(h->own, &g);
      h->batch_graph_kernels = h->kernels - k0;
      h->kernels = k0;
      if (irc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return irc ? irc : cuda_fail(ce);
      }
      const cudaError_t ie = cudaGraphInstantiate(&h->batch_graph, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        h->batch_graph = nullptr;
        return cuda_fail(ie);
      }
      h->batch_graph_key = key;
    }
    QB_CUDA(cudaEventRecord(h->ev[0], h->st));
    QB_CUDA(cudaGraphLaunch(h->batch_graph, h->st));
    QB_CUDA(cudaEventRecord(h->ev[3], h->st));
    h->kernels += h->batch_graph_kernels;
  } else {
    if ((rc = issue(h->st, true))) return rc;
  }
  h->h2d += h2d_bytes;
  h->d2h += d2h_bytes;
  QB_CUDA(cudaStreamSynchronize(h->st));
  const uint64_t* he = static_cast<const uint64_t*>(h->hout.p);
  const uint64_t* hk = he + m;
  const float* hp = reinterpret_cast<const float*>(hk + m);
  const int got = *reinterpret_cast<const int*>(reinterpret_cast<const char*>(h->hout.p) + 2 * mb + (size_t)m * 4);
  if (tc_err) {
    unsigned e = 0;
    memcpy(&e, static_cast<const char*>(h->hout.p) + res_bytes, sizeof(unsigned));
    if (e & qb::kErrTimeout) return QB_ETIMEOUT;
  }
  if (got > cap) {
    *overflow = true;
    return QB_OK;
  }
  float p1 = 0.f, p2 = 0.f, km = 0.f;
  if (graph) {  // one launch: its whole device time is reported as pass 1 and as the kernel time
    QB_CUDA(cudaEventElapsedTime(&p1, h->ev[0], h->ev[3]));
    km = p1;
  } else {
    QB_CUDA(cudaEventElapsedTime(&p1, h->ev[0], h->ev[1]));
    QB_CUDA(cudaEventElapsedTime(&p2, h->ev[2], h->ev[3]));
    QB_CUDA(cudaEventElapsedTime(&km, h->ev[4], h->ev[5]));
  }
  for (int j = 0; j < m; ++j) {
    const qb::BatchInst& I = insts[j];
    qb_result& R = r[ids[j]];
    memset(&R, 0, sizeof(R));
    if (he[j] == ~0ull || hk[j] == ~0ull) {
      R.status = QB_ECUDA;
      return QB_ECUDA;
    }
    const uint64_t key = hk[j];
    const uint64_t x = I.natural ? key : ((qb::gray64(key >> I.B) << I.B) | (key & qb::mask64(I.B)));
    R.best_x = x;
    R.best_e = qb::unord_f64(he[j]);
    R.best_e_int = I.is_int ? (int64_t)llround(R.best_e) : 0;
    R.order_key = key;
    R.pass1_min = I.kind != qb::kBatchExact ? (double)hp[j] : R.best_e;
    R.err_bound = I.eps;
    R.states = (int64_t)1 << I.n;
    R.form_used = I.kind == qb::kBatchGray ? QB_FORM_GRAY : (I.kind == qb::kBatchTC ? QB_FORM_TC : QB_FORM_EXACT);
    const qb_handle::Tuned& T = h->tuned[I.is_int ? 1 : 0][I.n];
    if (I.kind == qb::kBatchGray) {
      R.rec_log2 = I.sbits;
      R.suffix_bits = I.b;
      R.unit_log2 = I.gubits + I.sbits;
      R.tuned = (T.gray_b || T.gray_sbits || T.form == QB_FORM_GRAY) ? 1 : 0;
    } else if (I.kind == qb::kBatchTC) {
      R.rec_log2 = I.gl;
      R.suffix_bits = 15;
      R.tc_kernel = I.tc_kernel;  // 4: the 16-bit pair kernel, 1: one state with fp32 minima
      R.tuned = (T.tc_gl || T.form == QB_FORM_TC) ? 1 : 0;
    } else {
      R.rec_log2 = I.fbits;
    }
    R.is_integer = I.is_int;
    R.found = 1;
    R.status = QB_OK;
    R.pass1_ms = p1;
    R.pass2_ms = p2;
    R.kernels = h->kernels;
    R.kernel_ms = km;
    R.h2d_bytes = h->h2d;
    R.d2h_bytes = h->d2h;
  }
  return QB_OK;
}

}  // namespace

extern "C" {

int qb_solve_batch(qb_handle* h, const qb_problem* problems, int32_t count, const qb_options* o, qb_result* r) {
  if (!h || !problems || !o || !r || count < 0) return QB_EINVAL;
  std::vector<int32_t> batched, single;
  const bool rule_ok = (o->tie_rule == QB_TIE_QBF && o->fixed_bits == 0) || o->tie_rule == QB_TIE_NATURAL;
  const bool form_ok = o->form == QB_FORM_AUTO || o->form == QB_FORM_GRAY;
  for (int32_t i = 0; i < count; ++i) {
    const qb_problem* p = &problems[i];
    if (p->n < 1 || p->n > qb::kMaxN || !p->q || p->ldq < p->n || dtype_size(p->dtype) == 0) return QB_EINVAL;
    if (rule_ok && form_ok && o->shard_count <= 1 && p->n <= kBatchMaxN)
      batched.push_back(i);
    else
      single.push_back(i);
  }
  if (!batched.empty()) {
    QB_CUDA(cudaSetDevice(h->device));
    h->st = o->stream ? static_cast<cudaStream_t>(o->stream) : h->own;
    h->pending = false;
    h->kernels = 0;
    h->h2d = h->d2h = 0;
    bool overflow = false;
    int rc = batch_run(h, problems, batched, o, r, &overflow);
    if (rc) return rc;
    if (overflow) single.insert(single.end(), batched.begin(), batched.end());  // too many candidates
  }
  std::sort(single.begin(), single.end());
  return batch_loop(h, problems, single, o, r);
}

int qb_prefix_minima(qb_handle* h, const qb_problem* p, int32_t prefix_bits, double* out) {
  if (!h || !p || !out) return QB_EINVAL;
  if (p->n < 1 || p->n > qb::kMaxN || !p->q || p->ldq < p->n || dtype_size(p->dtype) == 0) return QB_EINVAL;
  const int n = p->n;
  const int A = prefix_bits < 0 ? n - std::min(n, 20) : prefix_bits;
  const int B = n - A;
  if (A < 0 || A > kPrefixMinimaMaxA || B > qb::kExactMaxFree) return QB_EINVAL;
  QB_CUDA(cudaSetDevice(h->device));
  h->st = h->own;
  h->pending = false;
  h->kernels = 0;
  h->h2d = h->d2h = 0;
  std::vector<double> W;
  double abs_sum = 0.0;
  bool is_int = false;
  int rc = load_problem(h, p, W, &abs_sum, &is_int);
  if (rc) return rc;
  if (abs_sum >= kTwo53) return QB_ERANGE;
  rc = upload_W(h, W);
  if (rc) return rc;
  // one exact record per prefix value: the 2^B states whose first A variables spell it
  qb::RecGeom geom{};
  geom.kind = qb::kGeomBlock;
  geom.n = n;
  geom.fbits = B;
  qb::TieRule rule{qb::kTieNatural, n, 0, 0, 0};
  const qb::ProblemDev pd{n, static_cast<const double*>(h->W.p)};
  const uint64_t count = 1ull << A;
  QB_CUDA(h->exout.ensure(count * sizeof(qb::ExactOut)));
  const size_t sm = qb::exact_smem_bytes(n, B);
  QB_CUDA(cudaFuncSetAttribute(qb::exact_records_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const uint64_t maxg = 1u << 30;
  for (uint64_t off = 0; off < count; off += maxg) {
    const uint64_t g = std::min<uint64_t>(maxg, count - off);
    qb::exact_records_kernel<<<(unsigned)g, qb::kExactThreads, sm, h->st>>>(
        pd, rule, geom, nullptr, nullptr, (int64_t)count, (int64_t)off, static_cast<qb::ExactOut*>(h->exout.p) + off, 0);
    ++h->kernels;
  }
  QB_CUDA(cudaGetLastError());
  QB_CUDA(h->hout.ensure(count * sizeof(qb::ExactOut)));
  QB_CUDA(cudaMemcpyAsync(h->hout.p, h->exout.p, count * sizeof(qb::ExactOut), cudaMemcpyDeviceToHost, h->st));
  QB_CUDA(cudaStreamSynchronize(h->st));
  const qb::ExactOut* eo = static_cast<const qb::ExactOut*>(h->hout.p);
  for (uint64_t i = 0; i < count; ++i) out[i] = eo[qb::gray64(i)].e;  // QBF's prefix visiting order
  return QB_OK;
}

int qb_autotune(qb_handle* h, int32_t n, int32_t dtype, int32_t* form_out) {
  if (!h || !form_out || n < 1 || n > qb::kMaxN || dtype_size(dtype) == 0) return QB_EINVAL;
  const bool is_int = dtype >= QB_I8;
  qb_handle::Tuned& T = h->tuned[is_int ? 1 : 0][n];
  if (n < 20) {  // the exact form is the only one below 20 variables
    T = qb_handle::Tuned{};
    T.form = QB_FORM_EXACT;
    *form_out = QB_FORM_EXACT;
    return QB_OK;
  }
  // a seeded synthetic problem of the dtype's class: integer entries in [-100, 100] for
  // integer dtypes (exact arithmetic), uniform [-1, 1) for float dtypes
  std::vector<double> Q((size_t)n * n);
  uint64_t st = 0x9E3779B97F4A7C15ull ^ (uint64_t)n;
  for (auto& v : Q) {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    v = is_int ? (double)((int64_t)(st % 201) - 100) : (double)(st >> 11) * 0x1.0p-52 - 1.0;
  }
  qb_problem p{};
  p.n = n;
  p.dtype = is_int ? QB_I64 : QB_F64;
  std::vector<int64_t> Qi;
  if (is_int) {
    Qi.assign(Q.begin(), Q.end());
    p.q = Qi.data();
  } else {
    p.q = Q.data();
  }
  p.ldq = n;
  // candidates: (form, tc_gl) and (form, gray_b, gray_sbits) around the defaults
  std::vector<qb_handle::Tuned> cands;
  {
    const GrayShape g0 = gray_shape(n);
    for (int db : {0, -1, 1, -2}) {
      const int b = g0.b + db;
      const GrayShape g = gray_shape(n, b);
      if (g.b != b) continue;  // outside the valid range
      for (int ds : {0, 1, 2}) {
        const int sb = std::min(g.a, std::max(5, n - 34)) + ds;
        if (sb > g.a) continue;
        qb_handle::Tuned t;
        t.form = QB_FORM_GRAY;
        t.gray_b = b;
        t.gray_sbits = sb;
        cands.push_back(t);
      }
    }
    if (qb::tc_supported(n)) {
      const int gl0 = qb::tc_default_gl(n);
      for (int pair = 0; pair < 2; ++pair)
        for (int d = 0; d <= 3; ++d) {
          if (gl0 + d > std::min(n - 15, qb::kTcMaxGl)) break;
          qb_handle::Tuned t;
          t.form = QB_FORM_TC;
          t.tc_gl = gl0 + d;
          t.tc_pair = pair;
          cands.push_back(t);
        }
    }
  }
  // time one shard of at most 2^36 states per candidate: pass 1 plus candidate re-evaluation
  const int shard_bits = std::max(0, n - 36);
  float best_ms = 0.f;
  qb_handle::Tuned best{};
  for (const qb_handle::Tuned& c : cands) {
    T = c;  // planning reads the handle's entry
    qb_options o{};
    o.form = c.form;
    o.tie_rule = QB_TIE_QBF;
    o.prefix_bits = -1;
    o.shard_index = 0;
    o.shard_count = 1 << shard_bits;
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {  // warm-up, then the timed call
      double lmin = 0.0;
      int rc = qb_solve_begin(h, &p, &o, &lmin);
      if (rc) {
        T = qb_handle::Tuned{};
        return rc;
      }
      qb_result r{};
      rc = qb_solve_finish(h, lmin, &r);
      if (rc) {
        T = qb_handle::Tuned{};
        return rc;
      }
      ms = r.pass1_ms + r.pass2_ms;
    }
    if (best_ms == 0.f || ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  T = best;
  *form_out = best.form;
  return QB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// qb_solve_noalloc: the whole Gray-form search on the caller's stream with no allocation.
//
// Some callers cannot allocate device memory during a solve: an application that hands
// out all of its device memory from its own pool up front, a real-time loop that must not
// block on the allocator (cudaMalloc and cudaFree synchronise the device), or code running
// where a new allocation would break a memory budget fixed at start-up.  For them this
// entry point keeps every intermediate buffer in one file-scope device array of fixed size
// (kNoAllocBytes, 16.9 MB) that each GPU holds from the moment the library's device code is
// loaded on it until the process exits.  The caller passes Q and the output on the device; the entry
// point calls no cudaMalloc, cudaFree, cudaMallocHost or allocating library routine and
// does not wait for the GPU.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that first call
// before any stream capture, and make it a complete, valid solve (20 <= n <= 36, finite Q)
// so that it also launches every kernel the entry point uses: with CUDA's lazy module
// loading the first launch of a kernel can load code and take device memory.  All calls share the one array and every call overwrites it:
// calls whose work overlaps on the GPU (other streams, other threads) race and must be
// serialised by the caller.
// ---------------------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxN = 36;
constexpr int kNoAllocMinN = 20;
constexpr int kNoAllocCands = 4096;
constexpr size_t kNoAllocW = 16 * 1024;                             // n*n doubles, n <= 36
constexpr size_t kNoAllocGtab = (size_t)1 << 16 << 5 << 2;          // 2^16 prefix steps x 32 floats
constexpr size_t kNoAllocRec = (size_t)1 << 21 << 2;                // 2^(n-10-sbits) <= 2^21 records x float
constexpr size_t kNoAllocCand = (size_t)kNoAllocCands * sizeof(uint64_t);
constexpr size_t kNoAllocOut = (size_t)kNoAllocCands * sizeof(qb::ExactOut);
constexpr size_t kNoAllocMisc = 256;
constexpr size_t kNoAllocBytes = kNoAllocW + kNoAllocGtab + kNoAllocRec + kNoAllocCand + kNoAllocOut + kNoAllocMisc;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct NoAllocMisc {  // lives at the end of g_noalloc_scratch
  double abs_sum;
  double threshold;
  uint32_t min_key;
  int cand_count;
  int bad_input;  // Q held a NaN / infinity, or a fractional value with is_integer set
};

static_assert(sizeof(NoAllocMisc) <= kNoAllocMisc, "misc block");
static_assert(kNoAllocBytes == 16924928, "scratch size stated in include/qubo_b200.h");

std::mutex g_noalloc_lock;
void* g_noalloc_addr[128] = {nullptr};

// W from Q, sum |Q_ij|, and the input checks that qb_solve makes on the host: every entry
// finite and, when the caller says Q is integer, integral (a fractional entry would make the
// exact path's zero error band drop the true minimum)
__global__ void noalloc_prep_kernel(const double* __restrict__ Q, int n, int is_int, double* __restrict__ W,
                                    NoAllocMisc* __restrict__ misc) {
  __shared__ double part[256];
  double s = 0.0;
  int bad = 0;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    const double q = Q[e];
    if (!isfinite(q) || (is_int && q != trunc(q))) bad = 1;
    s += fabs(q);
    W[e] = (i == j) ? q : q + Q[j * n + i];
  }
  bad = __syncthreads_or(bad);
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = blockDim.x / 2; off; off >>= 1) {
    if (threadIdx.x < off) part[threadIdx.x] += part[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    misc->abs_sum = part[0];
    misc->min_key = 0xffffffffu;
    misc->cand_count = 0;
    misc->bad_input = bad;
  }
}

__global__ void noalloc_threshold_kernel(NoAllocMisc* __restrict__ misc, int is_int) {
  const double m = (double)qb::key2f(misc->min_key);
  const double S = misc->abs_sum;
  // the Gray form's per-state bound on |fp32 pass-1 value - exact energy| (300 ulp of S)
  const bool exact_int = is_int && S < 16777216.0;
  const double eps = exact_int ? 0.0 : 300.0 * S * 5.9604644775390625e-08;
  double thr = m + 2.0 * eps;
  if (eps > 0.0) thr += fabs(thr) * 1e-12;
  // nothing to re-walk when the answer is already known: rejected input, or exact integer
  // arithmetic with no negative energy (X = 0, E = 0 is minimal and has the smallest key)
  if (misc->bad_input || (exact_int && m >= 0.0)) thr = -__longlong_as_double(0x7ff0000000000000ll);
  misc->threshold = thr;
  misc->cand_count = 0;
}

__global__ void noalloc_select_kernel(const float* __restrict__ rec, int64_t count, const NoAllocMisc* misc,
                                      uint64_t* __restrict__ cand, int* __restrict__ cand_count, int cap) {
  const double thr = misc->threshold;
  if (thr == -__longlong_as_double(0x7ff0000000000000ll)) return;  // nothing to select
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    if ((double)rec[i] <= thr) {
      const int s = atomicAdd(cand_count, 1);
      if (s < cap) cand[s] = (uint64_t)i;
    }
  }
}

__global__ void noalloc_final_kernel(const qb::ExactOut* __restrict__ eo, const NoAllocMisc* __restrict__ misc,
                                     int cap, int is_int, qb_noalloc_result* __restrict__ out) {
  __shared__ qb::ExactOut best[256];
  const int cnt = misc->cand_count;
  const int m = cnt < cap ? cnt : cap;
  qb::ExactOut b{__longlong_as_double(0x7ff0000000000000ll), ~0ull, 0ull};
  for (int i = threadIdx.x; i < m; i += blockDim.x)
    if (eo[i].e < b.e || (eo[i].e == b.e && eo[i].key < b.key)) b = eo[i];
  best[threadIdx.x] = b;
  __syncthreads();
  for (int off = blockDim.x / 2; off; off >>= 1) {
    if (threadIdx.x < off) {
      const qb::ExactOut& o = best[threadIdx.x + off];
      if (o.e < best[threadIdx.x].e || (o.e == best[threadIdx.x].e && o.key < best[threadIdx.x].key))
        best[threadIdx.x] = o;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double pmin = (double)qb::key2f(misc->min_key);
    const bool exact_int = is_int && misc->abs_sum < 16777216.0;
    if (misc->bad_input) {
      out->best_e = 0.0;
      out->best_x = 0ull;
      out->order_key = 0ull;
      out->status = QB_EINVAL;
    } else if (is_int && misc->abs_sum >= 9007199254740992.0) {  // sum |Q_ij| >= 2^53: FP64 not exact
      out->best_e = 0.0;
      out->best_x = 0ull;
      out->order_key = 0ull;
      out->status = QB_ERANGE;
    } else if (exact_int && pmin >= 0.0) {  // E(0) = 0 is minimal; X = 0 has the smallest key
      out->best_e = 0.0;
      out->best_x = 0ull;
      out->order_key = 0ull;
      out->status = QB_OK;
    } else {
      out->best_e = best[0].e;
      out->best_x = best[0].x;
      out->order_key = best[0].key;
      out->status = cnt > cap ? QB_EOVERFLOW : (m > 0 ? QB_OK : QB_ECUDA);
    }
    out->candidates = cnt;
  }
}

// Queues the search on `st`; `device` is current.
int noalloc_run(int device, const double* q_dev, int n, int is_integer, int prefix_bits, qb_noalloc_result* out_dev,
                cudaStream_t st) {
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> g(g_noalloc_lock);
    if (!g_noalloc_addr[device]) {  // first call on this device: resolve the array's address
      void* a = nullptr;
      QB_CUDA(cudaGetSymbolAddress(&a, g_noalloc_scratch));
      g_noalloc_addr[device] = a;
    }
    base = static_cast<unsigned char*>(g_noalloc_addr[device]);
  }
  const int A = prefix_bits < 0 ? n - std::min(n, 20) : prefix_bits;
  if (A > n) return QB_EINVAL;
  double* W = reinterpret_cast<double*>(base);
  float* gtab = reinterpret_cast<float*>(base + kNoAllocW);
  float* rec = reinterpret_cast<float*>(base + kNoAllocW + kNoAllocGtab);
  uint64_t* cand = reinterpret_cast<uint64_t*>(base + kNoAllocW + kNoAllocGtab + kNoAllocRec);
  qb::ExactOut* eo = reinterpret_cast<qb::ExactOut*>(base + kNoAllocW + kNoAllocGtab + kNoAllocRec + kNoAllocCand);
  NoAllocMisc* misc =
      reinterpret_cast<NoAllocMisc*>(base + kNoAllocW + kNoAllocGtab + kNoAllocRec + kNoAllocCand + kNoAllocOut);
  // the Gray-form plan of qb_solve for this n (one shard)
  const int b = std::max(13, n - 16), a = n - b, cbbits = b - 13;
  const int sbits = std::min(a, std::max(5, n - 34));
  const int ubits = std::min(a, std::max(7, std::max(sbits, std::min(a, a + cbbits - 11))));
  qb::RecGeom geom{};
  geom.kind = qb::kGeomGray;
  geom.n = n;
  geom.a = a;
  geom.b = b;
  geom.sbits = sbits;
  geom.cbbits = cbbits;
  geom.gubits = ubits - sbits;
  const uint64_t units = 1ull << (a - ubits + cbbits);
  const uint64_t nrec = units << (geom.gubits + 3);
  const qb::TieRule rule{qb::kTieQBF, n, 0, A, n - A};
  int sms = 0;
  QB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const qb::ProblemDev pd{n, W};
  noalloc_prep_kernel<<<1, 256, 0, st>>>(q_dev, n, is_integer ? 1 : 0, W, misc);
  const size_t sm0 = qb::gray_gtab_smem(n, a);
  QB_CUDA(cudaFuncSetAttribute(qb::gray_gtab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm0));
  qb::gray_gtab_kernel<<<(unsigned)std::min<uint64_t>((1ull << a) / 8 + 1, (uint64_t)sms * 4), 256, sm0, st>>>(pd, a, b, gtab);
  qb::GrayParams gp{};
  gp.P = pd;
  gp.a = a;
  gp.b = b;
  gp.cbbits = cbbits;
  gp.sbits = sbits;
  gp.gubits = geom.gubits;
  gp.unit_begin = 0;
  gp.gtab = gtab;
  gp.rec = rec;
  const size_t sm1 = qb::gray_pass1_smem(n, a);
  QB_CUDA(cudaFuncSetAttribute(qb::gray_pass1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
  qb::gray_pass1_kernel<<<(unsigned)units, qb::kGrayThreads, sm1, st>>>(gp);
  const unsigned rb = (unsigned)std::min<uint64_t>((nrec + 255) / 256, (uint64_t)sms * 8);
  qb::rec_min_kernel<<<rb, 256, 0, st>>>(rec, (int64_t)nrec, &misc->min_key);
  noalloc_threshold_kernel<<<1, 1, 0, st>>>(misc, is_integer ? 1 : 0);
  noalloc_select_kernel<<<rb, 256, 0, st>>>(rec, (int64_t)nrec, misc, cand, &misc->cand_count, kNoAllocCands);
  int maxf = 0;
  {
    uint64_t bb, ff;
    qb::record_states(geom, 0, &bb, &ff);
    maxf = __builtin_popcountll(ff & qb::mask64(n));
  }
  const size_t sm2 = qb::exact_smem_bytes(n, maxf);
  QB_CUDA(cudaFuncSetAttribute(qb::exact_records_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
  qb::exact_records_kernel<<<kNoAllocCands, qb::kExactThreads, sm2, st>>>(pd, rule, geom, cand, &misc->cand_count, 0, 0,
                                                                         eo, 0);
  noalloc_final_kernel<<<1, 256, 0, st>>>(eo, misc, kNoAllocCands, is_integer ? 1 : 0, out_dev);
  QB_CUDA(cudaGetLastError());
  return QB_OK;
}

}  // namespace

extern "C" int qb_solve_noalloc(int device, const double* q_dev, int32_t n, int32_t is_integer, int32_t prefix_bits,
                                qb_noalloc_result* out_dev, void* stream) {
  if (!q_dev || !out_dev) return QB_EINVAL;
  if (n < kNoAllocMinN || n > kNoAllocMaxN) return QB_ETOOBIG;
  int ndev = 0;
  QB_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev || device >= 128) return QB_ENODEV;
  int prev = 0;
  QB_CUDA(cudaGetDevice(&prev));
  if (prev != device) QB_CUDA(cudaSetDevice(device));
  const int rc = noalloc_run(device, q_dev, n, is_integer, prefix_bits, out_dev, static_cast<cudaStream_t>(stream));
  if (prev != device) cudaSetDevice(prev);
  return rc;
}
