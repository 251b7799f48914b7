/*
 * oracle/qbf_port.c -- TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline).
 *
 * A plain-C restatement of the reference's exhaustive QUBO search, used to
 * check the CUDA path and to time the reference algorithm on host cores.
 * Nothing in the product path links or calls this file.
 *
 * Follows (paths inside cloud-ru-tech/evo-quantum-qubolib):
 *   src/qubo_lib/solvers/qbf.py:429-446  define_chunk_size (default B = min(N, 20))
 *   src/qubo_lib/solvers/qbf.py:246-289  build_cache: diag_BB (suffix energies) and
 *                                        ABBA = (Q_0B + Q_1A^T) X_B^T (cross rows)
 *   src/qubo_lib/solvers/qbf.py:188-230  iterate_prefix_interval: Gray-ordered prefix
 *                                        loop, chunk +/-= ABBA[row], argmin (first index)
 *   src/qubo_lib/solvers/qbf.py:291-325  gray_code_iterator: step i has gray value
 *                                        i ^ (i >> 1); row index = A - 1 - flipped bit
 *   src/qubo_lib/solvers/qbf.py:232-244  do_correction every correction_period steps
 *   src/qubo_lib/solvers/qbf.py:395-412  update_global_minima: strict '<' against a
 *                                        running best that starts at (E=0, pref=0, x=0)
 *   src/qubo_lib/problems/reduced_problem.py:31-46  bit fixing: prefix_E and the reduced Q
 *   src/qubo_lib/solvers/parallel.py:145-157, 273-300  Parallel: 2^k MSB-first task
 *                                        prefixes, min over best_E + prefix_E
 *
 * Arithmetic: integer Q is accumulated exactly (int32 when sum|Q| < 2^31, else int64);
 * float Q in IEEE double (the FP64 semantics the GPU results are compared with).
 * The reference accumulates in Q's own dtype; where that dtype could wrap or round,
 * this port gives the exact / FP64 answer instead.
 *
 * State encoding: X is the MSB-first integer of the whole state, variable i <-> bit
 * (n-1-i).  prefix = X >> B (A bits), suffix = X & (2^B - 1).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct oq_result {
  double best_e;        /* energy of the returned state (exact for integer Q) */
  int64_t best_e_int;   /* same, integer Q only */
  uint64_t best_x;      /* MSB-first state integer */
  uint64_t glob_pref;   /* Gray *value* of the winning prefix (QBF's glob_pref) */
  uint64_t glob_x;      /* winning suffix integer (QBF's glob_X) */
  int64_t epochs;       /* 2^A prefix steps */
  int32_t A, B;
  int32_t status;       /* 0 ok, <0 error */
} oq_result;

/* Energy of one state, exact for integer-valued Q (< 2^53), FP64 otherwise. */
double oq_energy(int n, const double* Q, uint64_t X) {
  double e = 0.0;
  for (int i = 0; i < n; ++i) {
    if (!((X >> (n - 1 - i)) & 1)) continue;
    for (int j = 0; j < n; ++j)
      if ((X >> (n - 1 - j)) & 1) e += Q[(size_t)i * n + j];
  }
  return e;
}

/* default (A, B) of qbf.py:443-446 */
void oq_default_split(int n, int* A, int* B) {
  int b = n < 20 ? n : 20;
  *B = b;
  *A = n - b;
}

/* Suffix energies E_suf(s) = s^T Q_1B s for all 2^B suffixes (qbf.py:249-251 computes the
 * same vector recursively).  Direct Gray walk with a local-field vector. */
#define OQ_DEFINE_TYPED(T, SUF)                                                       \
static void suffix_energies_##SUF(int n, int A, const double* Q, T* out) {            \
  int B = n - A;                                                                      \
  T* h = (T*)calloc((size_t)B + 1, sizeof(T)); /* h[j] = sum_{m!=j} W_jm s_m */       \
  T e = 0;                                                                            \
  uint64_t g = 0;                                                                     \
  out[0] = 0;                                                                         \
  for (uint64_t i = 1; i < ((uint64_t)1 << B); ++i) {                                 \
    int bit = __builtin_ctzll(i);           /* integer bit of the suffix */           \
    int v = A + (B - 1 - bit);              /* variable index */                      \
    int on = !((g >> bit) & 1);                                                       \
    T d = (T)Q[(size_t)v * n + v] + h[B - 1 - bit];                                   \
    e = on ? e + d : e - d;                                                           \
    for (int j = 0; j < B; ++j) {                                                     \
      int u = A + j;                                                                  \
      if (u == v) continue;                                                           \
      T w = (T)(Q[(size_t)v * n + u] + Q[(size_t)u * n + v]);                         \
      h[j] = on ? h[j] + w : h[j] - w;                                                \
    }                                                                                 \
    g ^= (uint64_t)1 << bit;                                                          \
    out[g] = e;                                                                       \
  }                                                                                   \
  free(h);                                                                            \
}                                                                                     \
                                                                                      \
/* qbf.py:188-230 with the build_cache of qbf.py:246-289.  Q is n*n row-major. */     \
static int qbf_solve_##SUF(int n, const double* Q, int A, int corr, oq_result* r) {   \
  int B = n - A;                                                                      \
  size_t M = (size_t)1 << B;                                                          \
  T* diag_bb = (T*)malloc(M * sizeof(T));                                             \
  T* abba = (T*)malloc((size_t)(A ? A : 1) * M * sizeof(T));                          \
  T* chunk = (T*)malloc(M * sizeof(T));                                               \
  if (!diag_bb || !abba || !chunk) { free(diag_bb); free(abba); free(chunk); return -2; } \
  suffix_energies_##SUF(n, A, Q, diag_bb);                                            \
  /* ABBA[k][s] = sum_j (Q[k][A+j] + Q[A+j][k]) * s_j, built incrementally over s */  \
  for (int k = 0; k < A; ++k) {                                                       \
    T* row = abba + (size_t)k * M;                                                    \
    row[0] = 0;                                                                       \
    for (size_t s = 1; s < M; ++s) {                                                  \
      int bit = __builtin_ctzll(s);                                                   \
      int j = B - 1 - bit;                                                            \
      T w = (T)(Q[(size_t)k * n + A + j] + Q[(size_t)(A + j) * n + k]);               \
      row[s] = row[s & (s - 1)] + w;                                                  \
    }                                                                                 \
  }                                                                                   \
  /* The prefix loop runs in contiguous ranges of Gray steps on several threads.  A range   \
   * starts at a multiple of the correction period, where the sequential loop has just     \
   * recomputed the running vector from scratch (do_correction): a range that starts by     \
   * the same recomputation repeats the sequential arithmetic bit for bit.  Each range keeps \
   * its first strict minimum; the ranges are combined in step order (the earliest wins     \
   * ties), then against the loop's initial best (E = 0 at state 0).                       \
   * Without periodic correction the loop stays on one thread. */                         \
  uint64_t steps = (uint64_t)1 << A;                                                  \
  uint64_t per = steps;                                                               \
  int nth = 1;                                                                        \
  if (corr > 0 && steps >= 2 * (uint64_t)corr) {                                      \
    nth = omp_get_max_threads();                                                      \
    uint64_t blocks = steps / (uint64_t)corr;                                         \
    if ((uint64_t)nth > blocks) nth = (int)blocks;                                    \
    per = ((blocks + (uint64_t)nth - 1) / (uint64_t)nth) * (uint64_t)corr;            \
    nth = (int)((steps + per - 1) / per);                                             \
  }                                                                                   \
  double* r_e = (double*)malloc((size_t)nth * sizeof(double));                        \
  uint64_t* r_p = (uint64_t*)malloc((size_t)nth * sizeof(uint64_t));                  \
  uint64_t* r_x = (uint64_t*)malloc((size_t)nth * sizeof(uint64_t));                  \
  int fail = 0;                                                                       \
  _Pragma("omp parallel for schedule(static, 1) num_threads(nth)")                    \
  for (int t = 0; t < nth; ++t) {                                                     \
    uint64_t i0 = (uint64_t)t * per, i1 = i0 + per < steps ? i0 + per : steps;        \
    T* ch = t == 0 ? chunk : (T*)malloc(M * sizeof(T));                               \
    r_e[t] = INFINITY; r_p[t] = 0; r_x[t] = 0;                                        \
    if (!ch) { fail = 1; continue; }                                                  \
    memcpy(ch, diag_bb, M * sizeof(T));                                               \
    uint64_t prev = 0;                                                                \
    if (i0 > 0) { /* the state of step i0 - 1 after its correction */                 \
      prev = (i0 - 1) ^ ((i0 - 1) >> 1);                                              \
      for (int k = 0; k < A; ++k)                                                     \
        if ((prev >> (A - 1 - k)) & 1) {                                              \
          const T* rk = abba + (size_t)k * M;                                         \
          for (size_t s = 0; s < M; ++s) ch[s] += rk[s];                              \
        }                                                                             \
    }                                                                                 \
    for (uint64_t i = i0; i < i1; ++i) {                                              \
      uint64_t gray = i ^ (i >> 1);                                                   \
      if (i > 0) {                                                                    \
        int bit = __builtin_ctzll(gray ^ prev);                                       \
        const T* row = abba + (size_t)(A - 1 - bit) * M;                              \
        if (gray > prev) { for (size_t s = 0; s < M; ++s) ch[s] += row[s]; }          \
        else             { for (size_t s = 0; s < M; ++s) ch[s] -= row[s]; }          \
        if (corr > 0 && (i + 1) % (uint64_t)corr == 0) { /* do_correction */          \
          memcpy(ch, diag_bb, M * sizeof(T));                                         \
          for (int k = 0; k < A; ++k)                                                 \
            if ((gray >> (A - 1 - k)) & 1) {                                          \
              const T* rk = abba + (size_t)k * M;                                     \
              for (size_t s = 0; s < M; ++s) ch[s] += rk[s];                          \
            }                                                                         \
        }                                                                             \
      }                                                                               \
      prev = gray;                                                                    \
      size_t x = 0; T best = ch[0];                                                   \
      for (size_t s = 1; s < M; ++s) if (ch[s] < best) { best = ch[s]; x = s; }       \
      double pe = 0.0;  /* prefix_E = b^T Q_0A b in FP64 (qbf.py:409) */              \
      for (int a = 0; a < A; ++a) {                                                   \
        if (!((gray >> (A - 1 - a)) & 1)) continue;                                   \
        for (int c = 0; c < A; ++c)                                                   \
          if ((gray >> (A - 1 - c)) & 1) pe += Q[(size_t)a * n + c];                  \
      }                                                                               \
      double cand = (double)best + pe;                                                \
      if (cand < r_e[t]) { r_e[t] = cand; r_p[t] = gray; r_x[t] = x; }                \
    }                                                                                 \
    if (t != 0) free(ch);                                                             \
  }                                                                                   \
  double glob_e = 0.0; uint64_t glob_pref = 0, glob_x = 0;                            \
  for (int t = 0; t < nth; ++t)                                                       \
    if (r_e[t] < glob_e) { glob_e = r_e[t]; glob_pref = r_p[t]; glob_x = r_x[t]; }    \
  free(r_e); free(r_p); free(r_x);                                                    \
  if (fail) { free(diag_bb); free(abba); free(chunk); return -2; }                    \
  r->best_e = glob_e;                                                                 \
  r->best_e_int = (int64_t)llround(glob_e);                                           \
  r->glob_pref = glob_pref; r->glob_x = glob_x;                                       \
  r->best_x = (glob_pref << B) | glob_x;                                              \
  r->epochs = (int64_t)steps; r->A = A; r->B = B; r->status = 0;                      \
  free(diag_bb); free(abba); free(chunk);                                             \
  return 0;                                                                           \
}

OQ_DEFINE_TYPED(int32_t, i32)
OQ_DEFINE_TYPED(int64_t, i64)
OQ_DEFINE_TYPED(double, f64)

static double abs_sum(int n, const double* Q) {
  double s = 0.0;
  for (size_t i = 0; i < (size_t)n * n; ++i) s += fabs(Q[i]);
  return s;
}

/* QBF().solve restated.  is_int: Q holds integers.  A < 0: default split.
 * corr: correction period (QBF default 1024; <= 0 disables). */
int oq_qbf_solve(int n, const double* Q, int is_int, int A, int corr, oq_result* r) {
  memset(r, 0, sizeof(*r));
  if (n < 1 || n > 62) return r->status = -1;
  int a = A, b;
  if (a < 0) oq_default_split(n, &a, &b);
  b = n - a;
  if (a < 0 || b < 0 || b > 30 || a > 40) return r->status = -1;
  int rc;
  if (is_int) {
    if (abs_sum(n, Q) < 2147483647.0) rc = qbf_solve_i32(n, Q, a, corr, r);
    else rc = qbf_solve_i64(n, Q, a, corr, r);
  } else {
    rc = qbf_solve_f64(n, Q, a, corr, r);
  }
  if (rc) r->status = rc;
  return rc;
}

/* ReducedProblem (reduced_problem.py:31-46): fix the first k variables to the MSB-first
 * bits of `task`.  Writes the (n-k)^2 reduced matrix and returns prefix_E. */
double oq_reduce(int n, const double* Q, int k, uint64_t task, double* Qr) {
  int m = n - k;
  double pe = 0.0;
  for (int i = 0; i < k; ++i) {
    if (!((task >> (k - 1 - i)) & 1)) continue;
    for (int j = 0; j < k; ++j)
      if ((task >> (k - 1 - j)) & 1) pe += Q[(size_t)i * n + j];
  }
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) Qr[(size_t)i * m + j] = Q[(size_t)(k + i) * n + (k + j)];
  for (int j = 0; j < m; ++j) {
    double d = 0.0;
    for (int i = 0; i < k; ++i)
      if ((task >> (k - 1 - i)) & 1) d += Q[(size_t)i * n + k + j] + Q[(size_t)(k + j) * n + i];
    Qr[(size_t)j * m + j] += d;
  }
  return pe;
}

/* Parallel(QBF, splits_cnt = 2^k).solve restated (parallel.py:145-157, 273-300), with a
 * deterministic cross-task tie rule: the lowest task id wins (the reference takes results
 * in arrival order).  A_sub < 0: each task uses QBF's default split of its n-k variables.
 * nthreads workers process tasks (OpenMP); <= 0 uses all available. */
int oq_parallel_solve(int n, const double* Q, int is_int, int k, int A_sub, int corr,
                      int nthreads, oq_result* r) {
  memset(r, 0, sizeof(*r));
  if (k < 0 || k >= n) return r->status = -1;
  int ntask = 1 << k;
  int m = n - k;
  oq_result* part = (oq_result*)calloc((size_t)ntask, sizeof(oq_result));
  double* pes = (double*)calloc((size_t)ntask, sizeof(double));
  int err = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int t = 0; t < ntask; ++t) {
    double* Qr = (double*)malloc((size_t)m * m * sizeof(double));
    pes[t] = oq_reduce(n, Q, k, (uint64_t)t, Qr);
    if (oq_qbf_solve(m, Qr, is_int, A_sub, corr, &part[t])) err = 1;
    free(Qr);
  }
  if (err) { free(part); free(pes); return r->status = -3; }
  double best = INFINITY; int bt = -1;
  for (int t = 0; t < ntask; ++t) {
    double adj = part[t].best_e + pes[t];
    if (adj < best) { best = adj; bt = t; }
  }
  r->best_e = best;
  r->best_e_int = (int64_t)llround(best);
  r->best_x = ((uint64_t)bt << m) | part[bt].best_x;
  r->glob_pref = part[bt].glob_pref;
  r->glob_x = part[bt].glob_x;
  r->epochs = ntask;
  r->A = part[bt].A; r->B = part[bt].B;
  free(part); free(pes);
  return 0;
}

/* Brute-force scan of all 2^n states (n <= 30): minimum energy (exact for integer Q)
 * and up to `cap` minimising states in increasing X.  Returns the number of minimisers. */
int64_t oq_all_minimisers(int n, const double* Q, uint64_t* out, int64_t cap, double* emin) {
  double* h = (double*)calloc((size_t)n, sizeof(double));
  double e = 0.0, best = 0.0;
  uint64_t g = 0;
  uint64_t total = (uint64_t)1 << n;
  /* pass 1: minimum via Gray walk with local fields */
  for (uint64_t i = 1; i < total; ++i) {
    int bit = __builtin_ctzll(i);
    int v = n - 1 - bit;
    int on = !((g >> bit) & 1);
    double d = Q[(size_t)v * n + v] + h[v];
    e = on ? e + d : e - d;
    for (int j = 0; j < n; ++j) {
      if (j == v) continue;
      double w = Q[(size_t)v * n + j] + Q[(size_t)j * n + v];
      h[j] = on ? h[j] + w : h[j] - w;
    }
    g ^= (uint64_t)1 << bit;
    if (e < best) best = e;
  }
  *emin = best;
  /* pass 2: collect minimisers by direct evaluation near the minimum */
  int64_t cnt = 0;
  for (uint64_t X = 0; X < total; ++X) {
    double ex = oq_energy(n, Q, X);
    if (ex == best) { if (cnt < cap) out[cnt] = X; ++cnt; }
  }
  free(h);
  return cnt;
}
