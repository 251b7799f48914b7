// Host-only harness for tests/test_host_planning.py: exports host-side planning from the
// library's own headers (the tensor-core shard plan, the record geometry, the tie order, the
// 16-bit pair form's eligibility, the power-of-two unit of its rounded form and its table of
// constants) so the test can check them on the CPU.
// Built by the test with g++; not part of the library.
#include "qb_tc2.cuh"

extern "C" {

int h_tc2_tab_size() { return (int)sizeof(qb::Tc2Tab); }

int h_tc2_u16_eligible(int n, const double* W, float* dmin) { return qb::tc2_u16_eligible(n, W, dmin) ? 1 : 0; }

int h_tc2_u16_quantized(int n, const double* W, double abs_sum, double* sigma, float* dmin, double* eps) {
  return qb::tc2_u16_quantized(n, W, abs_sum, sigma, dmin, eps) ? 1 : 0;
}

void h_tc2_u16_tables(const float* gamma, float dmin, qb::Tc2Tab* out) { qb::tc2_u16_tables(gamma, dmin, out); }

// tc_plan of one shard: u64 {tile_begin, tile_end, rec_begin, rec_count, states},
// f64 {scale, eps}, i32 {nt, gl, exact}
void h_tc_plan(int n, int is_int, double abs_sum, int shard_idx, int shard_cnt, int gl, uint64_t* u64, double* f64,
               int* i32) {
  qb::TcPlan p;
  qb::tc_plan(n, is_int != 0, abs_sum, shard_idx, shard_cnt, &p, gl);
  const uint64_t u[5] = {p.tile_begin, p.tile_end, p.rec_begin, p.rec_count, p.states};
  for (int i = 0; i < 5; ++i) u64[i] = u[i];
  f64[0] = p.scale;
  f64[1] = p.eps;
  i32[0] = p.nt;
  i32[1] = p.gl;
  i32[2] = p.exact ? 1 : 0;
}

// record_states of one record of a geometry: its base state and free-bit mask
void h_record_states(int kind, int n, int a, int b, int sbits, int cbbits, int gubits, int gl, int fbits, uint64_t r,
                     uint64_t* base, uint64_t* freem) {
  qb::RecGeom g{};
  g.kind = kind;
  g.n = n;
  g.a = a;
  g.b = b;
  g.sbits = sbits;
  g.cbbits = cbbits;
  g.gubits = gubits;
  g.gl = gl;
  g.fbits = fbits;
  qb::record_states(g, r, base, freem);
}

uint64_t h_grayrank64(uint64_t g) { return qb::grayrank64(g); }

// the order key that decides ties between equal minima
uint64_t h_tie_key(int kind, int n, int k, int A, int B, uint64_t X) {
  const qb::TieRule r{kind, n, k, A, B};
  return qb::tie_key(r, X);
}

}  // extern "C"
