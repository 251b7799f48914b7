// Host-only harness for tests/test_tc2_tables.py: exports the 16-bit pair form's host-side
// planning (eligibility, the power-of-two unit of the rounded form, the per-problem table of
// constants) from the library's own header so the test can check their algebra on the CPU.
// Built by the test with g++; not part of the library.
#include "qb_tc2.cuh"

extern "C" {

int h_tc2_tab_size() { return (int)sizeof(qb::Tc2Tab); }

int h_tc2_u16_eligible(int n, const double* W, float* dmin) { return qb::tc2_u16_eligible(n, W, dmin) ? 1 : 0; }

int h_tc2_u16_quantized(int n, const double* W, double abs_sum, double* sigma, float* dmin, double* eps) {
  return qb::tc2_u16_quantized(n, W, abs_sum, sigma, dmin, eps) ? 1 : 0;
}

void h_tc2_u16_tables(const float* gamma, float dmin, qb::Tc2Tab* out) { qb::tc2_u16_tables(gamma, dmin, out); }

}  // extern "C"
