// Host (double) instantiation of the library's per-layer adjoint header, for the CPU
// finite-difference test in tests/test_adjoint_cpu.py. Compiled by that test with g++.
#include "../p2r_tests_b200/csrc/p2r_adjoint.cuh"

using namespace p2r::adj;

namespace {
double kfact_of(double bz) { return 100 / (-0.299792458 * bz); }
}  // namespace

extern "C" {

// One layer forward in double, state in place; returns the update's chi2.
double adjh_layer_fwd(double* p6, double* c21, int q, double bz, const double* hp3, const double* hc6, double dr) {
  double p[6], c[21], hp[3], hc[6];
  for (int i = 0; i < 6; ++i) p[i] = p6[i];
  for (int i = 0; i < 21; ++i) c[i] = c21[i];
  for (int i = 0; i < 3; ++i) hp[i] = hp3[i];
  for (int i = 0; i < 6; ++i) hc[i] = hc6[i];
  const double k = q * kfact_of(bz);
  const double chi2 = layer_fwd(p, c, k, 1.0 / k, hp, hc, dr);
  for (int i = 0; i < 6; ++i) p6[i] = p[i];
  for (int i = 0; i < 21; ++i) c21[i] = c[i];
  return chi2;
}

// Its reverse. pb6 / cb21: in = adjoints of the outputs, out = adjoints of the inputs.
void adjh_layer_rev(const double* p6, const double* c21, int q, double bz, const double* hp3, const double* hc6,
                    double dr, double* pb6, double* cb21, double chi2b, double* hpb3, double* hcb6, double* drb,
                    double* bzb) {
  double p[6], c[21], hp[3], hc[6], pb[6], cb[21], hpb[3], hcb[6];
  for (int i = 0; i < 6; ++i) p[i] = p6[i], pb[i] = pb6[i];
  for (int i = 0; i < 21; ++i) c[i] = c21[i], cb[i] = cb21[i];
  for (int i = 0; i < 3; ++i) hp[i] = hp3[i];
  for (int i = 0; i < 6; ++i) hc[i] = hc6[i];
  const double k = q * kfact_of(bz), kinv = 1.0 / k;
  double d = 0, kbar = 0, kinvbar = 0;
  layer_rev(p, c, k, kinv, hp, hc, dr, pb, cb, chi2b, hpb, hcb, d, kbar, kinvbar);
  for (int i = 0; i < 6; ++i) pb6[i] = pb[i];
  for (int i = 0; i < 21; ++i) cb21[i] = cb[i];
  for (int i = 0; i < 3; ++i) hpb3[i] = hpb[i];
  for (int i = 0; i < 6; ++i) hcb6[i] = hcb[i];
  *drb = d;
  // k = q * kfact(bz), dk/dbz = -k / bz
  *bzb = (kbar - kinvbar * kinv * kinv) * (-k / bz);
}

}  // extern "C"
