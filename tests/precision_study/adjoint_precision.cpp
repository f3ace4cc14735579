// Per-region precision study of the hand-written adjoint (p2r_tests_b200/csrc/p2r_adjoint.cuh).
//
// The adjoint header is compiled here on the CPU with a scalar type Q that carries a double and,
// inside the arithmetic regions selected by two bit masks (one for the forward pass, one for the
// reverse sweep), rounds every operand and every result to float: exactly FP32 arithmetic for
// + - * / and sqrt, and the float rounding of sin / cos. Regions are the header's
// P2R_PREC_REGION markers:
//   forward functions  path (helix iterations, Jacobian entries, parameters), covprop (J C J^T),
//                      upd (KalmanUpdate with chi2; its 2x2 determinant stays in double, as in
//                      the FP32 production forward)
//   reverse functions  pathrev (helix iterations, alpha and z), covrev (S, W = S J, J^T S J),
//                      jbar (J-bar = W C), jent (Jacobian entries to their inputs),
//                      updrec (the update's recomputed gain and residual), updrev (its reverse)
// The forward pass and the recomputation inside the reverse sweep are separate masks, as they
// would be separate code in a mixed-precision kernel. tape32 rounds the tape (the propagated state
// stored per layer) to float.
//
// The driver follows the stride-1 tape structure of rev_tape_kernel: forward pass storing the
// propagated state entering every update; reverse from the last layer: update reverse from the
// tape, input state rebuilt with one update of the previous entry, propagation recomputed and
// reversed. Test infrastructure only: tests/precision_study/run_study.py builds and drives it.
#include <cmath>
#include <cstdint>

namespace p2r_study {
enum Region : int { path = 0, covprop, upd, pathrev, covrev, jbar, jent, updrec, updrev, kRegions };
thread_local int g_region = path;
thread_local unsigned g_mask = 0;  // regions rounded to FP32 in the current pass
thread_local unsigned long long g_ops[kRegions] = {};  // arithmetic operations per region
inline void enter(Region r) { g_region = r; }
inline bool f32() { return (g_mask >> g_region) & 1u; }
}  // namespace p2r_study

#define P2R_PREC_REGION(name) ::p2r_study::enter(::p2r_study::name)

namespace p2r {
namespace adj {

struct Q {
  double v;
  Q() : v(0) {}
  Q(double x) : v(x) {}
  operator double() const { return v; }
};
inline double rd(double x) { return p2r_study::f32() ? (double)(float)x : x; }
inline Q mk(double x) {
  ++p2r_study::g_ops[p2r_study::g_region];
  return Q(rd(x));
}
// Q with a double operand: arithmetic the header writes in double on purpose (the update's
// 2x2 determinant, TBB:457), never rounded
#define P2R_Q_BINOP(op)                                                        \
  inline Q operator op(Q a, Q b) { return mk(rd(a.v) op rd(b.v)); }          \
  inline Q operator op(Q a, double b) { return Q(a.v op b); }                 \
  inline Q operator op(double a, Q b) { return Q(a op b.v); }                 \
  inline Q operator op(Q a, float b) { return mk(rd(a.v) op rd(b)); }        \
  inline Q operator op(float a, Q b) { return mk(rd(a) op rd(b.v)); }        \
  inline Q operator op(Q a, int b) { return mk(rd(a.v) op rd((double)b)); }  \
  inline Q operator op(int a, Q b) { return mk(rd((double)a) op rd(b.v)); }
P2R_Q_BINOP(+)
P2R_Q_BINOP(-)
P2R_Q_BINOP(*)
P2R_Q_BINOP(/)
#undef P2R_Q_BINOP
inline Q operator-(Q a) { return Q(-a.v); }
inline Q& operator+=(Q& a, Q b) { return a = a + b; }
inline Q& operator-=(Q& a, Q b) { return a = a - b; }
inline Q& operator*=(Q& a, Q b) { return a = a * b; }
inline bool operator<(Q a, Q b) { return a.v < b.v; }
inline bool operator>(Q a, Q b) { return a.v > b.v; }
inline bool operator!=(Q a, Q b) { return a.v != b.v; }
inline bool operator==(Q a, Q b) { return a.v == b.v; }
inline Q sqrt_(Q x) { return mk(std::sqrt(rd(x.v))); }
inline Q abs_(Q x) { return Q(std::fabs(x.v)); }
inline void sincos_(Q x, Q* s, Q* c) {
  const double a = rd(x.v);
  *s = mk(std::sin(a));
  *c = mk(std::cos(a));
}

}  // namespace adj
}  // namespace p2r

#include "../../p2r_tests_b200/csrc/p2r_adjoint.cuh"

using p2r::adj::Q;

namespace {

inline Q tape_round(Q x, bool f) { return f ? Q((double)(float)x.v) : x; }

}  // namespace

extern "C" {

// One track's chained forward + adjoint (nlayer layers) in the stride-1 tape structure.
// par0[6], cov0[21], q; hits nlayer x 9 (pos 3, cov 6); dr[nlayer]; bz; seeds g_par[6],
// g_cov[21], g_chi2. Outputs: d/d par0 (6), cov0 (21), hits (nlayer x 9), dr (nlayer),
// bz (1). fwd_mask / rev_mask: regions in FP32 in the forward pass / the reverse sweep.
void study_track(const double* par0, const double* cov0, int q, const double* hits, int nlayer, const double* dr,
                 double bz, const double* g_par, const double* g_cov, double g_chi2, unsigned fwd_mask,
                 unsigned rev_mask, int tape32, double* o_par, double* o_cov, double* o_hits, double* o_dr,
                 double* o_bz) {
  namespace adj = p2r::adj;
  const Q kfact = Q(100.0 / (-0.299792458 * bz));
  p2r_study::g_mask = fwd_mask;
  p2r_study::enter(p2r_study::path);
  const Q k = Q((double)q) * kfact;
  const Q kinv = Q(1.0) / k;
  Q par[6], cov[21];
  for (int i = 0; i < 6; ++i) par[i] = Q(par0[i]);
  for (int i = 0; i < 21; ++i) cov[i] = Q(cov0[i]);
  Q tp[64][6], tc[64][21];
  for (int l = 0; l < nlayer; ++l) {
    Q hp[3], hc[6];
    for (int i = 0; i < 3; ++i) hp[i] = Q(hits[l * 9 + i]);
    for (int i = 0; i < 6; ++i) hc[i] = Q(hits[l * 9 + 3 + i]);
    adj::PropTape<Q> t;
    p2r_study::enter(p2r_study::path);
    const Q r = adj::hipo(hp[0], hp[1]) + Q(dr[l]);
    adj::prop_fwd(par, cov, k, kinv, r, t, par, cov);
    for (int i = 0; i < 6; ++i) tp[l][i] = tape_round(par[i], tape32);
    for (int i = 0; i < 21; ++i) tc[l][i] = tape_round(cov[i], tape32);
    adj::upd_fwd(par, cov, hp, hc);
  }
  // reverse sweep
  p2r_study::g_mask = rev_mask;
  Q pb[6], cb[21];
  for (int i = 0; i < 6; ++i) pb[i] = Q(g_par[i]);
  for (int i = 0; i < 21; ++i) cb[i] = Q(g_cov[i]);
  const Q chi2b = Q(g_chi2);
  Q kbar = 0, kinvbar = 0;
  for (int l = nlayer - 1; l >= 0; --l) {
    Q hp[3], hc[6], hpb[3], hcb[6];
    for (int i = 0; i < 3; ++i) hp[i] = Q(hits[l * 9 + i]);
    for (int i = 0; i < 6; ++i) hc[i] = Q(hits[l * 9 + 3 + i]);
    adj::upd_rev(tp[l], tc[l], hp, hc, pb, cb, chi2b, hpb, hcb);
    Q sp[6], sc[21];
    if (l == 0) {
      for (int i = 0; i < 6; ++i) sp[i] = Q(par0[i]);
      for (int i = 0; i < 21; ++i) sc[i] = Q(cov0[i]);
    } else {
      Q hq[3], hqc[6];
      for (int i = 0; i < 6; ++i) sp[i] = tp[l - 1][i];
      for (int i = 0; i < 21; ++i) sc[i] = tc[l - 1][i];
      for (int i = 0; i < 3; ++i) hq[i] = Q(hits[(l - 1) * 9 + i]);
      for (int i = 0; i < 6; ++i) hqc[i] = Q(hits[(l - 1) * 9 + 3 + i]);
      adj::upd_fwd(sp, sc, hq, hqc);
    }
    p2r_study::enter(p2r_study::path);
    const Q rh = adj::hipo(hp[0], hp[1]);
    const Q r = rh + Q(dr[l]);
    adj::PropTape<Q> t;
    Q pp[6], pc[21];
    adj::prop_fwd(sp, sc, k, kinv, r, t, pp, pc);
    Q pin[6], cin[21], rbar = 0;
    adj::prop_rev(t, sp, sc, k, kinv, r, pb, cb, pin, cin, rbar, kbar, kinvbar);
    for (int i = 0; i < 6; ++i) pb[i] = pin[i];
    for (int i = 0; i < 21; ++i) cb[i] = cin[i];
    p2r_study::enter(p2r_study::pathrev);
    if (rh > Q(0.0)) {
      const Q irh = Q(1.0) / rh;
      hpb[0] += rbar * hp[0] * irh;
      hpb[1] += rbar * hp[1] * irh;
    }
    for (int i = 0; i < 3; ++i) o_hits[l * 9 + i] = hpb[i].v;
    for (int i = 0; i < 6; ++i) o_hits[l * 9 + 3 + i] = hcb[i].v;
    o_dr[l] = rbar.v;
  }
  for (int i = 0; i < 6; ++i) o_par[i] = pb[i].v;
  for (int i = 0; i < 21; ++i) o_cov[i] = cb[i].v;
  // k = q kfact(Bz): dk/dBz = -k / Bz (kinv = 1/k)
  *o_bz = ((kbar.v - kinvbar.v * kinv.v * kinv.v) * (-k.v / bz));
  p2r_study::g_mask = 0;
}

int study_regions(void) { return p2r_study::kRegions; }

// Arithmetic operations (+ - * / sqrt sin cos, each counted once) per region since the last
// reset, in the calling thread; reset clears them.
void study_ops(unsigned long long* out, int reset) {
  for (int r = 0; r < p2r_study::kRegions; ++r) {
    out[r] = p2r_study::g_ops[r];
    if (reset) p2r_study::g_ops[r] = 0;
  }
}

}  // extern "C"
