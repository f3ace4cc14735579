// Hand-written reverse-mode derivative (adjoint) of one layer of the p2r hot path:
// propagateToR (TBB:656-812) followed by KalmanUpdate (TBB:433-642), plus the update's
// chi2 = res^T inv(R) res. Templated on the scalar type and usable on host and device:
// the device kernel instantiates it in float, a host unit test in double (checked against
// central finite differences of the double forward in this same header).
//
// The forward formulas are the reference's (see p2r_math.cuh for the float production
// forward); the derivatives are those of the implemented arithmetic: the five fixed
// helix iterations, the 4th-order sincos4 polynomials and the 1 um convergence branch of
// the path derivatives (TBB:714) held fixed at the primal point.
//
// Symmetric matrices are packed lower-triangle (TBB:46-54). The adjoint of a packed
// covariance treats each packed element as one variable: an off-diagonal slot collects
// the derivatives of both (i,j) and (j,i) uses.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define P2R_HD __host__ __device__ __forceinline__
#else
#define P2R_HD inline
#endif
#if defined(__CUDA_ARCH__)
#define P2R_UNROLL _Pragma("unroll")
#else
#define P2R_UNROLL
#endif

// Precision-study markers: each names the arithmetic region the statements after it belong to
// (path, covprop, upd in the forward functions; pathrev, covrev, jbar, jent, updrec, updrev in
// the reverse ones). They expand to nothing unless a study build defines P2R_PREC_REGION
// (tests/precision_study/adjoint_precision.cpp, which runs this code with chosen regions
// rounded to FP32).
#ifndef P2R_PREC_REGION
#define P2R_PREC_REGION(name)
#endif

namespace p2r {
namespace adj {

P2R_HD constexpr int S6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

P2R_HD float sqrt_(float x) { return sqrtf(x); }
P2R_HD double sqrt_(double x) { return sqrt(x); }
P2R_HD float abs_(float x) { return fabsf(x); }
P2R_HD double abs_(double x) { return fabs(x); }
P2R_HD void sincos_(float x, float* s, float* c) {
#if defined(__CUDA_ARCH__)
  sincosf(x, s, c);
#else
  *s = sinf(x);
  *c = cosf(x);
#endif
}
P2R_HD void sincos_(double x, double* s, double* c) {
#if defined(__CUDA_ARCH__)
  sincos(x, s, c);
#else
  *s = sin(x);
  *c = cos(x);
#endif
}

template <class T>
P2R_HD T hipo(T x, T y) { return sqrt_(x * x + y * y); }

// sincos4 (TBB:644-652) with omc = 1 - c formed without cancellation, and its derivative
template <class T>
P2R_HD void sincos4(T x, T& s, T& c, T& omc) {
  const T x2 = x * x;
  omc = T(0.5f) * x2 - T(0.04166667f) * x2 * x2;
  c = T(1) - omc;
  s = x - T(0.16666667f) * x * x2;
}
template <class T>
P2R_HD T sincos4_bar(T x, T sbar, T cbar) {
  return cbar * (-x + T(4) * T(0.04166667f) * x * x * x) + sbar * (T(1) - T(3) * T(0.16666667f) * x * x);
}

// Forward values of one propagateToR that its reverse needs.
template <class T>
struct PropTape {
  T r00, pt, cP, sP;
  T xo[5], yo[5], px[5], py[5], r0[5];  // at the start of each helix iteration
  T D, dDdx, dDdy, dDdipt, dDdphi;
  T alpha, dadx, dady, dadipt, dadphi, sa, ca, omc, cT, sT, isT;
  T J00, J01, J03, J04, J10, J11, J13, J14, J20, J21, J23, J24, J25, J40, J41, J43, J44;
};

// propagateToR of (ip, ic) to radius r with k = q*kfact, kinv = 1/k, recording the tape.
template <class T>
P2R_HD void prop_fwd(const T (&ip)[6], const T (&ic)[21], T k, T kinv, T r, PropTape<T>& t, T (&op)[6],
                     T (&oc)[21]) {
  P2R_PREC_REGION(path);
  const T xin = ip[0], yin = ip[1], zin = ip[2], iptin = ip[3], phiin = ip[4], thetain = ip[5];
  t.r00 = hipo(xin, yin);
  t.pt = T(1) / iptin;
  sincos_(phiin, &t.sP, &t.cP);
  T px = t.cP * t.pt, py = t.sP * t.pt;
  T dDdx = 0, dDdy = 0;
  if (t.r00 > T(0)) {
    const T ir00 = T(1) / t.r00;
    dDdx = -xin * ir00;
    dDdy = -yin * ir00;
  }
  T dDdipt = 0, dDdphi = 0, D = 0, sina, cosa, omc;
  T xo = xin, yo = yin;
  const T pt = t.pt;
P2R_UNROLL
  for (int i = 0; i < 5; ++i) {
    t.xo[i] = xo;
    t.yo[i] = yo;
    t.px[i] = px;
    t.py[i] = py;
    const T r0 = hipo(xo, yo);
    t.r0[i] = r0;
    const T id = r - r0;
    D += id;
    sincos4(id * iptin * kinv, sina, cosa, omc);
    // path derivatives once the step is below 1 um (TBB:714); before that the reference adds
    // increments scaled by oor0 = 0, which leave the sums unchanged and are skipped here
    if (i + 1 != 5 && r0 > T(0) && abs_(r - r0) < T(0.0001f)) {
      const T oor0 = T(1) / r0;
      // the increments of TBB:716-734 with their shared terms formed once (a1, a2: the
      // momentum after the step; k*dadx = kn*xo, k*dady = kn*yo since k*kinv = 1)
      const T a1 = px * cosa - py * sina, a2 = py * cosa + px * sina;
      const T kn = -iptin * oor0;
      const T g = (T(1) + kn * (xo * a1 + yo * a2)) * oor0;
      dDdx -= xo * g;
      dDdy -= yo * g;
      const T tt = id * kinv * iptin;  // dadipt * ipt
      dDdipt -= k * (xo * (a1 * tt - a2 + py) + yo * (a2 * tt + a1 - px)) * pt * oor0;
      dDdphi += k * (xo * (py * sina + px * cosa - px) - yo * (a2 - py)) * oor0;
    }
    xo = xo + k * (px * sina - py * omc);
    yo = yo + k * (py * sina + px * omc);
    const T pxold = px;
    px = px * cosa - py * sina;
    py = py * cosa + pxold * sina;
  }
  t.D = D;
  t.dDdx = dDdx;
  t.dDdy = dDdy;
  t.dDdipt = dDdipt;
  t.dDdphi = dDdphi;
  t.alpha = D * iptin * kinv;
  t.dadx = dDdx * iptin * kinv;
  t.dady = dDdy * iptin * kinv;
  t.dadipt = (iptin * dDdipt + D) * kinv;
  t.dadphi = dDdphi * iptin * kinv;
  sincos4(t.alpha, t.sa, t.ca, t.omc);
  const T cP = t.cP, sP = t.sP, ca = t.ca, sa = t.sa, alpha = t.alpha;
  const T dadx = t.dadx, dady = t.dady, dadipt = t.dadipt, dadphi = t.dadphi;
  // TBB:753-807 with their shared factors formed once: U = cos(phi + alpha), V = sin(phi + alpha),
  // w = ipt dadipt, k pt; e.g. J03 = k (cP (w ca - sa) + sP (omc - w sa)) pt^2 = k pt^2 (w U - V + sP)
  const T U = cP * ca - sP * sa, V = sP * ca + cP * sa, w = iptin * dadipt, d1 = dadphi + T(1);
  const T kp = k * pt, kp2 = kp * pt;
  t.J00 = T(1) + dadx * U * kp;
  t.J01 = dady * U * kp;
  t.J03 = (w * U - V + sP) * kp2;
  t.J04 = (d1 * U - cP) * kp;
  t.J10 = dadx * V * kp;
  t.J11 = T(1) + dady * V * kp;
  t.J13 = (w * V + U - cP) * kp2;
  t.J14 = (d1 * V - sP) * kp;
  sincos_(thetain, &t.sT, &t.cT);
  t.isT = T(1) / t.sT;
  const T cT = t.cT, isT = t.isT;
  const T G = kp * cT * isT;  // rows 2 and 4 share (dadx, dady, ., ., dadphi, .): J2 = G (those) + ...
  t.J20 = G * dadx;
  t.J21 = G * dady;
  t.J23 = G * pt * (w - alpha);
  t.J24 = G * dadphi;
  t.J25 = -kp * alpha * isT * isT;
  t.J40 = dadx;
  t.J41 = dady;
  t.J43 = dadipt;
  t.J44 = T(1) + dadphi;
  P2R_PREC_REGION(covprop);
  // rows 0, 1, 2, 4 of J*C (rows 3 and 5 are rows 3 and 5 of C); not kept on the tape:
  // the reverse forms J-bar as (S J) C instead of S (J C)
  T T0[6], T1[6], T2[6], T4[6];
P2R_UNROLL
  for (int j = 0; j < 6; ++j) {
    const T c0 = ic[S6(0, j)], c1 = ic[S6(1, j)], c2 = ic[S6(2, j)], c3 = ic[S6(3, j)], c4 = ic[S6(4, j)],
            c5 = ic[S6(5, j)];
    T0[j] = t.J00 * c0 + t.J01 * c1 + t.J03 * c3 + t.J04 * c4;
    T1[j] = t.J10 * c0 + t.J11 * c1 + t.J13 * c3 + t.J14 * c4;
    const T n = dadx * c0 + dady * c1 + dadphi * c4;  // row 4 = n + dadipt c3 + c4, row 2 = G n + ...
    T2[j] = G * n + c2 + t.J23 * c3 + t.J25 * c5;
    T4[j] = n + dadipt * c3 + c4;
  }
  // C' = (J C) J^T, lower triangle
P2R_UNROLL
  for (int i = 0; i < 6; ++i) {
    T Ti[6];
P2R_UNROLL
    for (int j = 0; j < 6; ++j)
      Ti[j] = i == 0 ? T0[j] : i == 1 ? T1[j] : i == 2 ? T2[j] : i == 4 ? T4[j] : ic[S6(i, j)];
    oc[S6(i, 0)] = Ti[0] * t.J00 + Ti[1] * t.J01 + Ti[3] * t.J03 + Ti[4] * t.J04;
    if (i >= 1) oc[S6(i, 1)] = Ti[0] * t.J10 + Ti[1] * t.J11 + Ti[3] * t.J13 + Ti[4] * t.J14;
    if (i >= 2) {
      const T n = Ti[0] * dadx + Ti[1] * dady + Ti[4] * dadphi;
      oc[S6(i, 2)] = G * n + Ti[2] + Ti[3] * t.J23 + Ti[5] * t.J25;
      if (i >= 4) oc[S6(i, 4)] = n + Ti[3] * dadipt + Ti[4];
    }
    if (i >= 3) oc[S6(i, 3)] = Ti[3];
    if (i >= 5) oc[S6(i, 5)] = Ti[5];
  }
  P2R_PREC_REGION(path);
  op[0] = xo;
  op[1] = yo;
  op[2] = zin + k * alpha * cT * pt * isT;
  op[3] = iptin;
  op[4] = phiin + alpha;
  op[5] = thetain;
}

// Reverse of prop_fwd. In: the tape, the input (ip, ic), adjoints pb_out / cb_out of the
// outputs. Out: adjoints pb_in / cb_in of the inputs (overwritten); rbar, kbar and kinvbar
// are accumulated (+=).
template <class T>
P2R_HD void prop_rev(const PropTape<T>& t, const T (&ip)[6], const T (&ic)[21], T k, T kinv, T r,
                     const T (&pb_out)[6], const T (&cb_out)[21], T (&pb_in)[6], T (&cb_in)[21], T& rbar, T& kbar,
                     T& kinvbar) {
  P2R_PREC_REGION(pathrev);
  const T x = ip[0], y = ip[1], ipt = ip[3];
  const T pt = t.pt, cP = t.cP, sP = t.sP, ca = t.ca, sa = t.sa, cT = t.cT, sT = t.sT, isT = t.isT;
  const T alpha = t.alpha, dadx = t.dadx, dady = t.dady, dadipt = t.dadipt, dadphi = t.dadphi;

  T xob = pb_out[0], yob = pb_out[1];
  const T zb = pb_out[2];
  T iptb = pb_out[3], phib = pb_out[4], alphab = pb_out[4], thetab = pb_out[5];
  // z' = z + k*alpha*cT*pt*isT
  kbar += zb * alpha * cT * pt * isT;
  alphab += zb * k * cT * pt * isT;
  T cTb = zb * k * alpha * pt * isT;
  T ptb = zb * k * alpha * cT * isT;
  T isTb = zb * k * alpha * cT * pt;

  P2R_PREC_REGION(covrev);
  // ---- C' = J C J^T: S = Gbar + Gbar^T, Jbar = S (J C) = (S J) C, cbar = packed(J^T S J)
  T S[6][6];
P2R_UNROLL
  for (int i = 0; i < 6; ++i)
P2R_UNROLL
    for (int j = 0; j < 6; ++j) S[i][j] = i == j ? T(2) * cb_out[S6(i, i)] : cb_out[S6(i, j)];
  // W = S J, column by column: column j gives column j of M = J^T W (into cb_in) and its share
  // of Jbar = W C, Jbar_ab += W_aj C_jb, at the non-trivial entries of J. W is never held whole
  // (the same operations in the same order as forming W first: J-bar sums over j = 0..5).
  T J00b = 0, J01b = 0, J03b = 0, J04b = 0, J10b = 0, J11b = 0, J13b = 0, J14b = 0;
  T J20b = 0, J21b = 0, J23b = 0, J24b = 0, J25b = 0, J40b = 0, J41b = 0, J43b = 0, J44b = 0;
P2R_UNROLL
  for (int j = 0; j < 6; ++j) {
    P2R_PREC_REGION(covrev);
    T w[6];
P2R_UNROLL
    for (int a = 0; a < 6; ++a) {
      if (j == 0) w[a] = S[a][0] * t.J00 + S[a][1] * t.J10 + S[a][2] * t.J20 + S[a][4] * t.J40;
      if (j == 1) w[a] = S[a][0] * t.J01 + S[a][1] * t.J11 + S[a][2] * t.J21 + S[a][4] * t.J41;
      if (j == 2) w[a] = S[a][2];
      if (j == 3) w[a] = S[a][0] * t.J03 + S[a][1] * t.J13 + S[a][2] * t.J23 + S[a][3] + S[a][4] * t.J43;
      if (j == 4) w[a] = S[a][0] * t.J04 + S[a][1] * t.J14 + S[a][2] * t.J24 + S[a][4] * t.J44;
      if (j == 5) w[a] = S[a][2] * t.J25 + S[a][5];
    }
    T M[6];
    M[0] = t.J00 * w[0] + t.J10 * w[1] + t.J20 * w[2] + t.J40 * w[4];
    M[1] = t.J01 * w[0] + t.J11 * w[1] + t.J21 * w[2] + t.J41 * w[4];
    M[2] = w[2];
    M[3] = t.J03 * w[0] + t.J13 * w[1] + t.J23 * w[2] + w[3] + t.J43 * w[4];
    M[4] = t.J04 * w[0] + t.J14 * w[1] + t.J24 * w[2] + t.J44 * w[4];
    M[5] = t.J25 * w[2] + w[5];
P2R_UNROLL
    for (int i = j; i < 6; ++i) cb_in[S6(i, j)] = i == j ? T(0.5f) * M[i] : M[i];
    P2R_PREC_REGION(jbar);
    const T c0 = ic[S6(j, 0)], c1 = ic[S6(j, 1)], c3 = ic[S6(j, 3)], c4 = ic[S6(j, 4)], c5 = ic[S6(j, 5)];
    J00b += w[0] * c0; J01b += w[0] * c1; J03b += w[0] * c3; J04b += w[0] * c4;
    J10b += w[1] * c0; J11b += w[1] * c1; J13b += w[1] * c3; J14b += w[1] * c4;
    J20b += w[2] * c0; J21b += w[2] * c1; J23b += w[2] * c3; J24b += w[2] * c4; J25b += w[2] * c5;
    J40b += w[4] * c0; J41b += w[4] * c1; J43b += w[4] * c3; J44b += w[4] * c4;
  }

  P2R_PREC_REGION(jent);
  // ---- Jacobian entries -> their inputs
  const T U = cP * ca - sP * sa, V = sP * ca + cP * sa, w = ipt * dadipt;
  T Ub = 0, Vb = 0, wb = 0, dadxb = 0, dadyb = 0, dadiptb = 0, dadphib = 0, cPb = 0, sPb = 0;
  const T kp = k * pt;
  {
    // J00 = 1 + k dadx U pt, J01 = k dady U pt, J10 = k dadx V pt, J11 = 1 + k dady V pt
    const T a = J00b * dadx + J01b * dady, b = J10b * dadx + J11b * dady;
    const T e = a * U + b * V;
    kbar += e * pt;
    ptb += e * k;
    Ub += a * kp;
    Vb += b * kp;
    dadxb += (J00b * U + J10b * V) * kp;
    dadyb += (J01b * U + J11b * V) * kp;
  }
  {
    // J03 = k Q3 pt^2, Q3 = w U - V + sP;  J13 = k Q13 pt^2, Q13 = w V + U - cP
    const T e = J03b * (w * U - V + sP) + J13b * (w * V + U - cP);
    kbar += e * pt * pt;
    ptb += T(2) * e * kp;
    const T g3 = J03b * kp * pt, g13 = J13b * kp * pt;
    wb += g3 * U + g13 * V;
    Ub += g3 * w + g13;
    Vb += g13 * w - g3;
    sPb += g3;
    cPb -= g13;
  }
  {
    // J04 = k Q4 pt, Q4 = (dadphi + 1) U - cP;  J14 = k Q14 pt, Q14 = (dadphi + 1) V - sP
    const T d1 = dadphi + T(1);
    const T e = J04b * (d1 * U - cP) + J14b * (d1 * V - sP);
    kbar += e * pt;
    ptb += e * k;
    const T g4 = J04b * kp, g14 = J14b * kp;
    dadphib += g4 * U + g14 * V;
    Ub += g4 * d1;
    Vb += g14 * d1;
    cPb -= g4;
    sPb -= g14;
  }
  {
    const T G = k * cT * pt * isT;
    const T Gb = J20b * dadx + J21b * dady + J23b * pt * (w - alpha) + J24b * dadphi;
    dadxb += J20b * G;
    dadyb += J21b * G;
    ptb += J23b * G * (w - alpha);
    wb += J23b * G * pt;
    alphab -= J23b * G * pt;
    dadphib += J24b * G;
    kbar += Gb * cT * pt * isT;
    cTb += Gb * k * pt * isT;
    ptb += Gb * k * cT * isT;
    isTb += Gb * k * cT * pt;
  }
  kbar -= J25b * alpha * pt * isT * isT;
  alphab -= J25b * k * pt * isT * isT;
  ptb -= J25b * k * alpha * isT * isT;
  isTb -= J25b * T(2) * k * alpha * pt * isT;
  dadxb += J40b;
  dadyb += J41b;
  dadiptb += J43b;
  dadphib += J44b;
  iptb += wb * dadipt;
  dadiptb += wb * ipt;
  cPb += Ub * ca + Vb * sa;
  sPb += -Ub * sa + Vb * ca;
  const T cab = Ub * cP + Vb * sP;
  const T sab = -Ub * sP + Vb * cP;
  alphab += sincos4_bar(alpha, sab, cab);
  thetab += -cTb * sT - isTb * cT * isT * isT;

  P2R_PREC_REGION(pathrev);
  // ---- alpha, dad* from D and the path derivatives
  T Db = alphab * ipt * kinv + dadiptb * kinv;
  iptb += alphab * t.D * kinv + dadxb * t.dDdx * kinv + dadyb * t.dDdy * kinv + dadiptb * t.dDdipt * kinv +
          dadphib * t.dDdphi * kinv;
  kinvbar += alphab * t.D * ipt + dadxb * t.dDdx * ipt + dadyb * t.dDdy * ipt + dadiptb * (ipt * t.dDdipt + t.D) +
             dadphib * t.dDdphi * ipt;
  const T dDdxb = dadxb * ipt * kinv, dDdyb = dadyb * ipt * kinv;
  const T dDdiptb = dadiptb * ipt * kinv, dDdphib = dadphib * ipt * kinv;

  // ---- the five helix iterations, last to first
  T pxb = 0, pyb = 0;
P2R_UNROLL
  for (int i = 4; i >= 0; --i) {
    const T xo = t.xo[i], yo = t.yo[i], px = t.px[i], py = t.py[i], r0 = t.r0[i];
    const T id = r - r0;
    const T a = id * ipt * kinv;
    T sai, cai, omci;
    sincos4(a, sai, cai, omci);
    // xo' = xo + k(px sa - py(1-ca)), yo' = yo + k(py sa + px(1-ca)),
    // px' = px ca - py sa, py' = py ca + px sa
    T sab_i = xob * k * px + yob * k * py - pxb * py + pyb * px;
    T cab_i = xob * k * py - yob * k * px + pxb * px + pyb * py;
    kbar += xob * (px * sai - py * omci) + yob * (py * sai + px * omci);
    const T pxb_n = xob * k * sai + yob * k * omci + pxb * cai + pyb * sai;
    const T pyb_n = -xob * k * omci + yob * k * sai - pxb * sai + pyb * cai;
    pxb = pxb_n;
    pyb = pyb_n;
    T idb = Db;
    T r0b = 0;
    const T ir0 = r0 > T(0) ? T(1) / r0 : T(0);  // one reciprocal per iteration, used twice
    if (i < 4) {
      const T o = abs_(r - r0) < T(0.0001f) ? ir0 : T(0);
      if (o != T(0)) {
        // Reverse of the increments in prop_fwd's factored form: with a1, a2 the momentum
        // after the step, s = xo a1 + yo a2, kn = -ipt o, g = (1 + kn s) o, tt = id kinv ipt:
        //   dDdx -= xo g,  dDdy -= yo g,
        //   dDdipt -= k E pt o,  E = xo (a1 tt - a2 + py) + yo (a2 tt + a1 - px),
        //   dDdphi += k F o,     F = xo (py sa + px ca - px) - yo (a2 - py).
        const T ca = cai, sa = sai;
        const T a1 = px * ca - py * sa, a2 = py * ca + px * sa;
        const T sxy = xo * a1 + yo * a2;
        const T kn = -ipt * o;
        const T g = (T(1) + kn * sxy) * o;
        const T tt = id * kinv * ipt;
        const T ex = a1 * tt - a2 + py, ey = a2 * tt + a1 - px;
        const T E = xo * ex + yo * ey;
        const T fx = py * sa + px * ca - px, fy = a2 - py;
        const T F = xo * fx - yo * fy;
        T ob = 0, a1b = 0, a2b = 0;
        // dDdx, dDdy
        const T gb = -(dDdxb * xo + dDdyb * yo);
        xob -= dDdxb * g;
        yob -= dDdyb * g;
        ob += gb * (T(1) + kn * sxy);
        const T knb = gb * o * sxy, sb = gb * o * kn;
        iptb -= knb * o;
        ob -= knb * ipt;
        xob += sb * a1;
        yob += sb * a2;
        a1b += sb * xo;
        a2b += sb * yo;
        // dDdipt
        const T Tb = -dDdiptb;
        kbar += Tb * E * pt * o;
        ptb += Tb * k * E * o;
        ob += Tb * k * E * pt;
        const T Eb = Tb * k * pt * o;
        xob += Eb * ex;
        yob += Eb * ey;
        a1b += Eb * (xo * tt + yo);
        a2b += Eb * (yo * tt - xo);
        pyb += Eb * xo;
        pxb -= Eb * yo;
        const T ttb = Eb * sxy;
        idb += ttb * kinv * ipt;
        kinvbar += ttb * id * ipt;
        iptb += ttb * id * kinv;
        // dDdphi
        kbar += dDdphib * F * o;
        ob += dDdphib * k * F;
        const T Fb = dDdphib * k * o;
        xob += Fb * fx;
        yob -= Fb * fy;
        pyb += Fb * (xo * sa + yo);
        pxb += Fb * xo * (ca - T(1));
        sab_i += Fb * xo * py;
        cab_i += Fb * xo * px;
        a2b -= Fb * yo;
        // a1 = px ca - py sa, a2 = py ca + px sa
        pxb += a1b * ca + a2b * sa;
        pyb += a2b * ca - a1b * sa;
        cab_i += a1b * px + a2b * py;
        sab_i += a2b * px - a1b * py;
        r0b -= ob * o * o;
      }
    }
    const T ab = sincos4_bar(a, sab_i, cab_i);
    idb += ab * ipt * kinv;
    iptb += ab * id * kinv;
    kinvbar += ab * id * ipt;
    rbar += idb;
    r0b -= idb;
    xob += r0b * xo * ir0;
    yob += r0b * yo * ir0;
  }
  // ---- initial values: dDdx0 = -x/r00, dDdy0 = -y/r00 (r00 > 0), px0 = cP pt, py0 = sP pt
  if (t.r00 > T(0)) {
    const T ir00 = T(1) / t.r00;
    const T r00b = (dDdxb * x + dDdyb * y) * ir00 * ir00;
    xob += (r00b * x - dDdxb) * ir00;
    yob += (r00b * y - dDdyb) * ir00;
  }
  cPb += pxb * pt;
  sPb += pyb * pt;
  ptb += pxb * cP + pyb * sP;
  phib += -cPb * sP + sPb * cP;
  iptb -= ptb * pt * pt;
  pb_in[0] = xob;
  pb_in[1] = yob;
  pb_in[2] = zb;
  pb_in[3] = iptb;
  pb_in[4] = phib;
  pb_in[5] = thetab;
}

// KalmanUpdate of (p, c) with hit (hp, hc): the reference's formulas (TBB:433-642) with the two
// quotients by 2 rh taken as one reciprocal and the rows of H*C (u = R00 C_m0 + R01 C_m1, v = C_m2)
// formed once for the gain and for C - K*(H*C), as the FP32 forward does; returns chi2. The
// determinant is taken in double (TBB:457).
template <class T>
P2R_HD T upd_fwd(T (&p)[6], T (&c)[21], const T (&hp)[3], const T (&hc)[6]) {
  P2R_PREC_REGION(upd);
  const T rh = hipo(hp[0], hp[1]);
  const T ih = T(0.5f) / rh;
  const T R00 = -(hp[1] + p[1]) * ih;
  const T R01 = (hp[0] + p[0]) * ih;
  const T e0 = (R00 * (c[0] + hc[0]) + R01 * (c[1] + hc[1])) * R00 + (R00 * (c[1] + hc[1]) + R01 * (c[2] + hc[2])) * R01;
  const T e1 = (c[3] + hc[3]) * R00 + (c[4] + hc[4]) * R01;
  const T e2 = c[5] + hc[5];
  const double det = (double)e0 * e2 - (double)e1 * e1;
  const T s = T(1.0 / det);
  const T i0 = s * e2, i1 = e1 * -s, i2 = s * e0;
  T u[6], v[6], K0[6], K1[6];
P2R_UNROLL
  for (int m = 0; m < 6; ++m) {
    u[m] = R00 * c[S6(m, 0)] + R01 * c[S6(m, 1)];
    v[m] = c[S6(m, 2)];
    K0[m] = u[m] * i0 + v[m] * i1;
    K1[m] = u[m] * i1 + v[m] * i2;
  }
  const T res0 = R00 * (hp[0] - p[0]) + R01 * (hp[1] - p[1]);
  const T res1 = hp[2] - p[2];
  const T chi2 = i0 * res0 * res0 + T(2) * i1 * res0 * res1 + i2 * res1 * res1;
P2R_UNROLL
  for (int m = 0; m < 6; ++m) p[m] = p[m] + K0[m] * res0 + K1[m] * res1;
P2R_UNROLL
  for (int i = 0; i < 6; ++i)
P2R_UNROLL
    for (int j = 0; j <= i; ++j) c[S6(i, j)] = c[S6(i, j)] - (K0[i] * u[j] + K1[i] * v[j]);
  return chi2;
}

// Reverse of upd_fwd at the input (p, c, hp, hc). pb / cb: in = adjoints of the updated
// state, out = adjoints of the state before the update (overwritten in place).
// chi2b: adjoint of the update's chi2. hpb / hcb: adjoints of the hit (overwritten).
template <class T>
P2R_HD void upd_rev(const T (&p)[6], const T (&c)[21], const T (&hp)[3], const T (&hc)[6], T (&pb)[6], T (&cb)[21],
                    T chi2b, T (&hpb)[3], T (&hcb)[6]) {
  P2R_PREC_REGION(updrec);
  const T rh = hipo(hp[0], hp[1]);
  const T den = T(2) * rh;
  const T iden = T(1) / den;  // one reciprocal for every quotient by den (and by rh = den / 2)
  const T R00 = -(hp[1] + p[1]) * iden, R01 = (hp[0] + p[0]) * iden;
  T A[6];
P2R_UNROLL
  for (int k = 0; k < 6; ++k) A[k] = c[k] + hc[k];
  const T e0 = R00 * R00 * A[0] + T(2) * R00 * R01 * A[1] + R01 * R01 * A[2];
  const T e1 = A[3] * R00 + A[4] * R01, e2 = A[5];
  const T s = T(1) / (e0 * e2 - e1 * e1);
  const T i0 = s * e2, i1 = -s * e1, i2 = s * e0;
  T B0[6], B1[6], K0[6], K1[6];
P2R_UNROLL
  for (int m = 0; m < 6; ++m) {
    B0[m] = R00 * c[S6(m, 0)] + R01 * c[S6(m, 1)];
    B1[m] = c[S6(m, 2)];
    K0[m] = B0[m] * i0 + B1[m] * i1;
    K1[m] = B0[m] * i1 + B1[m] * i2;
  }
  const T res0 = R00 * (hp[0] - p[0]) + R01 * (hp[1] - p[1]), res1 = hp[2] - p[2];

  P2R_PREC_REGION(updrev);
  // C' = C - K0 B0^T - K1 B1^T (lower triangle); p' = p + K0 res0 + K1 res1
  T K0b[6], K1b[6], B0b[6], B1b[6];
P2R_UNROLL
  for (int m = 0; m < 6; ++m) {
    T a0 = 0, a1 = 0, b0 = 0, b1 = 0;
P2R_UNROLL
    for (int j = 0; j <= m; ++j) {
      a0 += cb[S6(m, j)] * B0[j];
      a1 += cb[S6(m, j)] * B1[j];
    }
P2R_UNROLL
    for (int i = m; i < 6; ++i) {
      b0 += cb[S6(i, m)] * K0[i];
      b1 += cb[S6(i, m)] * K1[i];
    }
    K0b[m] = -a0 + pb[m] * res0;
    K1b[m] = -a1 + pb[m] * res1;
    B0b[m] = -b0;
    B1b[m] = -b1;
  }
  T res0b = 0, res1b = 0;
P2R_UNROLL
  for (int m = 0; m < 6; ++m) {
    res0b += pb[m] * K0[m];
    res1b += pb[m] * K1[m];
  }
  // chi2 = i0 res0^2 + 2 i1 res0 res1 + i2 res1^2
  T i0b = chi2b * res0 * res0, i1b = chi2b * T(2) * res0 * res1, i2b = chi2b * res1 * res1;
  res0b += chi2b * (T(2) * i0 * res0 + T(2) * i1 * res1);
  res1b += chi2b * (T(2) * i1 * res0 + T(2) * i2 * res1);
  // K0 = B0 i0 + B1 i1, K1 = B0 i1 + B1 i2
P2R_UNROLL
  for (int m = 0; m < 6; ++m) {
    i0b += K0b[m] * B0[m];
    i1b += K0b[m] * B1[m] + K1b[m] * B0[m];
    i2b += K1b[m] * B1[m];
    B0b[m] += K0b[m] * i0 + K1b[m] * i1;
    B1b[m] += K0b[m] * i1 + K1b[m] * i2;
  }
  // B0_m = R00 C_m0 + R01 C_m1, B1_m = C_m2 (cb keeps the direct C' = C ... path)
  T R00b = 0, R01b = 0;
P2R_UNROLL
  for (int m = 0; m < 6; ++m) {
    R00b += B0b[m] * c[S6(m, 0)];
    R01b += B0b[m] * c[S6(m, 1)];
    cb[S6(m, 0)] += B0b[m] * R00;
    cb[S6(m, 1)] += B0b[m] * R01;
    cb[S6(m, 2)] += B1b[m];
  }
  // (i0, i1, i2) = (e2, -e1, e0) / det
  T e2b = i0b * s, e1b = -i1b * s, e0b = i2b * s;
  const T sb = i0b * e2 - i1b * e1 + i2b * e0;
  const T detb = -sb * s * s;
  e0b += detb * e2;
  e2b += detb * e0;
  e1b -= T(2) * detb * e1;
  // residual
  R00b += res0b * (hp[0] - p[0]);
  R01b += res0b * (hp[1] - p[1]);
  hpb[0] = res0b * R00;
  hpb[1] = res0b * R01;
  hpb[2] = res1b;
  pb[0] -= res0b * R00;
  pb[1] -= res0b * R01;
  pb[2] -= res1b;
  // e0 = R00^2 A0 + 2 R00 R01 A1 + R01^2 A2, e1 = A3 R00 + A4 R01, e2 = A5
  R00b += e0b * (T(2) * R00 * A[0] + T(2) * R01 * A[1]) + e1b * A[3];
  R01b += e0b * (T(2) * R00 * A[1] + T(2) * R01 * A[2]) + e1b * A[4];
  hcb[0] = e0b * R00 * R00;
  hcb[1] = e0b * T(2) * R00 * R01;
  hcb[2] = e0b * R01 * R01;
  hcb[3] = e1b * R00;
  hcb[4] = e1b * R01;
  hcb[5] = e2b;
P2R_UNROLL
  for (int k = 0; k < 6; ++k) cb[k] += hcb[k];
  // R00 = -(hy + y)/den, R01 = (hx + x)/den, den = 2 hipo(hx, hy)
  hpb[1] -= R00b * iden;
  pb[1] -= R00b * iden;
  hpb[0] += R01b * iden;
  pb[0] += R01b * iden;
  const T rhb = T(2) * (-(R00b * R00 + R01b * R01) * iden);
  if (rh > T(0)) {
    const T irh = T(2) * iden;
    hpb[0] += rhb * hp[0] * irh;
    hpb[1] += rhb * hp[1] * irh;
  }
}

// One full layer, forward (state in place; returns chi2): propagate to hipo(hp) + dr, update.
template <class T>
P2R_HD T layer_fwd(T (&p)[6], T (&c)[21], T k, T kinv, const T (&hp)[3], const T (&hc)[6], T dr) {
  PropTape<T> t;
  const T r = hipo(hp[0], hp[1]) + dr;
  prop_fwd(p, c, k, kinv, r, t, p, c);
  return upd_fwd(p, c, hp, hc);
}

// Reverse of layer_fwd at the state (p, c) BEFORE the layer. pb / cb: in = adjoints of the
// state after the layer, out = adjoints of the state before it. chi2b: adjoint of this
// layer's chi2. hpb / hcb (overwritten), drb, kbar, kinvbar (accumulated).
template <class T>
P2R_HD void layer_rev(const T (&p)[6], const T (&c)[21], T k, T kinv, const T (&hp)[3], const T (&hc)[6], T dr,
                      T (&pb)[6], T (&cb)[21], T chi2b, T (&hpb)[3], T (&hcb)[6], T& drb, T& kbar, T& kinvbar) {
  PropTape<T> t;
  const T rh = hipo(hp[0], hp[1]);
  const T r = rh + dr;
  T pp[6], pc[21];
  prop_fwd(p, c, k, kinv, r, t, pp, pc);
  upd_rev(pp, pc, hp, hc, pb, cb, chi2b, hpb, hcb);
  T pin[6], cin[21], rbar = 0;
  prop_rev(t, p, c, k, kinv, r, pb, cb, pin, cin, rbar, kbar, kinvbar);
P2R_UNROLL
  for (int i = 0; i < 6; ++i) pb[i] = pin[i];
P2R_UNROLL
  for (int i = 0; i < 21; ++i) cb[i] = cin[i];
  drb += rbar;
  if (rh > T(0)) {
    const T irh = T(1) / rh;
    hpb[0] += rbar * hp[0] * irh;
    hpb[1] += rbar * hp[1] * irh;
  }
}

}  // namespace adj
}  // namespace p2r
