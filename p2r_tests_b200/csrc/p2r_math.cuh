// Per-track device arithmetic of the p2r hot path, with the whole track state in registers.
//
// Reference: src/propagate-tor-test_tbb.cpp (cerati/p2r-tests), "TBB" below.
//   sincos4          TBB:644-652
//   propagateToR     TBB:656-812 (transport Jacobian TBB:753-807; J*C TBB:296-341;
//                    (J*C)*J^T TBB:343-373)
//   KalmanUpdate     TBB:433-642
// The reference evaluates these per Matriplex block with one SIMD loop per stage and
// materialises the 6x6 Jacobian, J*C and K*H*C in memory. Here one thread owns one track: the
// 6 parameters and 21 covariance elements stay in registers across layers, the Jacobian is a
// set of scalars (its unit rows 3 and 5 and its structural zeros are never formed, and rows 2
// and 4, which share the factors dadx, dady, dadphi, are applied through one shared
// combination), and J*C, (J*C)*J^T and C - K*(H*C) are expanded at compile time over the
// non-zero terms.
//
// Every multiply, add and fused multiply-add is written out (fmul / fadd / fsub / ffma, all
// round-to-nearest, never re-associated or contracted by the compiler), so every kernel that
// uses these functions (fused, per-layer, persistent queue, any launch shape) produces
// bit-identical results. Where the reference's expression has a common factor that does not
// change along the helix iterations (ipt/k, k*pt, k*pt/sin(theta)) it is formed once; that
// and the fused forms change results only at the rounding level, checked against the
// reference by the parity tests.
#pragma once
#include <cuda_runtime.h>

namespace p2r {

// packed lower-triangle index of a symmetric 6x6 (TBB:46-54)
__host__ __device__ constexpr int S6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }  // a*b + c

// ---------------------------------------------------------------- division and square root
// Three builds:
//  default            the hardware approximations (rcp.approx, rsqrt.approx) refined by one
//                     Newton-Raphson step each (the textbook iteration, e.g. Markstein,
//                     IBM J. Res. Dev. 34(1), 1990): y <- y + y (1 - b y) for 1/b, a/b = a y;
//                     for sqrt(x), r ~ 1/sqrt(x), s = x r, s <- s + (r/2)(x - s s). Within
//                     about an ulp of the rounded quotient / root (p2r_math_check measures it),
//                     without the special-case paths of a correctly rounded sequence: the
//                     arguments here are finite and normal and, for sqrt, positive
//  P2R_IEEE_MATH      IEEE-rounded (a / b, sqrtf)
//  P2R_FAST_MATH      the approximations alone (div.approx / sqrt.approx, about 2 ulp)
// Every other operation is the same in all three.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
#if defined(P2R_FAST_MATH)
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float fsqrt(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
#elif !defined(P2R_IEEE_MATH)
#define P2R_REFINED_MATH 1
__device__ __forceinline__ float frcp(float b) {
  const float y = rcp_approx(b);
  return ffma(y, ffma(-b, y, 1.f), y);
}
__device__ __forceinline__ float fdiv(float a, float b) { return fmul(a, frcp(b)); }
// For x >= 0 (the path takes square roots of sums of squares only): x = 0 is lifted to the
// smallest normal float for the reciprocal square root, so sqrt(+-0) = +-0 without a branch.
__device__ __forceinline__ float fsqrt(float x) {
  const float r = rsqrt_approx(fmaxf(x, 1.17549435e-38f));
  const float s = fmul(x, r);
  return ffma(fmul(0.5f, r), ffma(-s, s, x), s);
}
#else
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float x) { return __fsqrt_rn(x); }
#endif

// sqrt(x^2 + y^2)
__device__ __forceinline__ float hipo(float x, float y) { return fsqrt(ffma(x, x, fmul(y, y))); }

// The inverse of the symmetric 2x2 [[e0, e1], [e1, e2]] with the determinant, its reciprocal
// and the three products in double, each entry rounded to float once (TBB:457-463 takes the
// determinant and its reciprocal in double). Rounding 1/det to float before the products, as
// the reference writes it, adds one rounding to every entry; measured on the CPU restatement of
// the chained filter, the single rounding lowers the fraction of covariance elements off FP64 by
// more than 1e-3 from 3.7 % to 3.1 % (the reference: 3.3 %) and the 99th percentile by 12 %.
__device__ __forceinline__ void inverse2_fp64(float e0, float e1, float e2, float& i0, float& i1, float& i2) {
  const double d0 = (double)e0, d1 = (double)e1, d2 = (double)e2;
  const double r = __drcp_rn(__dsub_rn(__dmul_rn(d0, d2), __dmul_rn(d1, d1)));
  i0 = (float)__dmul_rn(r, d2);
  i1 = (float)__dmul_rn(-r, d1);
  i2 = (float)__dmul_rn(r, d0);
}

// 4th-order cos / 3rd-order sin for the small per-step turning angles (TBB:644-652), as
// s and omc = 1 - cos = x^2/2 - x^4/24. Products with cos are formed as v - v*omc: the same
// polynomial without rounding 1 - omc first, and without forming 1 - (1 - ...) in float,
// which cancels for the sub-milliradian angles of the later helix iterations (the
// reference's -ffast-math build simplifies 1 - cosa to this form as well; evaluated as
// written, the chained filter loses about a factor 2.5 in accuracy on 1/pT).
__device__ __forceinline__ void sincos4(float x, float& s, float& omc) {
  const float x2 = fmul(x, x);
  omc = fmul(x2, ffma(-0.04166667f, x2, 0.5f));
  s = ffma(fmul(-0.16666667f, x), x2, x);
}
__device__ __forceinline__ float mulcos(float v, float omc) { return ffma(-v, omc, v); }  // v*cos

// ---------------------------------------------------------------- propagateToR
// Propagates (ip, ic) to the cylinder of radius r. k = q*kfact, kinv = 1/k.
// op/oc may be the same arrays as ip/ic: every input is read before any output is written.
__device__ __forceinline__ void propagate_to_r(const float (&ip)[6], const float (&ic)[21], float k, float kinv,
                                               float r, float (&op)[6], float (&oc)[21]) {
  const float xin = ip[0], yin = ip[1], zin = ip[2];
  const float iptin = ip[3], phiin = ip[4], thetain = ip[5];
  float r0 = hipo(xin, yin);
  const float pt = fdiv(1.f, iptin);
  const float ik = fmul(iptin, kinv);  // turning angle per unit of path length
  const float kpt = fmul(k, pt);

  float sinP, cosP;
  sincosf(phiin, &sinP, &cosP);  // phi can be large: no approximation (TBB:688-689)
  float pxin = fmul(cosP, pt);
  float pyin = fmul(sinP, pt);
  float dDdx = r0 > 0.f ? -fdiv(xin, r0) : 0.f;
  float dDdy = r0 > 0.f ? -fdiv(yin, r0) : 0.f;
  float D = 0.f, dDdipt = 0.f, dDdphi = 0.f;
  float sina, omc;
  float xo = xin, yo = yin;

#pragma unroll
  for (int i = 0; i < 5; ++i) {  // 5 fixed iterations (TBB:655, TBB:701)
    r0 = hipo(xo, yo);
    const float id = fsub(r, r0);
    D = fadd(D, id);
    sincos4(fmul(id, ik), sina, omc);
    // momentum direction after the step: (px ca - py sa, py ca + px sa)
    const float pxca = mulcos(pxin, omc), pyca = mulcos(pyin, omc);
    const float a1 = ffma(-pyin, sina, pxca);
    const float a2 = ffma(pxin, sina, pyca);
    // Path derivatives, only once the step is below 1 um (TBB:714). The reference scales every
    // derivative increment by oor0 = 0 until then; adding a finite x * 0 leaves the sums
    // unchanged, so those increments are skipped.
    if (i + 1 != 5 && r0 > 0.f && fabsf(id) < 0.0001f) {
      const float noor0 = -fdiv(1.f, r0);  // -1/r0
      const float kn = fmul(iptin, noor0);  // k*dadx/xo = k*dady/yo of TBB:716-717
      // dDdx -= (xo*(1 + tx*a1) + yo*tx*a2) * oor0 and dDdy -= (xo*ty*a1 + yo*(1 + ty*a2)) * oor0
      // with tx = kn*xo, ty = kn*yo: xo resp. yo times (1 + kn*(xo*a1 + yo*a2)) * oor0
      const float g = fmul(ffma(kn, ffma(xo, a1, fmul(yo, a2)), 1.f), noor0);
      dDdx = ffma(xo, g, dDdx);
      dDdy = ffma(yo, g, dDdy);
      // dDdipt -= k*(xo*e1 + yo*e2)*pt*oor0 with t = dadipt*ipt,
      //   e1 = pxca*t - pysa*t - pyca - pxsa + pyin = a1*t + (pyin - a2)
      //   e2 = pyca*t + pxsa*t - pysa + pxca - pxin = a2*t + (a1 - pxin)
      const float t = fmul(id, ik);
      const float u = fsub(pyin, a2);
      const float e1 = ffma(a1, t, u);
      const float e2 = ffma(a2, t, fsub(a1, pxin));
      dDdipt = ffma(ffma(xo, e1, fmul(yo, e2)), fmul(kpt, noor0), dDdipt);
      // dDdphi += k*(xo*(pysa - pxin + pxca) - yo*(pxsa - pyin + pyca)) * oor0
      //         = k*(xo*f1 + yo*u) * oor0,  f1 = pyin*sina + pxca - pxin
      const float f1 = fsub(ffma(pyin, sina, pxca), pxin);
      dDdphi = ffma(ffma(yo, u, fmul(xo, f1)), fmul(-k, noor0), dDdphi);
    }
    xo = ffma(k, ffma(pxin, sina, fmul(-pyin, omc)), xo);  // xo + k*(pxin*sina - pyin*omc)
    yo = ffma(k, ffma(pyin, sina, fmul(pxin, omc)), yo);   // yo + k*(pyin*sina + pxin*omc)
    pxin = a1;
    pyin = a2;
  }

  const float alpha = fmul(D, ik);
  const float dadx = fmul(dDdx, ik);
  const float dady = fmul(dDdy, ik);
  const float dadipt = fmul(ffma(iptin, dDdipt, D), kinv);
  const float dadphi = fmul(dDdphi, ik);
  sincos4(alpha, sina, omc);

  // Non-trivial Jacobian entries (TBB:753-807); J22 = J33 = J55 = 1, the rest of rows
  // 3 and 5 and J02 J05 J12 J15 J42 J45 are 0. cP*ca - cP and sP*ca - sP are formed as
  // -cP*omc and -sP*omc (the same polynomial, without the cancellation).
  const float cc = ffma(-sinP, sina, mulcos(cosP, omc));  // cos(phi + alpha)
  const float sc = ffma(cosP, sina, mulcos(sinP, omc));   // sin(phi + alpha)
  const float kxp = fmul(kpt, dadx), kyp = fmul(kpt, dady);
  const float J00 = ffma(kxp, cc, 1.f);  // 1 + k*dadx*cc*pt
  const float J01 = fmul(kyp, cc);
  const float J10 = fmul(kxp, sc);
  const float J11 = ffma(kyp, sc, 1.f);
  const float ia = fmul(iptin, dadipt);
  const float u1 = fsub(mulcos(ia, omc), sina);  // ipt*dadipt*cosa - sina
  const float u2 = ffma(-ia, sina, omc);   // omc - ipt*dadipt*sina
  const float kpt2 = fmul(kpt, pt);
  const float J03 = fmul(ffma(cosP, u1, fmul(sinP, u2)), kpt2);   // k*(cP*u1 + sP*u2)*pt^2
  const float J13 = fmul(ffma(sinP, u1, fmul(-cosP, u2)), kpt2);  // k*(sP*u1 - cP*u2)*pt^2
  // k*(cP*dadphi*ca - sP*dadphi*sa - sP*sa + cP*ca - cP)*pt
  const float J04 = fmul(ffma(dadphi, cc, -ffma(sinP, sina, fmul(cosP, omc))), kpt);
  // k*(sP*dadphi*ca + cP*dadphi*sa + sP*ca + cP*sa - sP)*pt
  const float J14 = fmul(ffma(dadphi, sc, ffma(cosP, sina, fmul(-sinP, omc))), kpt);
  float sinT, cosT;
  sincosf(thetain, &sinT, &cosT);  // theta can be large: no approximation (TBB:767-769)
  const float isinT = fdiv(1.f, sinT);
  const float kpi = fmul(kpt, isinT);  // k*pt/sinT
  const float kpc = fmul(kpi, cosT);   // k*pt*cosT/sinT
  // rows 2 and 4 share (dadx, dady, ., ., dadphi, .): J2 = kpc*(dadx, dady, 0, 0, dadphi, 0)
  // + (0, 0, 1, J23, 0, J25) and J4 = (dadx, dady, 0, dadipt, 1 + dadphi, 0), so for a vector v
  // with n = dadx*v0 + dady*v1 + dadphi*v4: v.J2 = kpc*n + v2 + J23*v3 + J25*v5 and
  // v.J4 = n + dadipt*v3 + v4
  const float J23 = fmul(fmul(fsub(ia, alpha), kpc), pt);
  const float J25 = fmul(fmul(-alpha, kpi), isinT);  // -k*alpha*pt/sinT^2
  auto nvec = [&](float v0, float v1, float v4) { return ffma(dadphi, v4, ffma(dady, v1, fmul(dadx, v0))); };
  auto dotJ2 = [&](float n, float v2, float v3, float v5) { return ffma(kpc, n, ffma(J25, v5, ffma(J23, v3, v2))); };
  auto dotJ4 = [&](float n, float v3, float v4) { return fadd(ffma(dadipt, v3, n), v4); };

  // T = J*C (TBB:296-341): rows 3 and 5 of T are rows 3 and 5 of C.
  float T0[6], T1[6], T2[6], T4[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const float c0 = ic[S6(0, j)], c1 = ic[S6(1, j)], c2 = ic[S6(2, j)];
    const float c3 = ic[S6(3, j)], c4 = ic[S6(4, j)], c5 = ic[S6(5, j)];
    T0[j] = ffma(J04, c4, ffma(J03, c3, ffma(J01, c1, fmul(J00, c0))));
    T1[j] = ffma(J14, c4, ffma(J13, c3, ffma(J11, c1, fmul(J10, c0))));
    const float n = nvec(c0, c1, c4);
    T2[j] = dotJ2(n, c2, c3, c5);
    T4[j] = dotJ4(n, c3, c4);
  }
  float T3[6], T5[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    T3[j] = ic[S6(3, j)];
    T5[j] = ic[S6(5, j)];
  }

  // C' = T*J^T, lower triangle (TBB:343-373).
  float nc[21];
#define P2R_ROW(i, Ti)                                                                                \
  {                                                                                                   \
    nc[S6(i, 0)] = ffma(Ti[4], J04, ffma(Ti[3], J03, ffma(Ti[1], J01, fmul(Ti[0], J00))));             \
    if (i >= 1) nc[S6(i, 1)] = ffma(Ti[4], J14, ffma(Ti[3], J13, ffma(Ti[1], J11, fmul(Ti[0], J10)))); \
    if (i >= 2) {                                                                                     \
      const float n = nvec(Ti[0], Ti[1], Ti[4]);                                                      \
      nc[S6(i, 2)] = dotJ2(n, Ti[2], Ti[3], Ti[5]);                                                   \
      if (i >= 4) nc[S6(i, 4)] = dotJ4(n, Ti[3], Ti[4]);                                              \
    }                                                                                                 \
    if (i >= 3) nc[S6(i, 3)] = Ti[3];                                                                 \
    if (i >= 5) nc[S6(i, 5)] = Ti[5];                                                                 \
  }
  P2R_ROW(0, T0)
  P2R_ROW(1, T1)
  P2R_ROW(2, T2)
  P2R_ROW(3, T3)
  P2R_ROW(4, T4)
  P2R_ROW(5, T5)
#undef P2R_ROW

  op[0] = xo;
  op[1] = yo;
  op[2] = ffma(alpha, kpc, zin);  // z + k*alpha*cosT*pt/sinT
  op[3] = iptin;
  op[4] = fadd(phiin, alpha);
  op[5] = thetain;
#pragma unroll
  for (int i = 0; i < 21; ++i) oc[i] = nc[i];
}

// ---------------------------------------------------------------- KalmanUpdate
// Kalman update of (p, c) with a hit at hp (covariance hc), in place (TBB:433-642).
// rhit = hipo(hp[0], hp[1]). Returns the update's chi2 = res^T inv(R) res when kChi2.
// kFp64Det: the 2x2 determinant and its reciprocal in double, as TBB:457-458 takes them.
// H = [[rotT00, rotT01, 0, 0, 0, 0], [0, 0, 1, 0, 0, 0]] projects onto the hit's (r-phi, z)
// plane; H*C is formed once (row 0: u, row 1: row 2 of C) and serves both the gain
// K = C*H^T*inv(R) and the update C - K*(H*C).
template <bool kFp64Det, bool kChi2>
__device__ __forceinline__ float kalman_update(float (&p)[6], float (&c)[21], const float (&hp)[3],
                                               const float (&hc)[6], float rhit) {
  // rotT00 = -(hp1 + p1)/(2 rhit), rotT01 = (hp0 + p0)/(2 rhit)
  const float inv2r = fdiv(0.5f, rhit);
  const float rotT00 = fmul(fadd(hp[1], p[1]), -inv2r);
  const float rotT01 = fmul(fadd(hp[0], p[0]), inv2r);

  const float s0 = fadd(c[0], hc[0]), s1 = fadd(c[1], hc[1]), s2 = fadd(c[2], hc[2]);
  const float e0 = ffma(ffma(rotT01, s2, fmul(rotT00, s1)), rotT01, fmul(ffma(rotT01, s1, fmul(rotT00, s0)), rotT00));
  const float e1 = ffma(fadd(c[4], hc[4]), rotT01, fmul(fadd(c[3], hc[3]), rotT00));
  const float e2 = fadd(c[5], hc[5]);
  // The determinant is kept in double in every build: the chained filter's accuracy follows
  // the precision of s closely (an extra 0.5 ulp of random error in s alone raises the
  // 99th-percentile covariance error by ~40 %, 2 ulp by ~4x; the other divisions and square
  // roots are insensitive at 2 ulp).
  float i0, i1, i2;
  if (kFp64Det) {
    inverse2_fp64(e0, e1, e2, i0, i1, i2);
  } else {
    const float s = fdiv(1.f, ffma(e0, e2, fmul(-e1, e1)));
    i0 = fmul(s, e2);
    i1 = fmul(-e1, s);
    i2 = fmul(s, e0);
  }

  float u[6], v[6];  // rows of H*C
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    u[j] = ffma(rotT01, c[S6(1, j)], fmul(rotT00, c[S6(0, j)]));
    v[j] = c[S6(2, j)];
  }
  float K0[6], K1[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    K0[m] = ffma(v[m], i1, fmul(u[m], i0));
    K1[m] = ffma(v[m], i2, fmul(u[m], i1));
  }
  const float res0 = ffma(rotT01, fsub(hp[1], p[1]), fmul(rotT00, fsub(hp[0], p[0])));
  const float res1 = fsub(hp[2], p[2]);
  float chi2 = 0.f;
  if (kChi2) chi2 = ffma(fmul(i2, res1), res1, ffma(fmul(fmul(2.f, i1), res0), res1, fmul(fmul(i0, res0), res0)));
#pragma unroll
  for (int m = 0; m < 6; ++m) p[m] = ffma(K1[m], res1, ffma(K0[m], res0, p[m]));

  // C' = C - K*(H*C), lower triangle (u and v hold the pre-update rows)
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) c[S6(i, j)] = ffma(-K1[i], v[j], ffma(-K0[i], u[j], c[S6(i, j)]));
  return chi2;
}

// phi wrapped into [-pi, pi]: the update step the reference leaves commented out
// (squashPhiMPlex, TBB:635, "ensure phi is between |pi|"; the function itself is not in the
// reference). phi - 2 pi n with n the nearest integer to phi / (2 pi), in one rounding.
__device__ __forceinline__ float squash_phi(float phi) {
  const float n = rintf(fmul(phi, 0.159154943f));
  return ffma(-n, 6.28318531f, phi);
}

}  // namespace p2r
