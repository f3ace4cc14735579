// Per-track device arithmetic of the p2r hot path, with the whole track state in registers.
//
// Reference: src/propagate-tor-test_tbb.cpp (cerati/p2r-tests), "TBB" below.
//   sincos4          TBB:644-652
//   propagateToR     TBB:656-812 (transport Jacobian TBB:753-807; J*C TBB:296-341;
//                    (J*C)*J^T TBB:343-373)
//   KalmanUpdate     TBB:433-642
// The reference evaluates these per Matriplex block with one SIMD loop per stage and
// materialises the 6x6 Jacobian and J*C in memory. Here one thread owns one track: the
// 6 parameters and 21 covariance elements stay in registers across layers, the Jacobian
// is a set of 17 scalars (its unit rows 3 and 5 and its structural zeros are never
// formed), and J*C and (J*C)*J^T are expanded at compile time over the non-zero terms,
// in the reference's summation order.
#pragma once
#include <cuda_runtime.h>

namespace p2r {

// packed lower-triangle index of a symmetric 6x6 (TBB:46-54)
__host__ __device__ constexpr int S6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// Division and square root, three builds:
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
  return fmaf(y, fmaf(-b, y, 1.f), y);
}
__device__ __forceinline__ float fdiv(float a, float b) { return a * frcp(b); }
__device__ __forceinline__ float fsqrt(float x) {
  if (!(x > 0.f)) return sqrtf(x);
  const float r = rsqrt_approx(x);
  const float s = x * r;
  return fmaf(0.5f * r, fmaf(-s, s, x), s);
}
#else
__device__ __forceinline__ float fdiv(float a, float b) { return a / b; }
__device__ __forceinline__ float fsqrt(float x) { return sqrtf(x); }
#endif

__device__ __forceinline__ float hipo(float x, float y) { return fsqrt(x * x + y * y); }

// 4th-order cos / 3rd-order sin for the small per-step turning angles (TBB:644-652).
// omc = 1 - c, evaluated as x^2/2 - x^4/24: the same polynomial without forming 1 - (1 - ...)
// in float, which cancels for the sub-milliradian angles of the later helix iterations (the
// reference's -ffast-math build simplifies 1 - cosa to this form as well; evaluated as
// written, the chained filter loses about a factor 2.5 in accuracy on 1/pT).
__device__ __forceinline__ void sincos4(float x, float& s, float& c, float& omc) {
  const float x2 = x * x;
  omc = 0.5f * x2 - 0.04166667f * x2 * x2;
  c = 1.f - omc;
  s = x - 0.16666667f * x * x2;
}

// Propagates (ip, ic) to the cylinder of radius r. k = q*kfact, kinv = 1/k.
// op/oc may be the same arrays as ip/ic: every input is read before any output is written.
__device__ __forceinline__ void propagate_to_r(const float (&ip)[6], const float (&ic)[21], float k, float kinv,
                                               float r, float (&op)[6], float (&oc)[21]) {
  const float xin = ip[0], yin = ip[1], zin = ip[2];
  const float iptin = ip[3], phiin = ip[4], thetain = ip[5];
  float r0 = hipo(xin, yin);
  const float pt = fdiv(1.f, iptin);

  float D = 0.f, cosa = 0.f, sina = 0.f, omc = 0.f;
  float sinP, cosP;
  sincosf(phiin, &sinP, &cosP);  // phi can be large: no approximation (TBB:688-689)
  float pxin = cosP * pt;
  float pyin = sinP * pt;
  float dDdx = r0 > 0.f ? -fdiv(xin, r0) : 0.f;
  float dDdy = r0 > 0.f ? -fdiv(yin, r0) : 0.f;
  float dDdipt = 0.f, dDdphi = 0.f;
  float xo = xin, yo = yin;

#pragma unroll
  for (int i = 0; i < 5; ++i) {  // 5 fixed iterations (TBB:655, TBB:701)
    r0 = hipo(xo, yo);
    const float id = r - r0;
    D += id;
    sincos4(id * iptin * kinv, sina, cosa, omc);
    if (i + 1 != 5) {
      // path derivatives, only once the step is below 1 um (TBB:714)
      const float oor0 = (r0 > 0.f && fabsf(r - r0) < 0.0001f) ? fdiv(1.f, r0) : 0.f;
      const float dadipt = id * kinv;
      const float dadx = -xo * iptin * kinv * oor0;
      const float dady = -yo * iptin * kinv * oor0;
      const float pxca = pxin * cosa;
      const float pxsa = pxin * sina;
      const float pyca = pyin * cosa;
      const float pysa = pyin * sina;
      float tmp = k * dadx;
      dDdx -= (xo * (1.f + tmp * (pxca - pysa)) + yo * tmp * (pyca + pxsa)) * oor0;
      tmp = k * dady;
      dDdy -= (xo * tmp * (pxca - pysa) + yo * (1.f + tmp * (pyca + pxsa))) * oor0;
      tmp = dadipt * iptin;
      dDdipt -= k * (xo * (pxca * tmp - pysa * tmp - pyca - pxsa + pyin) +
                     yo * (pyca * tmp + pxsa * tmp - pysa + pxca - pxin)) * pt * oor0;
      dDdphi += k * (xo * (pysa - pxin + pxca) - yo * (pxsa - pyin + pyca)) * oor0;
    }
    xo = xo + k * (pxin * sina - pyin * omc);
    yo = yo + k * (pyin * sina + pxin * omc);
    const float pxold = pxin;
    pxin = pxin * cosa - pyin * sina;
    pyin = pyin * cosa + pxold * sina;
  }

  const float alpha = D * iptin * kinv;
  const float dadx = dDdx * iptin * kinv;
  const float dady = dDdy * iptin * kinv;
  const float dadipt = (iptin * dDdipt + D) * kinv;
  const float dadphi = dDdphi * iptin * kinv;
  sincos4(alpha, sina, cosa, omc);

  // non-trivial Jacobian entries (TBB:753-807); J22 = J33 = J55 = 1, the rest of rows
  // 3 and 5 and J02 J05 J12 J15 J42 J45 are 0.
  const float J00 = 1.f + k * dadx * (cosP * cosa - sinP * sina) * pt;
  const float J01 = k * dady * (cosP * cosa - sinP * sina) * pt;
  const float J03 = k * (cosP * (iptin * dadipt * cosa - sina) + sinP * (omc - iptin * dadipt * sina)) * pt * pt;
  const float J04 = k * (cosP * dadphi * cosa - sinP * dadphi * sina - sinP * sina + cosP * cosa - cosP) * pt;
  const float J10 = k * dadx * (sinP * cosa + cosP * sina) * pt;
  const float J11 = 1.f + k * dady * (sinP * cosa + cosP * sina) * pt;
  const float J13 = k * (sinP * (iptin * dadipt * cosa - sina) + cosP * (iptin * dadipt * sina - omc)) * pt * pt;
  const float J14 = k * (sinP * dadphi * cosa + cosP * dadphi * sina + sinP * cosa + cosP * sina - sinP) * pt;
  float sinT, cosT;
  sincosf(thetain, &sinT, &cosT);  // theta can be large: no approximation (TBB:767-769)
  const float isinT = fdiv(1.f, sinT);
  const float J20 = k * cosT * dadx * pt * isinT;
  const float J21 = k * cosT * dady * pt * isinT;
  const float J23 = k * cosT * (iptin * dadipt - alpha) * pt * pt * isinT;
  const float J24 = k * dadphi * cosT * pt * isinT;
  const float J25 = -k * alpha * pt * isinT * isinT;
  const float J40 = dadx, J41 = dady, J43 = dadipt, J44 = 1.f + dadphi;

  // T = J*C (TBB:296-341): rows 3 and 5 of T are rows 3 and 5 of C.
  float T0[6], T1[6], T2[6], T4[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const float c0 = ic[S6(0, j)], c1 = ic[S6(1, j)], c2 = ic[S6(2, j)];
    const float c3 = ic[S6(3, j)], c4 = ic[S6(4, j)], c5 = ic[S6(5, j)];
    T0[j] = J00 * c0 + J01 * c1 + J03 * c3 + J04 * c4;
    T1[j] = J10 * c0 + J11 * c1 + J13 * c3 + J14 * c4;
    T2[j] = J20 * c0 + J21 * c1 + c2 + J23 * c3 + J24 * c4 + J25 * c5;
    T4[j] = J40 * c0 + J41 * c1 + J43 * c3 + J44 * c4;
  }
  float T3[6], T5[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    T3[j] = ic[S6(3, j)];
    T5[j] = ic[S6(5, j)];
  }

  // C' = T*J^T, lower triangle (TBB:343-373).
  float nc[21];
#define P2R_ROW(i, Ti)                                                                        \
  {                                                                                         \
    nc[S6(i, 0)] = Ti[0] * J00 + Ti[1] * J01 + Ti[3] * J03 + Ti[4] * J04;                   \
    if (i >= 1) nc[S6(i, 1)] = Ti[0] * J10 + Ti[1] * J11 + Ti[3] * J13 + Ti[4] * J14;       \
    if (i >= 2) nc[S6(i, 2)] = Ti[0] * J20 + Ti[1] * J21 + Ti[2] + Ti[3] * J23 + Ti[4] * J24 + Ti[5] * J25; \
    if (i >= 3) nc[S6(i, 3)] = Ti[3];                                                       \
    if (i >= 4) nc[S6(i, 4)] = Ti[0] * J40 + Ti[1] * J41 + Ti[3] * J43 + Ti[4] * J44;       \
    if (i >= 5) nc[S6(i, 5)] = Ti[5];                                                       \
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
  op[2] = zin + k * alpha * cosT * pt * isinT;
  op[3] = iptin;
  op[4] = phiin + alpha;
  op[5] = thetain;
#pragma unroll
  for (int i = 0; i < 21; ++i) oc[i] = nc[i];
}

// Kalman update of (p, c) with a hit at hp (covariance hc), in place (TBB:433-642).
// rhit = hipo(hp[0], hp[1]). Returns the update's chi2 = res^T inv(R) res when kChi2.
// kFp64Det: the 2x2 determinant in double, as TBB:457-458 takes it.
template <bool kFp64Det, bool kChi2>
__device__ __forceinline__ float kalman_update(float (&p)[6], float (&c)[21], const float (&hp)[3],
                                               const float (&hc)[6], float rhit) {
#if defined(P2R_FAST_MATH) || defined(P2R_REFINED_MATH)
  const float inv2r = fdiv(0.5f, rhit);
  const float rotT00 = -(hp[1] + p[1]) * inv2r;
  const float rotT01 = (hp[0] + p[0]) * inv2r;
#else
  const float rotT00 = -(hp[1] + p[1]) / (2.f * rhit);
  const float rotT01 = (hp[0] + p[0]) / (2.f * rhit);
#endif

  const float e0 = (rotT00 * (c[0] + hc[0]) + rotT01 * (c[1] + hc[1])) * rotT00 +
                   (rotT00 * (c[1] + hc[1]) + rotT01 * (c[2] + hc[2])) * rotT01;
  const float e1 = (c[3] + hc[3]) * rotT00 + (c[4] + hc[4]) * rotT01;
  const float e2 = c[5] + hc[5];
  float s;
  if (kFp64Det) {
    // determinant and reciprocal in FP64, rounded once to float, as TBB:457-459 does.
    // Kept exact in every build: the chained filter's accuracy follows the precision of s
    // closely (an extra 0.5 ulp of random error in s alone raises the 99th-percentile
    // covariance error by ~40 %, 2 ulp by ~4x; the other divisions and square roots are
    // insensitive at 2 ulp).
    const double det = (double)e0 * e2 - (double)e1 * e1;
    s = (float)(1.0 / det);
  } else {
    s = fdiv(1.f, e0 * e2 - e1 * e1);
  }
  const float i0 = s * e2;
  const float i1 = e1 * -s;
  const float i2 = s * e0;

  // gain rows m: K = C H^T inv(R), H = [[rotT00, rotT01, 0...], [0, 0, 1, 0...]]
  float K0[6], K1[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const float cm0 = c[S6(m, 0)], cm1 = c[S6(m, 1)], cm2 = c[S6(m, 2)];
    K0[m] = cm0 * (rotT00 * i0) + cm1 * (rotT01 * i0) + cm2 * i1;
    K1[m] = cm0 * (rotT00 * i1) + cm1 * (rotT01 * i1) + cm2 * i2;
  }
  const float res0 = rotT00 * (hp[0] - p[0]) + rotT01 * (hp[1] - p[1]);
  const float res1 = hp[2] - p[2];
  float chi2 = 0.f;
  if (kChi2) chi2 = i0 * res0 * res0 + 2.f * i1 * res0 * res1 + i2 * res1 * res1;
#pragma unroll
  for (int m = 0; m < 6; ++m) p[m] = p[m] + K0[m] * res0 + K1[m] * res1;

  // C' = C - K H C, lower triangle
  float nc[21];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j)
      nc[S6(i, j)] = c[S6(i, j)] - (K0[i] * rotT00 * c[S6(0, j)] + K0[i] * rotT01 * c[S6(1, j)] + K1[i] * c[S6(2, j)]);
#pragma unroll
  for (int i = 0; i < 21; ++i) c[i] = nc[i];
  return chi2;
}

}  // namespace p2r
