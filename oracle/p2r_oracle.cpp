// p2r oracle: a CPU restatement of the reference's hot path, written per track.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load this library (oracle/_build/libp2r_oracle.so), and only as the
// checker; the product path never calls it.
//
// Parity pinning: the float instantiation is checked against the reference's own
// functions compiled from its source (oracle/ref_harness.cpp -> oracle/_ref/) and against
// the golden vectors in tests/golden/, which that harness generated. The double
// instantiation gives the error of every reported float result.
//
// Reference: src/propagate-tor-test_tbb.cpp of cerati/p2r-tests ("TBB" below).
//   Matriplex layout     TBB:56-125  element (lane it, component ip) at data[it + ip*bsize]
//   symmetric packing    TBB:46-54   lower triangle, (i>=j) -> i*(i+1)/2 + j
//   block indexing       TBB:147-153 (tracks), TBB:212-217 (hits)
//   hipo / sincos4       TBB:428-431 / TBB:644-652
//   propagateToR         TBB:656-812 (with MultHelixProp TBB:296-341, Transp TBB:343-373)
//   KalmanUpdate         TBB:433-642
//   driver loop          TBB:870-926 (restart); chained as in cuda_v4.cu:840-846
//
// Extensions that are zero / identity at their default values:
//   dr[layer]   radius offset added to the propagation target radius (default 0)
//   kfact       100/(-0.299792458*Bz) (TBB:654 hard-codes Bz = 3.8112 T)
//   chi2        res_loc^T * inv(resErr_loc) * res_loc of each update, summed over layers
//               (the reference leaves Chi2Similarity commented out, TBB:631)
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

inline int sym6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

template <class T>
struct Trk {
  T par[6];   // x, y, z, ipt, phi, theta
  T cov[21];  // symmetric 6x6, lower triangle
  int q;
};

template <class T>
struct Hit {
  T pos[3];
  T cov[6];  // symmetric 3x3, lower triangle
};

template <class T>
inline T hypot2(T x, T y) { return std::sqrt(x * x + y * y); }  // TBB:428-431

// TBB:644-652 (4th-order cos, 3rd-order sin). omc = 1 - c is evaluated as x^2/2 - x^4/24,
// the algebraically identical form the reference's -ffast-math build computes for its
// 1 - cosa (TBB:738-739, 756, 763); formed as 1 - c in float it cancels for the tiny
// angles of the later helix iterations.
template <class T>
inline void sincos4_(T x, T& s, T& c, T& omc) {
  const T x2 = x * x;
  omc = T(0.5) * x2 - T(0.04166667f) * x2 * x2;
  c = T(1) - omc;
  s = x - T(0.16666667f) * x * x2;
}

// Helix propagation of one track to the radius of `hitpos` (+ dr), TBB:656-812.
// Writes the propagated parameters and J*C*J^T into `out` (out may alias in).
template <class T>
void propagate_to_r(const Trk<T>& in, const T* hitpos, T dr, T kfact, Trk<T>& out) {
  const T xin = in.par[0], yin = in.par[1], zin = in.par[2];
  const T iptin = in.par[3], phiin = in.par[4], thetain = in.par[5];
  T r0 = hypot2(xin, yin);
  const T k = T(in.q) * kfact;
  const T r = hypot2(hitpos[0], hitpos[1]) + dr;
  const T kinv = T(1) / k;
  const T pt = T(1) / iptin;

  T D = 0, cosa = 0, sina = 0, id = 0, omc = 0;
  const T cosP = std::cos(phiin), sinP = std::sin(phiin);
  T px = cosP * pt, py = sinP * pt;
  T dDdx = r0 > T(0) ? -xin / r0 : T(0);
  T dDdy = r0 > T(0) ? -yin / r0 : T(0);
  T dDdipt = 0, dDdphi = 0;
  T xo = xin, yo = yin;

  const int niter = 5;  // TBB:655
  for (int i = 0; i < niter; ++i) {
    r0 = hypot2(xo, yo);
    id = r - r0;
    D += id;
    sincos4_(id * iptin * kinv, sina, cosa, omc);
    if (i + 1 != niter) {
      // derivatives of the total path w.r.t. x, y, ipt, phi, only once the step is
      // below 1 um (TBB:714); the branch is part of the algorithm.
      const T oor0 = (r0 > T(0) && std::fabs(r - r0) < T(0.0001f)) ? T(1) / r0 : T(0);
      const T dadipt = id * kinv;
      const T dadx = -xo * iptin * kinv * oor0;
      const T dady = -yo * iptin * kinv * oor0;
      const T pxca = px * cosa, pxsa = px * sina, pyca = py * cosa, pysa = py * sina;
      T tmp = k * dadx;
      dDdx -= (xo * (T(1) + tmp * (pxca - pysa)) + yo * tmp * (pyca + pxsa)) * oor0;
      tmp = k * dady;
      dDdy -= (xo * tmp * (pxca - pysa) + yo * (T(1) + tmp * (pyca + pxsa))) * oor0;
      tmp = dadipt * iptin;
      dDdipt -= k * (xo * (pxca * tmp - pysa * tmp - pyca - pxsa + py) +
                     yo * (pyca * tmp + pxsa * tmp - pysa + pxca - px)) * pt * oor0;
      dDdphi += k * (xo * (pysa - px + pxca) - yo * (pxsa - py + pyca)) * oor0;
    }
    xo = xo + k * (px * sina - py * omc);
    yo = yo + k * (py * sina + px * omc);
    const T pxold = px;
    px = px * cosa - py * sina;
    py = py * cosa + pxold * sina;
  }

  const T alpha = D * iptin * kinv;
  const T dadx = dDdx * iptin * kinv;
  const T dady = dDdy * iptin * kinv;
  const T dadipt = (iptin * dDdipt + D) * kinv;
  const T dadphi = dDdphi * iptin * kinv;
  sincos4_(alpha, sina, cosa, omc);

  // Transport Jacobian, dense 6x6 (TBB:753-807).
  T J[6][6] = {};
  J[0][0] = T(1) + k * dadx * (cosP * cosa - sinP * sina) * pt;
  J[0][1] = k * dady * (cosP * cosa - sinP * sina) * pt;
  J[0][3] = k * (cosP * (iptin * dadipt * cosa - sina) + sinP * (omc - iptin * dadipt * sina)) * pt * pt;
  J[0][4] = k * (cosP * dadphi * cosa - sinP * dadphi * sina - sinP * sina + cosP * cosa - cosP) * pt;
  J[1][0] = k * dadx * (sinP * cosa + cosP * sina) * pt;
  J[1][1] = T(1) + k * dady * (sinP * cosa + cosP * sina) * pt;
  J[1][3] = k * (sinP * (iptin * dadipt * cosa - sina) + cosP * (iptin * dadipt * sina - omc)) * pt * pt;
  J[1][4] = k * (sinP * dadphi * cosa + cosP * dadphi * sina + sinP * cosa + cosP * sina - sinP) * pt;
  const T cosT = std::cos(thetain);
  const T isinT = T(1) / std::sin(thetain);
  J[2][0] = k * cosT * dadx * pt * isinT;
  J[2][1] = k * cosT * dady * pt * isinT;
  J[2][2] = T(1);
  J[2][3] = k * cosT * (iptin * dadipt - alpha) * pt * pt * isinT;
  J[2][4] = k * dadphi * cosT * pt * isinT;
  J[2][5] = -k * alpha * pt * isinT * isinT;
  J[3][3] = T(1);
  J[4][0] = dadx;
  J[4][1] = dady;
  J[4][3] = dadipt;
  J[4][4] = T(1) + dadphi;
  J[5][5] = T(1);

  // C' = J * C * J^T, accumulated in increasing column order as MultHelixProp /
  // MultHelixPropTransp do (TBB:296-373); structural zeros contribute exact zeros.
  T C[6][6], JC[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) C[i][j] = in.cov[sym6(i, j)];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      T s = 0;
      for (int m = 0; m < 6; ++m)
        if (J[i][m] != T(0)) s += J[i][m] * C[m][j];
      JC[i][j] = s;
    }
  T outcov[21];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      T s = 0;
      for (int m = 0; m < 6; ++m)
        if (J[j][m] != T(0)) s += JC[i][m] * J[j][m];
      outcov[sym6(i, j)] = s;
    }

  out.q = in.q;
  out.par[0] = xo;
  out.par[1] = yo;
  out.par[2] = zin + k * alpha * cosT * pt * isinT;
  out.par[3] = iptin;
  out.par[4] = phiin + alpha;
  out.par[5] = thetain;
  for (int i = 0; i < 21; ++i) out.cov[i] = outcov[i];
}

// Kalman update of one track with one hit, in place (TBB:433-642). The residual
// covariance is the 2x2 projection onto the plane tangent to the hit's cylinder; its
// determinant is taken in double as TBB:457-458 does. Returns the chi2 of the update
// (pre-update residual, inverse residual covariance).
template <class T>
T kalman_update(Trk<T>& t, const Hit<T>& h) {
  const T* C = t.cov;
  const T* H = h.cov;
  const T r = hypot2(h.pos[0], h.pos[1]);
  const T rotT00 = -(h.pos[1] + t.par[1]) / (T(2) * r);
  const T rotT01 = (h.pos[0] + t.par[0]) / (T(2) * r);

  T e0 = (rotT00 * (C[0] + H[0]) + rotT01 * (C[1] + H[1])) * rotT00 +
         (rotT00 * (C[1] + H[1]) + rotT01 * (C[2] + H[2])) * rotT01;
  T e1 = (C[3] + H[3]) * rotT00 + (C[4] + H[4]) * rotT01;
  T e2 = C[5] + H[5];
  const double det = (double)e0 * e2 - (double)e1 * e1;
  const T s = T(1.0 / det);
  const T i0 = s * e2;
  const T i1 = -s * e1;
  const T i2 = s * e0;

  // gain K = C H^T inv, with H = [[rotT00, rotT01, 0, 0, 0, 0], [0, 0, 1, 0, 0, 0]]
  T K[6][2];
  for (int m = 0; m < 6; ++m) {
    const T cm0 = C[sym6(m, 0)], cm1 = C[sym6(m, 1)], cm2 = C[sym6(m, 2)];
    K[m][0] = cm0 * (rotT00 * i0) + cm1 * (rotT01 * i0) + cm2 * i1;
    K[m][1] = cm0 * (rotT00 * i1) + cm1 * (rotT01 * i1) + cm2 * i2;
  }
  const T res0 = rotT00 * (h.pos[0] - t.par[0]) + rotT01 * (h.pos[1] - t.par[1]);
  const T res1 = h.pos[2] - t.par[2];
  const T chi2 = i0 * res0 * res0 + T(2) * i1 * res0 * res1 + i2 * res1 * res1;
  for (int m = 0; m < 6; ++m) t.par[m] = t.par[m] + K[m][0] * res0 + K[m][1] * res1;

  T nc[21];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      const T khc = K[i][0] * rotT00 * C[sym6(0, j)] + K[i][0] * rotT01 * C[sym6(1, j)] + K[i][1] * C[sym6(2, j)];
      nc[sym6(i, j)] = C[sym6(i, j)] - khc;
    }
  for (int i = 0; i < 21; ++i) t.cov[i] = nc[i];
  return chi2;
}

// Matriplex <-> per-track access for one track. `bs` = bsize.
template <class T>
void load_trk(const float* blk, int bs, int it, Trk<T>& t) {
  for (int i = 0; i < 6; ++i) t.par[i] = T(blk[it + i * bs]);
  for (int i = 0; i < 21; ++i) t.cov[i] = T(blk[(6 + i) * bs + it]);
  int32_t q;
  std::memcpy(&q, &blk[27 * bs + it], 4);
  t.q = q;
}
template <class T>
void load_hit(const float* blk, int bs, int it, Hit<T>& h) {
  for (int i = 0; i < 3; ++i) h.pos[i] = T(blk[it + i * bs]);
  for (int i = 0; i < 6; ++i) h.cov[i] = T(blk[(3 + i) * bs + it]);
}

// Runs every track of `nblocks` Matriplex blocks through its layers.
//   mode 0 = restart (each layer starts again from the input track, TBB:894),
//   mode 1 = chained (the state is carried from layer to layer),
//   mode 2 = chained propagation only (no KalmanUpdate; for propagateToR-alone checks).
//   nlay_lane (nullable): per-track layer count; lanes stop updating after it.
// Output: float path -> MPTRK layout into out_f (28*bsize words per block);
//         both paths -> per-track par (6) and cov (21) in double into par_d / cov_d
//         (nullable), the chi2 into chi2_d (nullable; chained: summed over layers,
//         restart: of the last layer's update, the only one that reaches the output), and
//         the covariance that entered the last update into prior_d (nullable, 21 per track).
template <class T>
void run_tracks(const float* trk, const float* hit, long nblocks, int bs, int nlayer, int mode,
                float kfact_f, double kfact_d, const double* dr, const int* nlay_lane, float* out_f,
                double* par_d, double* cov_d, double* chi2_d, double* prior_d) {
  const T kfact = sizeof(T) == sizeof(float) ? T(kfact_f) : T(kfact_d);
  const long tw = 28L * bs, hw = 9L * bs;
  for (long b = 0; b < nblocks; ++b) {
    for (int it = 0; it < bs; ++it) {
      Trk<T> in, st;
      load_trk(trk + b * tw, bs, it, in);
      st = in;
      T chi2 = 0;
      const int nl = nlay_lane ? nlay_lane[b * bs + it] : nlayer;
      if (prior_d)  // a lane with no layer keeps its input covariance
        for (int i = 0; i < 21; ++i) prior_d[(b * bs + it) * 21 + i] = double(st.cov[i]);
      for (int l = 0; l < nlayer && l < nl; ++l) {
        Hit<T> h;
        load_hit(hit + (b * nlayer + l) * hw, bs, it, h);
        const T drl = dr ? T(dr[l]) : T(0);
        if (mode == 0)
          propagate_to_r(in, h.pos, drl, kfact, st);
        else
          propagate_to_r(st, h.pos, drl, kfact, st);
        if (mode == 2) {  // propagation only: no update, the output covariance is its own scale
          if (prior_d)
            for (int i = 0; i < 21; ++i) prior_d[(b * bs + it) * 21 + i] = double(st.cov[i]);
          continue;
        }
        if (prior_d)  // covariance entering the last update (the scale its rounding acts on)
          for (int i = 0; i < 21; ++i) prior_d[(b * bs + it) * 21 + i] = double(st.cov[i]);
        // restart: only the last layer's update survives, and so does only its chi2
        if (mode == 0) chi2 = 0;
        chi2 += kalman_update(st, h);
      }
      const long tr = b * bs + it;
      if (out_f) {
        float* ob = out_f + b * tw;
        for (int i = 0; i < 6; ++i) ob[i * bs + it] = float(st.par[i]);
        for (int i = 0; i < 21; ++i) ob[(6 + i) * bs + it] = float(st.cov[i]);
        int32_t q = st.q;
        std::memcpy(&ob[27 * bs + it], &q, 4);
      }
      if (par_d)
        for (int i = 0; i < 6; ++i) par_d[tr * 6 + i] = double(st.par[i]);
      if (cov_d)
        for (int i = 0; i < 21; ++i) cov_d[tr * 21 + i] = double(st.cov[i]);
      if (chi2_d) chi2_d[tr] = double(chi2);
    }
  }
}

}  // namespace

extern "C" {

// kfact for a field of bz tesla, rounded to float as TBB:654 rounds its constant.
float orc_kfact_f32(double bz) { return float(100 / (-0.299792458 * bz)); }
double orc_kfact_f64(double bz) { return 100 / (-0.299792458 * bz); }

// Whole-array runs. Track blocks are laid out ev-major (block ib + nb*ev, TBB:147-153)
// and hit blocks as lay + b*nlayer with b = ib + nb*ev (TBB:215-217), so a flat block
// index b covers both.
void orc_run_f32(const float* trk, const float* hit, long nblocks, int bsize, int nlayer, int mode,
                 double bz, const double* dr, const int* nlay_lane, float* out, double* par_d,
                 double* cov_d, double* chi2_d, double* prior_d) {
  run_tracks<float>(trk, hit, nblocks, bsize, nlayer, mode, orc_kfact_f32(bz), orc_kfact_f64(bz), dr,
                    nlay_lane, out, par_d, cov_d, chi2_d, prior_d);
}

void orc_run_f64(const float* trk, const float* hit, long nblocks, int bsize, int nlayer, int mode,
                 double bz, const double* dr, const int* nlay_lane, float* out, double* par_d,
                 double* cov_d, double* chi2_d, double* prior_d) {
  run_tracks<double>(trk, hit, nblocks, bsize, nlayer, mode, orc_kfact_f32(bz), orc_kfact_f64(bz), dr,
                     nlay_lane, out, par_d, cov_d, chi2_d, prior_d);
}

// Single-layer, single-track entry points in double for finite-difference gradient
// checks: one propagate + update per call, state in/out as par[6], cov[21].
double orc_step_f64(const double* par_in, const double* cov_in, int q, const double* hitpos,
                    const double* hitcov, double dr, double bz, double* par_out, double* cov_out) {
  Trk<double> t;
  for (int i = 0; i < 6; ++i) t.par[i] = par_in[i];
  for (int i = 0; i < 21; ++i) t.cov[i] = cov_in[i];
  t.q = q;
  Hit<double> h;
  for (int i = 0; i < 3; ++i) h.pos[i] = hitpos[i];
  for (int i = 0; i < 6; ++i) h.cov[i] = hitcov[i];
  propagate_to_r(t, h.pos, dr, orc_kfact_f64(bz), t);
  const double chi2 = kalman_update(t, h);
  for (int i = 0; i < 6; ++i) par_out[i] = t.par[i];
  for (int i = 0; i < 21; ++i) cov_out[i] = t.cov[i];
  return chi2;
}

}  // extern "C"
