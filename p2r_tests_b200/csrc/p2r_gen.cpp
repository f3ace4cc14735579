// Host-side input generators for the Matriplex track / hit arrays.
//
// 1. p2r_gen_fixture: the reference's own input recipe (prepareTracks / prepareHits,
//    src/propagate-tor-test_tbb.cpp:243-293, with randn TBB:127-145): every element of
//    one seed track and of one hit per layer is multiplied by (1 + smear*N(0,1)), the
//    track covariance additionally by 100, drawing Gaussians with the Marsaglia polar
//    method on glibc rand() in the reference's element order (par 6, cov 21 per lane;
//    then per layer pos 3, cov 6 per lane). The seed track and hits are caller-supplied.
//
// 2. p2r_gen_helix: seeded synthetic events of true helices (FP64) in a solenoidal
//    field, with hits on concentric cylinders, for workloads the reference has no
//    generator for (see p2r_gen_params in include/p2r.h). Deterministic for a given seed,
//    independent of thread count (counter-based random numbers keyed by the global track
//    index).
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "p2r_internal.h"

namespace {

// ---------------------------------------------------------------- fixture recipe
struct PolarGauss {  // Marsaglia polar method on rand(), one spare value kept
  bool have = false;
  float spare = 0.f;
  float next() {
    if (have) {
      have = false;
      return spare;
    }
    float u1, u2, w;
    do {
      u1 = -1 + ((float)rand() / RAND_MAX) * 2;
      u2 = -1 + ((float)rand() / RAND_MAX) * 2;
      w = (float)((double)u1 * u1 + (double)u2 * u2);
    } while (w >= 1 || w == 0);
    const float mult = std::sqrt((-2 * std::log(w)) / w);
    spare = u2 * mult;
    have = true;
    return u1 * mult;
  }
};

// ---------------------------------------------------------------- helix recipe
inline uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct TrackRng {  // independent stream per (seed, track)
  uint64_t key, ctr = 0;
  TrackRng(uint64_t seed, uint64_t track) : key(mix64(seed ^ mix64(track + 0x51ED270B27E3D4A1ull))) {}
  double uniform() {  // (0, 1)
    const uint64_t v = mix64(key + (ctr++) * 0xD1B54A32D192ED03ull);
    return ((v >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  }
  double gauss() {  // Box-Muller, one value per call
    const double u1 = uniform(), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

inline int sym6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// Position and direction after transverse path length s on a helix from the origin with
// initial azimuth phi0, charge q and bending radius R (cm). The momentum azimuth turns
// by -q*s/R, the sense the propagation's alpha = id*ipt/k has for k = q*kfact.
inline void helix_at(double phi0, int q, double R, double cot_theta, double s, double* x, double* y,
                     double* z, double* phi) {
  const double a = phi0 - q * s / R;
  *x = -(R / q) * (std::sin(a) - std::sin(phi0));
  *y = (R / q) * (std::cos(a) - std::cos(phi0));
  *z = s * cot_theta;
  *phi = a;
}

// transverse path length at which a helix from the origin reaches radius rho
// (|pos(s)| = 2R sin(s / 2R)); NaN if it never does.
inline double path_to_radius(double R, double rho) {
  const double t = rho / (2.0 * R);
  return t <= 1.0 ? 2.0 * R * std::asin(t) : NAN;
}

}  // namespace

extern "C" {

int p2r_gen_fixture(const float* seed_par6, const float* seed_cov21, int seed_q, const float* hits_lx9,
                    int n_input_hits, int bsize, int64_t nevts, int64_t nb, int nlayer, double smear,
                    void* trk_out, void* hit_out) {
  if (!seed_par6 || !seed_cov21 || !hits_lx9 || !trk_out || !hit_out)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_fixture: null pointer");
  if (bsize < 1 || nevts < 0 || nb < 0 || nlayer < 1 || nlayer > n_input_hits)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_fixture: bad sizes (nlayer must be <= number of input hits)");
  float* trk = (float*)trk_out;
  float* hit = (float*)hit_out;
  const int64_t tw = 28LL * bsize, hw = 9LL * bsize;
  PolarGauss g;
  for (int64_t ie = 0; ie < nevts; ++ie)
    for (int64_t ib = 0; ib < nb; ++ib) {
      float* blk = trk + (ib + nb * ie) * tw;
      for (int it = 0; it < bsize; ++it) {
        // the reference's smear is a double literal, so the scaling runs in double
        for (int ip = 0; ip < 6; ++ip) blk[it + ip * bsize] = (float)((1 + smear * g.next()) * seed_par6[ip]);
        for (int ip = 0; ip < 21; ++ip)
          blk[(6 + ip) * bsize + it] = (float)((1 + smear * g.next()) * seed_cov21[ip] * 100);
        int32_t q = seed_q;
        std::memcpy(&blk[27 * bsize + it], &q, 4);
      }
    }
  for (int lay = 0; lay < nlayer; ++lay) {
    const float* h = hits_lx9 + 9 * lay;
    for (int64_t ie = 0; ie < nevts; ++ie)
      for (int64_t ib = 0; ib < nb; ++ib) {
        float* blk = hit + (lay + nlayer * (ib + nb * ie)) * hw;
        for (int it = 0; it < bsize; ++it) {
          for (int ip = 0; ip < 3; ++ip) blk[it + ip * bsize] = (float)((1 + smear * g.next()) * h[ip]);
          for (int ip = 0; ip < 6; ++ip) blk[(3 + ip) * bsize + it] = (float)((1 + smear * g.next()) * h[3 + ip]);
        }
      }
  }
  return P2R_OK;
}

int p2r_gen_helix(const p2r_gen_params* gp, int bsize, int64_t nevts, int64_t nb, int nlayer,
                  const int32_t* ntrk_event, void* trk_out, void* hit_out, int nthreads) {
  if (!gp || !trk_out || !hit_out) return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_helix: null pointer");
  if (bsize < 1 || nevts < 0 || nb < 0 || nlayer < 1 || gp->bz == 0.0 || gp->r_last <= gp->r_first)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_helix: bad sizes or geometry");
  float* trk = (float*)trk_out;
  float* hit = (float*)hit_out;
  const int64_t tw = 28LL * bsize, hw = 9LL * bsize;
  const int64_t nblocks = nevts * nb;
  const double kB = 0.299792458 * gp->bz;  // GeV/cm -> bending: R[cm] = 100*pT/kB
  auto work = [&](int64_t b0, int64_t b1) {
    for (int64_t b = b0; b < b1; ++b) {
      const int64_t ev = b / nb, ib = b % nb;
      const int64_t ntr = ntrk_event ? ntrk_event[ev] : nb * bsize;
      float* tb = trk + b * tw;
      for (int it = 0; it < bsize; ++it) {
        const int64_t itrk = ib * bsize + it;  // track index within the event
        TrackRng rng(gp->seed, (uint64_t)(ev * nb * bsize + itrk));
        const double phi0 = -M_PI + 2 * M_PI * rng.uniform();
        const double theta = gp->theta_min + (gp->theta_max - gp->theta_min) * rng.uniform();
        const double pt = gp->pt * (1.0 + gp->pop_smear * rng.gauss());
        const double rseed = gp->r_seed * (1.0 + gp->pop_smear * rng.gauss());
        const int q = rng.uniform() < 0.5 ? -1 : 1;
        const int qturn = gp->bz > 0 ? q : -q;  // turning sense of the momentum azimuth
        const double R = 100.0 * std::fabs(pt) / std::fabs(kB);
        const double cot = std::cos(theta) / std::sin(theta);
        double par[6];
        const double s0 = path_to_radius(R, rseed);
        helix_at(phi0, qturn, R, cot, s0, &par[0], &par[1], &par[2], &par[4]);
        par[3] = 1.0 / std::fabs(pt);
        par[5] = theta;
        const bool live = itrk < ntr;
        const double d[6] = {gp->cov_pos, gp->cov_pos, gp->cov_pos, gp->cov_ang, gp->cov_ang, gp->cov_ang};
        for (int ip = 0; ip < 6; ++ip) {
          const double v = par[ip] + gp->est_smear * std::sqrt(d[ip]) * rng.gauss();
          tb[it + ip * bsize] = live ? (float)v : (float)par[ip];
        }
        for (int ip = 0; ip < 21; ++ip) tb[(6 + ip) * bsize + it] = 0.f;
        for (int i = 0; i < 6; ++i) tb[(6 + sym6(i, i)) * bsize + it] = (float)d[i];
        int32_t qq = q;
        std::memcpy(&tb[27 * bsize + it], &qq, 4);
        for (int lay = 0; lay < nlayer; ++lay) {
          float* hb = hit + (lay + (int64_t)nlayer * b) * hw;
          const double rho = nlayer > 1 ? gp->r_first + (gp->r_last - gp->r_first) * lay / (nlayer - 1) : gp->r_first;
          const double s = path_to_radius(R, rho);
          double hx, hy, hz, hphi;
          helix_at(phi0, qturn, R, cot, s, &hx, &hy, &hz, &hphi);
          const double hpos[3] = {hx + gp->hit_sigma * rng.gauss(), hy + gp->hit_sigma * rng.gauss(),
                                  hz + gp->hit_sigma * rng.gauss()};
          for (int ip = 0; ip < 3; ++ip) hb[it + ip * bsize] = (float)hpos[ip];
          const double hv = gp->hit_sigma * gp->hit_sigma;
          const double hc[6] = {hv, 0, hv, 0, 0, hv};
          for (int ip = 0; ip < 6; ++ip) hb[(3 + ip) * bsize + it] = (float)hc[ip];
        }
      }
    }
  };
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  if (nblocks < 64 || nt == 1) {
    work(0, nblocks);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) pool.emplace_back(work, nblocks * t / nt, nblocks * (t + 1) / nt);
    for (auto& th : pool) th.join();
  }
  return P2R_OK;
}

void p2r_gen_params_default(p2r_gen_params* gp) {
  gp->seed = 20240001ull;
  gp->bz = 3.8;
  gp->r_seed = 15.0;
  gp->r_first = 20.0;
  gp->r_last = 100.0;
  gp->pt = 4.0;
  gp->pop_smear = 0.10;
  gp->theta_min = 0.3;
  gp->theta_max = 2.8;
  gp->cov_pos = 1e-4;
  gp->cov_ang = 1e-3;
  gp->est_smear = 1.0;
  gp->hit_sigma = 1e-3;
}

}  // extern "C"
