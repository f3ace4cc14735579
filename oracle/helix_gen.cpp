// Seeded synthetic helix events for the oracle side of the benchmark.
//
// TEST INFRASTRUCTURE ONLY. bench.py's reference arm and CPU-baseline leg generate their
// inputs here so that the timed reference path maps no library of the product. The recipe is
// the product's own workload definition (p2r_gen_helix, documented with p2r_gen_params in
// include/p2r.h), restated so its output is bit-identical to the product's host generator;
// tests/test_oracle_golden.py checks that equality on the benchmark's seeds.
//
// The reference has no generator for these workloads: its own inputs come from one fixture
// track smeared per element (prepareTracks / prepareHits, src/propagate-tor-test_tbb.cpp:243-293).
//
// Recipe, per track (event ev, track index i within the event, global index ev*nb*bsize + i):
//   random stream: splitmix64 counter stream keyed by (seed, global index); uniforms in (0, 1)
//   from the top 53 bits; Gaussians by Box-Muller, one value per two uniforms.
//   draws in order: phi0, theta, pT smear, seed-radius smear, charge, 6 estimate displacements,
//   then per layer 3 hit smears.
//   geometry in double: a helix from the origin, bending radius R = 100 pT / (0.299792458 |Bz|),
//   position after transverse path s: x = -(R/q)(sin(phi0 - q s/R) - sin phi0),
//   y = (R/q)(cos(phi0 - q s/R) - cos phi0), z = s cot(theta); the path to radius rho is
//   2R asin(rho / 2R).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

class Stream {
 public:
  Stream(uint64_t seed, uint64_t index) : key_(splitmix(seed ^ splitmix(index + 0x51ED270B27E3D4A1ull))) {}
  double u() {
    const uint64_t v = splitmix(key_ + (n_++) * 0xD1B54A32D192ED03ull);
    return ((v >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  }
  double n() {
    const double a = u(), b = u();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
  }

 private:
  uint64_t key_, n_ = 0;
};

struct Point {
  double x, y, z, phi;
};

Point on_helix(double phi0, int turn, double R, double cot_theta, double s) {
  const double a = phi0 - turn * s / R;
  return {-(R / turn) * (std::sin(a) - std::sin(phi0)), (R / turn) * (std::cos(a) - std::cos(phi0)), s * cot_theta,
          a};
}

double path_at_radius(double R, double rho) {
  const double t = rho / (2.0 * R);
  return t <= 1.0 ? 2.0 * R * std::asin(t) : NAN;
}

}  // namespace

extern "C" {

// prm: seed as the first 8 bytes (uint64), then the doubles bz, r_seed, r_first, r_last, pt,
// pop_smear, theta_min, theta_max, cov_pos, cov_ang, est_smear, hit_sigma (the field order of
// p2r_gen_params). Writes nevts*nb MPTRK blocks and nevts*nb*nlayer MPHIT blocks.
// Returns 0, or 1 on bad arguments.
int orc_gen_helix(uint64_t seed, const double* prm, int bsize, long nevts, long nb, int nlayer,
                  const int* ntrk_event, float* trk, float* hit, int nthreads) {
  if (!prm || !trk || !hit || bsize < 1 || nevts < 0 || nb < 0 || nlayer < 1) return 1;
  const double bz = prm[0], r_seed = prm[1], r_first = prm[2], r_last = prm[3], pt_nom = prm[4];
  const double pop = prm[5], th_lo = prm[6], th_hi = prm[7], cov_pos = prm[8], cov_ang = prm[9];
  const double est = prm[10], sig = prm[11];
  if (bz == 0.0 || r_last <= r_first) return 1;
  const long tw = 28L * bsize, hw = 9L * bsize, nblocks = nevts * nb;
  const double kB = 0.299792458 * bz;
  auto fill = [&](long b0, long b1) {
    for (long b = b0; b < b1; ++b) {
      const long ev = b / nb, ib = b % nb;
      const long live_tracks = ntrk_event ? ntrk_event[ev] : nb * bsize;
      float* tb = trk + b * tw;
      for (int lane = 0; lane < bsize; ++lane) {
        const long i = ib * bsize + lane;
        Stream rs(seed, (uint64_t)(ev * nb * bsize + i));
        const double phi0 = -M_PI + 2 * M_PI * rs.u();
        const double theta = th_lo + (th_hi - th_lo) * rs.u();
        const double pt = pt_nom * (1.0 + pop * rs.n());
        const double rho0 = r_seed * (1.0 + pop * rs.n());
        const int q = rs.u() < 0.5 ? -1 : 1;
        const int turn = bz > 0 ? q : -q;
        const double R = 100.0 * std::fabs(pt) / std::fabs(kB);
        const double cot = std::cos(theta) / std::sin(theta);
        const Point s = on_helix(phi0, turn, R, cot, path_at_radius(R, rho0));
        const double truth[6] = {s.x, s.y, s.z, 1.0 / std::fabs(pt), s.phi, theta};
        const double var[6] = {cov_pos, cov_pos, cov_pos, cov_ang, cov_ang, cov_ang};
        const bool live = i < live_tracks;
        for (int c = 0; c < 6; ++c) {
          const double v = truth[c] + est * std::sqrt(var[c]) * rs.n();
          tb[c * bsize + lane] = (float)(live ? v : truth[c]);
        }
        for (int c = 0; c < 21; ++c) tb[(6 + c) * bsize + lane] = 0.f;
        for (int d = 0; d < 6; ++d) tb[(6 + d * (d + 3) / 2) * bsize + lane] = (float)var[d];
        const int32_t qq = q;
        std::memcpy(&tb[27 * bsize + lane], &qq, 4);
        const double hv = sig * sig;
        for (int l = 0; l < nlayer; ++l) {
          float* hb = hit + (l + (long)nlayer * b) * hw;
          const double rho = nlayer > 1 ? r_first + (r_last - r_first) * l / (nlayer - 1) : r_first;
          const Point h = on_helix(phi0, turn, R, cot, path_at_radius(R, rho));
          const double hx = h.x + sig * rs.n();
          const double hy = h.y + sig * rs.n();
          const double hz = h.z + sig * rs.n();
          hb[0 * bsize + lane] = (float)hx;
          hb[1 * bsize + lane] = (float)hy;
          hb[2 * bsize + lane] = (float)hz;
          const double hc[6] = {hv, 0, hv, 0, 0, hv};
          for (int c = 0; c < 6; ++c) hb[(3 + c) * bsize + lane] = (float)hc[c];
        }
      }
    }
  };
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  nt = nt < 1 ? 1 : (nt > 64 ? 64 : nt);
  if (nblocks < 64 || nt == 1) {
    fill(0, nblocks);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) pool.emplace_back(fill, nblocks * t / nt, nblocks * (t + 1) / nt);
    for (auto& th : pool) th.join();
  }
  return 0;
}

}  // extern "C"
