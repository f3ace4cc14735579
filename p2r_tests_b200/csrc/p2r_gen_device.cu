// Device-side synthetic-helix generator: the recipe of p2r_gen_helix (p2r_gen.cpp) with the
// same counter-based random streams, one thread per track slot, writing the Matriplex track
// and hit arrays directly in device memory. It replaces the host generation plus the
// host-to-device copy of the inputs (the reference builds its inputs on the host,
// prepareTracks / prepareHits, TBB:243-293).
//
// Every double-precision multiply that feeds an add is written with __dmul_rn / __dadd_rn so
// no operation is fused: the arithmetic is the host generator's operation for operation. The
// transcendental functions (log, sin, cos, asin) are CUDA's; they may differ from the host C
// library's by an ulp of double, which survives the rounding to float only rarely, so the
// arrays equal the host generator's bit for bit except for isolated 1-ulp (float) differences.
#include <cuda_runtime.h>
#include <stdint.h>

#include "p2r_internal.h"

namespace {

constexpr double kPi = 3.141592653589793;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct DevRng {  // the host generator's stream for (seed, track)
  uint64_t key, ctr;
  __device__ DevRng(uint64_t seed, uint64_t track) : key(mix64(seed ^ mix64(track + 0x51ED270B27E3D4A1ull))), ctr(0) {}
  __device__ double uniform() {  // (0, 1)
    const uint64_t v = mix64(key + (ctr++) * 0xD1B54A32D192ED03ull);
    return __dmul_rn(__dadd_rn((double)(v >> 11), 0.5), 1.0 / 9007199254740992.0);
  }
  __device__ double gauss() {  // Box-Muller, one value per call
    const double u1 = uniform(), u2 = uniform();
    return __dmul_rn(sqrt(__dmul_rn(-2.0, log(u1))), cos(__dmul_rn(6.283185307179586, u2)));
  }
};

__device__ __forceinline__ void helix_at(double phi0, int q, double R, double cot_theta, double s, double* x,
                                         double* y, double* z, double* phi) {
  const double a = __dsub_rn(phi0, __ddiv_rn(__dmul_rn((double)q, s), R));
  const double rq = __ddiv_rn(R, (double)q);
  *x = __dmul_rn(-rq, __dsub_rn(sin(a), sin(phi0)));
  *y = __dmul_rn(rq, __dsub_rn(cos(a), cos(phi0)));
  *z = __dmul_rn(s, cot_theta);
  *phi = a;
}

__device__ __forceinline__ double path_to_radius(double R, double rho) {
  const double t = __ddiv_rn(rho, __dmul_rn(2.0, R));
  return t <= 1.0 ? __dmul_rn(__dmul_rn(2.0, R), asin(t)) : __longlong_as_double(0x7ff8000000000000ll);
}

__device__ __forceinline__ int sym6(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

__global__ void __launch_bounds__(128) gen_helix_kernel(p2r_gen_params gp, int bsize, long long nevts, long long nb,
                                                        int nlayer, const int32_t* ntrk_event, float* trk,
                                                        float* hit) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nevts * nb * bsize) return;
  const long long b = g / bsize;
  const int it = (int)(g - b * bsize);
  const long long ev = b / nb, ib = b - ev * nb;
  const long long ntr = ntrk_event ? ntrk_event[ev] : nb * bsize;
  const long long itrk = ib * bsize + it;
  const long long tw = 28LL * bsize, hw = 9LL * bsize;
  float* tb = trk + b * tw;
  const double kB = __dmul_rn(0.299792458, gp.bz);

  DevRng rng(gp.seed, (uint64_t)(ev * nb * bsize + itrk));
  const double phi0 = __dadd_rn(-kPi, __dmul_rn(2 * kPi, rng.uniform()));
  const double theta = __dadd_rn(gp.theta_min, __dmul_rn(__dsub_rn(gp.theta_max, gp.theta_min), rng.uniform()));
  const double pt = __dmul_rn(gp.pt, __dadd_rn(1.0, __dmul_rn(gp.pop_smear, rng.gauss())));
  const double rseed = __dmul_rn(gp.r_seed, __dadd_rn(1.0, __dmul_rn(gp.pop_smear, rng.gauss())));
  const int q = rng.uniform() < 0.5 ? -1 : 1;
  const int qturn = gp.bz > 0 ? q : -q;
  const double R = __ddiv_rn(__dmul_rn(100.0, fabs(pt)), fabs(kB));
  const double cot = __ddiv_rn(cos(theta), sin(theta));
  double par[6];
  const double s0 = path_to_radius(R, rseed);
  helix_at(phi0, qturn, R, cot, s0, &par[0], &par[1], &par[2], &par[4]);
  par[3] = __ddiv_rn(1.0, fabs(pt));
  par[5] = theta;
  const bool live = itrk < ntr;
  const double d[6] = {gp.cov_pos, gp.cov_pos, gp.cov_pos, gp.cov_ang, gp.cov_ang, gp.cov_ang};
#pragma unroll
  for (int ip = 0; ip < 6; ++ip) {
    const double v = __dadd_rn(par[ip], __dmul_rn(__dmul_rn(gp.est_smear, sqrt(d[ip])), rng.gauss()));
    tb[it + ip * bsize] = live ? (float)v : (float)par[ip];
  }
#pragma unroll
  for (int ip = 0; ip < 21; ++ip) tb[(6 + ip) * bsize + it] = 0.f;
#pragma unroll
  for (int i = 0; i < 6; ++i) tb[(6 + sym6(i, i)) * bsize + it] = (float)d[i];
  tb[27 * bsize + it] = __int_as_float(q);
  const double hv = __dmul_rn(gp.hit_sigma, gp.hit_sigma);
  for (int lay = 0; lay < nlayer; ++lay) {
    float* hb = hit + (lay + (long long)nlayer * b) * hw;
    const double rho =
        nlayer > 1 ? __dadd_rn(gp.r_first, __ddiv_rn(__dmul_rn(__dsub_rn(gp.r_last, gp.r_first), (double)lay),
                                                      (double)(nlayer - 1)))
                   : gp.r_first;
    const double s = path_to_radius(R, rho);
    double hx, hy, hz, hphi;
    helix_at(phi0, qturn, R, cot, s, &hx, &hy, &hz, &hphi);
    const double gx = rng.gauss(), gy = rng.gauss(), gz = rng.gauss();
    hb[it] = (float)__dadd_rn(hx, __dmul_rn(gp.hit_sigma, gx));
    hb[it + bsize] = (float)__dadd_rn(hy, __dmul_rn(gp.hit_sigma, gy));
    hb[it + 2 * bsize] = (float)__dadd_rn(hz, __dmul_rn(gp.hit_sigma, gz));
    hb[it + 3 * bsize] = (float)hv;
    hb[it + 4 * bsize] = 0.f;
    hb[it + 5 * bsize] = (float)hv;
    hb[it + 6 * bsize] = 0.f;
    hb[it + 7 * bsize] = 0.f;
    hb[it + 8 * bsize] = (float)hv;
  }
}

}  // namespace

extern "C" int p2r_gen_helix_device(const p2r_gen_params* gp, int32_t bsize, int64_t nevts, int64_t nb,
                                    int32_t nlayer, const int32_t* ntrk_event, void* trk_out, void* hit_out,
                                    void* stream) {
  P2rRange range("p2r_gen_helix_device");
  if (!gp) return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_helix_device: null parameters");
  if (bsize < 1 || nevts < 0 || nb < 0 || nlayer < 1 || gp->bz == 0.0 || gp->r_last <= gp->r_first)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_helix_device: bad sizes or geometry");
  const long long nslots = (long long)nevts * nb * bsize;
  if (nslots == 0) return p2r_clear_error();
  if (!trk_out || !hit_out) return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_helix_device: null array pointer");
  if (int rc = p2r_check_aligned("p2r_gen_helix_device", 4, {trk_out, hit_out, ntrk_event})) return rc;
  const long long grid = (nslots + 127) / 128;
  if (grid > 0x7fffffffLL) return p2r_set_error(P2R_ERR_INVALID, "p2r_gen_helix_device: too many track slots");
  gen_helix_kernel<<<(unsigned)grid, 128, 0, (cudaStream_t)stream>>>(*gp, bsize, nevts, nb, nlayer, ntrk_event,
                                                                      (float*)trk_out, (float*)hit_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_gen_helix_device: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}
