// p2r_driver: the reference program's main (src/propagate-tor-test_tbb.cpp:814-1055) over
// the C ABI: build the inputs, time NITER passes of the driver loop, print the same stdout
// lines the reference prints (so its build.py / read_throughput.py regex
// `done ntracks=(\d+) tot time=(\S+) ` reads the result) and the same validation summary.
//
// Sizes are run-time flags instead of the reference's -D macros (TBB:15-38):
//   --ntrks N --nevts E --nlayer L --bsize B --niter K --bz T --mode restart|chained
//   --input helix            synthetic helices (p2r_gen_helix defaults, Bz from --bz)
//   --input fixture FILE     the reference's recipe (TBB:243-293) on a seed track and hits
//                            read from FILE: 6 par, 21 cov, q, then n_hits x (3 pos, 6 cov),
//                            whitespace-separated, hits in the order the reference lists them
//   --transfer               time host->device, kernel and device->host (p2r_forward_host)
//                            instead of the kernel on resident arrays
// Build: compiled by p2r_tests_b200/build.py against libp2r_b200.so.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "p2r.h"

namespace {

struct Args {
  long ntrks = 9600, nevts = 100;
  int nlayer = 20, bsize = 32, niter = 5;
  double bz = 3.8;
  bool chained = true, transfer = false;
  std::string input = "helix", fixture;
};

int usage(const char* prog) {
  std::printf(
      "usage: %s [--ntrks N] [--nevts E] [--nlayer L] [--bsize B] [--niter K] [--bz T]\n"
      "          [--mode restart|chained] [--input helix | --input fixture FILE] [--transfer]\n",
      prog);
  return 0;
}

bool parse(int argc, char** argv, Args& a, bool& help) {
  for (int i = 1; i < argc; ++i) {
    const std::string k = argv[i];
    auto next = [&](const char* what) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", what);
        return nullptr;
      }
      return argv[++i];
    };
    const char* v = nullptr;
    if (k == "--help" || k == "-h") {
      help = true;
    } else if (k == "--ntrks" && (v = next("--ntrks"))) {
      a.ntrks = std::atol(v);
    } else if (k == "--nevts" && (v = next("--nevts"))) {
      a.nevts = std::atol(v);
    } else if (k == "--nlayer" && (v = next("--nlayer"))) {
      a.nlayer = std::atoi(v);
    } else if (k == "--bsize" && (v = next("--bsize"))) {
      a.bsize = std::atoi(v);
    } else if (k == "--niter" && (v = next("--niter"))) {
      a.niter = std::atoi(v);
    } else if (k == "--bz" && (v = next("--bz"))) {
      a.bz = std::atof(v);
    } else if (k == "--mode" && (v = next("--mode"))) {
      const std::string m = v;
      if (m != "restart" && m != "chained") {
        std::fprintf(stderr, "--mode must be restart or chained\n");
        return false;
      }
      a.chained = m == "chained";
    } else if (k == "--transfer") {
      a.transfer = true;
    } else if (k == "--input" && (v = next("--input"))) {
      a.input = v;
      if (a.input != "helix" && a.input != "fixture") {
        std::fprintf(stderr, "--input must be helix or fixture FILE\n");
        return false;
      }
      if (a.input == "fixture") {
        if (!(v = next("--input fixture"))) return false;
        a.fixture = v;
      }
    } else {
      std::fprintf(stderr, "unknown or incomplete argument %s\n", k.c_str());
      return false;
    }
  }
  return true;
}

#define CK(call)                                                                                   \
  do {                                                                                             \
    int rc_ = (call);                                                                              \
    if (rc_ != P2R_OK) {                                                                           \
      std::fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, p2r_last_error_string());           \
      return 2;                                                                                    \
    }                                                                                              \
  } while (0)
#define CU(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      std::fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));                      \
      return 3;                                                                                    \
    }                                                                                              \
  } while (0)

}  // namespace

int main(int argc, char** argv) {
  Args a;
  bool help = false;
  if (!parse(argc, argv, a, help)) return 1;
  if (help) return usage(argv[0]);
  if (p2r_abi_version() != P2R_ABI_VERSION) {  // a library from another header loaded at run time
    std::fprintf(stderr, "libp2r_b200 ABI version %d, this program was built for %d\n", p2r_abi_version(),
                 P2R_ABI_VERSION);
    return 1;
  }
  if (a.bsize < 1|| a.ntrks < a.bsize || a.nevts < 1 || a.nlayer < 1 || a.niter < 1) {
    std::fprintf(stderr, "bad sizes\n");
    return 1;
  }
  const long nb = a.ntrks / a.bsize;  // the reference drops ntrks % bsize tracks (TBB:22)
  p2r_config cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.bsize = a.bsize;
  cfg.nlayer = a.nlayer;
  cfg.nevts = a.nevts;
  cfg.nb = nb;
  cfg.bz = a.bz;
  cfg.mode = a.chained ? P2R_MODE_CHAINED : P2R_MODE_RESTART;

  const size_t trk_words = (size_t)a.nevts * nb * 28 * a.bsize;
  const size_t hit_words = (size_t)a.nevts * nb * a.nlayer * 9 * a.bsize;
  std::vector<float> trk(trk_words), hit(hit_words), out(trk_words);
  float last_hit[3] = {0, 0, 0};

  std::printf("produce nevts=%ld ntrks=%ld bsize=%d nlayer=%d input=%s mode=%s\n", a.nevts, a.ntrks, a.bsize,
              a.nlayer, a.input.c_str(), a.chained ? "chained" : "restart");
  std::printf("NITER=%d\n", a.niter);
  auto setup_start = std::chrono::steady_clock::now();
  if (a.input == "fixture") {
    std::ifstream f(a.fixture);
    std::vector<float> v;
    float x;
    while (f >> x) v.push_back(x);
    if (v.size() < 28 + 9 || (v.size() - 28) % 9 != 0) {
      std::fprintf(stderr, "fixture file %s: expected 6+21+1 then n x 9 numbers\n", a.fixture.c_str());
      return 1;
    }
    const int nhits = (int)((v.size() - 28) / 9);
    // the input echo of the reference's main (TBB:822-830); cov is packed lower-triangular
    std::printf("track in pos: x=%f, y=%f, z=%f, r=%f, pt=%f, phi=%f, theta=%f \n", v[0], v[1], v[2],
                std::sqrt(v[0] * v[0] + v[1] * v[1]), 1. / v[3], v[4], v[5]);
    std::printf("track in cov: xx=%.2e, yy=%.2e, zz=%.2e \n", v[6 + 0], v[6 + 2], v[6 + 5]);
    for (int lay = 0; lay < a.nlayer && lay < nhits; ++lay) {
      const float* h = v.data() + 28 + 9 * lay;
      std::printf("hit in layer=%d, pos: x=%f, y=%f, z=%f, r=%f \n", lay, h[0], h[1], h[2],
                  std::sqrt(h[0] * h[0] + h[1] * h[1]));
    }
    srand(1);  // glibc's default seed: the sequence a fresh run of the reference sees
    CK(p2r_gen_fixture(v.data(), v.data() + 6, (int32_t)v[27], v.data() + 28, nhits, a.bsize, a.nevts, nb, a.nlayer,
                       1e-5, trk.data(), hit.data()));
    for (int i = 0; i < 3; ++i) last_hit[i] = v[28 + 9 * (a.nlayer - 1) + i];
  } else {
    p2r_gen_params gp;
    p2r_gen_params_default(&gp);
    gp.bz = a.bz;
    CK(p2r_gen_helix(&gp, a.bsize, a.nevts, nb, a.nlayer, nullptr, trk.data(), hit.data(), 0));
    // unsmeared last-layer position of track 0 (the summary's reference point, TBB:948-951)
    for (int i = 0; i < 3; ++i) last_hit[i] = hit[((size_t)(a.nlayer - 1) * 9 + i) * a.bsize];
  }
  void *d_trk = nullptr, *d_hit = nullptr, *d_out = nullptr;
  CU(cudaMalloc(&d_trk, trk_words * 4));
  CU(cudaMalloc(&d_hit, hit_words * 4));
  CU(cudaMalloc(&d_out, trk_words * 4));
  if (a.transfer) {
    CU(cudaHostRegister(trk.data(), trk_words * 4, cudaHostRegisterDefault));
    CU(cudaHostRegister(hit.data(), hit_words * 4, cudaHostRegisterDefault));
    CU(cudaHostRegister(out.data(), trk_words * 4, cudaHostRegisterDefault));
  } else {
    CU(cudaMemcpy(d_trk, trk.data(), trk_words * 4, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d_hit, hit.data(), hit_words * 4, cudaMemcpyHostToDevice));
  }
  cudaStream_t st;
  CU(cudaStreamCreate(&st));
  // one untimed pass (module loading, first-touch)
  if (a.transfer)
    CK(p2r_forward_host(&cfg, trk.data(), hit.data(), out.data(), d_trk, d_hit, d_out, 10, st));
  else
    CK(p2r_forward(&cfg, d_trk, d_hit, d_out, nullptr, nullptr, st));
  CU(cudaStreamSynchronize(st));
  auto setup_stop = std::chrono::steady_clock::now();
  std::printf("done preparing!\n");

  auto wall_start = std::chrono::steady_clock::now();
  for (int itr = 0; itr < a.niter; ++itr) {
    if (a.transfer)
      CK(p2r_forward_host(&cfg, trk.data(), hit.data(), out.data(), d_trk, d_hit, d_out, 10, st));
    else
      CK(p2r_forward(&cfg, d_trk, d_hit, d_out, nullptr, nullptr, st));
  }
  CU(cudaStreamSynchronize(st));
  auto wall_stop = std::chrono::steady_clock::now();
  const double wall_time = std::chrono::duration<double>(wall_stop - wall_start).count();
  const double setup_time = std::chrono::duration<double>(setup_stop - setup_start).count();
  const long ntracks = a.nevts * a.ntrks * a.niter;
  // the lines the reference prints (TBB:931-933); build.py:83 parses the second
  std::printf("setup time time=%f (s)\n", setup_time);
  std::printf("done ntracks=%ld tot time=%f (s) time/trk=%e (s)\n", ntracks, wall_time, wall_time / ntracks);
  std::printf("formatted %d %ld %ld %d %ld %f 0 %f %d\n", a.niter, a.nevts, a.ntrks, a.bsize, nb, wall_time, setup_time,
              1);
  // restart: only the last layer reaches the output and only that one is computed
  std::printf("track-layer updates/s=%e\n", (double)ntracks * (a.chained ? a.nlayer : 1) / wall_time);

  if (!a.transfer) CU(cudaMemcpy(out.data(), d_out, trk_words * 4, cudaMemcpyDeviceToHost));
  p2r_summary_stats s;
  CK(p2r_summary(out.data(), a.bsize, a.nevts, nb, last_hit, &s));
  // the validation printout (TBB:1036-1048)
  std::printf("track x avg=%f std/avg=%f\n", s.avg_x, std::fabs(s.std_x / s.avg_x));
  std::printf("track y avg=%f std/avg=%f\n", s.avg_y, std::fabs(s.std_y / s.avg_y));
  std::printf("track z avg=%f std/avg=%f\n", s.avg_z, std::fabs(s.std_z / s.avg_z));
  std::printf("track r avg=%f std/avg=%f\n", s.avg_r, std::fabs(s.std_r / s.avg_z));
  std::printf("track dx/x avg=%f std=%f\n", s.avg_dx, s.std_dx);
  std::printf("track dy/y avg=%f std=%f\n", s.avg_dy, s.std_dy);
  std::printf("track dz/z avg=%f std=%f\n", s.avg_dz, s.std_dz);
  std::printf("track dr/r avg=%f std=%f\n", s.avg_dr, s.std_dr);
  std::printf("track pt avg=%f\n", s.avg_pt);
  std::printf("track phi avg=%f\n", s.avg_phi);
  std::printf("track theta avg=%f\n", s.avg_theta);
  std::printf("number of tracks with nans=%ld\n", (long)s.nnans);
  std::printf("number of tracks failed=%ld\n", (long)s.nfail);

  if (a.transfer) {
    cudaHostUnregister(trk.data());
    cudaHostUnregister(hit.data());
    cudaHostUnregister(out.data());
  }
  cudaFree(d_trk);
  cudaFree(d_hit);
  cudaFree(d_out);
  cudaStreamDestroy(st);
  return 0;
}
