// FP32 FMA throughput probe: the measured denominator of the hot path's compute roofline.
// Each thread advances 8 independent FMA chains (enough independent work to cover the
// FMA latency at full occupancy) for `iters` iterations; the result is stored so nothing
// is eliminated. FLOPs per launch = 2 * 8 * iters * blocks * threads.
#include <cuda_runtime.h>

#include "p2r_internal.h"

namespace {

__global__ void __launch_bounds__(256) fma_probe_kernel(long long iters, float* out) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
  float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
  const float m = 0.999999f, c = 1e-7f;
  for (long long i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a0 = fmaf(a0, m, c);
      a1 = fmaf(a1, m, c);
      a2 = fmaf(a2, m, c);
      a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c);
      a5 = fmaf(a5, m, c);
      a6 = fmaf(a6, m, c);
      a7 = fmaf(a7, m, c);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

}  // namespace

// FLOPs per launch = 2 * 32 * iters * blocks * threads (4 unrolled rounds of 8 chains).
extern "C" int p2r_fp32_fma_probe(int64_t iters, int32_t blocks, int32_t threads, float* out, void* stream) {
  if (!out || iters < 1 || blocks < 1 || threads < 32 || threads > 256 || threads % 32)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_fp32_fma_probe: bad arguments");
  fma_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_fp32_fma_probe: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}
