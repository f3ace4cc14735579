// FP32 FMA throughput probe: the measured denominator of the hot path's compute roofline.
// Each thread advances 8 independent FMA chains (enough independent work to cover the
// FMA latency at full occupancy) for `iters` iterations; the result is stored so nothing
// is eliminated. FLOPs per launch = 2 * 32 * iters * blocks * threads (8 chains, 4 rounds).
#include <cuda_runtime.h>

#include "p2r_internal.h"
#include "p2r_math.cuh"

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

// The same FLOPs with sm_100's packed f32x2 FMA (two lanes per instruction; 8 chains of two
// lanes, 2 unrolled rounds): the FP32 peak seen by code that issues the packed form.
__device__ __forceinline__ unsigned long long pack2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float sum2(unsigned long long r) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
  return a + b;
}
__global__ void __launch_bounds__(256) fma2_probe_kernel(long long iters, float* out) {
  unsigned long long a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = pack2(threadIdx.x * 1e-7f + i * 1e-7f, threadIdx.x * 1e-7f + i * 2e-7f);
  const unsigned long long m = pack2(0.999999f, 0.999999f), c = pack2(1e-7f, 1e-7f);
  for (long long it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int i = 0; i < 8; ++i) asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[i]) : "l"(m), "l"(c));
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += sum2(a[i]);
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP64 FMA throughput probe (the denominator of the FP64 adjoint's compute roofline): the FP32
// probe's structure in double, 8 independent chains x 4 unrolled rounds per iteration.
__global__ void __launch_bounds__(256) dfma_probe_kernel(long long iters, double* out) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
  double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
  const double m = 0.999999999, c = 1e-9;
  for (long long i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a0 = fma(a0, m, c);
      a1 = fma(a1, m, c);
      a2 = fma(a2, m, c);
      a3 = fma(a3, m, c);
      a4 = fma(a4, m, c);
      a5 = fma(a5, m, c);
      a6 = fma(a6, m, c);
      a7 = fma(a7, m, c);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

// The hot path's own division and square root (p2r::fdiv, p2r::fsqrt) over caller arrays,
// so their error against the correctly rounded results can be measured.
__global__ void math_check_kernel(long long n, const float* __restrict__ a, const float* __restrict__ b,
                                  float* __restrict__ quot, float* __restrict__ root) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    quot[i] = p2r::fdiv(a[i], b[i]);
    root[i] = p2r::fsqrt(a[i]);
  }
}

}  // namespace

extern "C" int p2r_fp32x2_fma_probe(int64_t iters, int32_t blocks, int32_t threads, float* out, void* stream) {
  if (!out || iters < 1 || blocks < 1 || threads < 32 || threads > 256 || threads % 32)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_fp32x2_fma_probe: bad arguments");
  if (int rc = p2r_check_aligned("p2r_fp32x2_fma_probe", 4, {out})) return rc;
  fma2_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_fp32x2_fma_probe: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}

extern "C" int32_t p2r_math_variant(void) {
#if defined(P2R_FAST_MATH)
  return P2R_MATH_FAST;
#elif defined(P2R_IEEE_MATH)
  return P2R_MATH_IEEE;
#else
  return P2R_MATH_REFINED;
#endif
}

extern "C" int p2r_math_check(int64_t n, const float* a, const float* b, float* quot, float* root, void* stream) {
  if (n < 0 || (n > 0 && (!a || !b || !quot || !root)))
    return p2r_set_error(P2R_ERR_INVALID, "p2r_math_check: bad arguments");
  if (int rc = p2r_check_aligned("p2r_math_check", 4, {a, b, quot, root})) return rc;
  if (n == 0) return p2r_clear_error();
  const long long blocks = (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16;
  math_check_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(n, a, b, quot, root);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_math_check: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}

// FLOPs per launch = 2 * 32 * iters * blocks * threads (4 unrolled rounds of 8 chains).
extern "C" int p2r_fp32_fma_probe(int64_t iters, int32_t blocks, int32_t threads, float* out, void* stream) {
  if (!out || iters < 1 || blocks < 1 || threads < 32 || threads > 256 || threads % 32)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_fp32_fma_probe: bad arguments");
  if (int rc = p2r_check_aligned("p2r_fp32_fma_probe", 4, {out})) return rc;
  fma_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_fp32_fma_probe: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}

// FLOPs per launch = 2 * 32 * iters * blocks * threads, in FP64.
extern "C" int p2r_fp64_fma_probe(int64_t iters, int32_t blocks, int32_t threads, double* out, void* stream) {
  if (!out || iters < 1 || blocks < 1 || threads < 32 || threads > 256 || threads % 32)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_fp64_fma_probe: bad arguments");
  if (int rc = p2r_check_aligned("p2r_fp64_fma_probe", 8, {out})) return rc;
  dfma_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_fp64_fma_probe: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}
