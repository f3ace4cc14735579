// The reference's two 3x3 gain routines, KalmanGainInv and KalmanGain
// (src/propagate-tor-test_tbb.cpp:376-426). The reference defines them but never calls them:
// its KalmanUpdate measures two coordinates and inverts a 2x2 (TBB:433-642). They are shipped
// here as stand-alone entry points with the reference's own element choice, so a caller that
// used them gets the same numbers.
//
// Element choice, as the reference indexes the packed arrays (it reads them as if they were
// packed upper-triangle row-major, while the arrays are packed lower-triangle, TBB:46-54):
//   M = A + B with A = track covariance words a[.], B = hit covariance words b[.]:
//       M = [[a0+b0, a1+b1, a2+b2], [a1+b1, a6+b3, a7+b4], [a2+b2, a7+b4, a11+b5]]
//   inv = adj(M) / det(M) with det and 1/det in double (TBB:383-388), written row-major to an
//   MP3x3 block (9 rows of bsize lanes);
//   gain (MP3x6, 18 rows) = rows r of the 6x6 covariance read with the same convention,
//       row r = (a[r], a[.], a[.]) from the upper-packed positions (r,0), (r,1), (r,2),
//   times inv (TBB:407-426).
// Arithmetic: every float operation is rounded as written (no contraction), as the
// reference's source states it; its -ffast-math build may fuse some of them.
#include <cuda_runtime.h>

#include "p2r_internal.h"

namespace {

// upper-triangle row-major packing of a symmetric 6x6, the index the reference's gain routine
// reads for element (r, c) (r, c in 0..5)
__host__ __device__ constexpr int upper6(int r, int c) {
  return r <= c ? r * 6 - r * (r - 1) / 2 + (c - r) : c * 6 - c * (c - 1) / 2 + (r - c);
}

__global__ void gain_inv_kernel(const float* __restrict__ trk, const float* __restrict__ hits, int layer,
                                int nlayer, long long nblocks, int bsize, float* __restrict__ inv) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nblocks * bsize) return;
  const long long b = t / bsize;
  const int it = (int)(t - b * bsize);
  const float* a = trk + b * 28LL * bsize + 6LL * bsize + it;                       // covariance rows
  const float* h = hits + ((long long)layer + b * nlayer) * 9LL * bsize + 3LL * bsize + it;  // hit cov
  auto A = [&](int k) { return a[(long long)k * bsize]; };
  auto B = [&](int k) { return h[(long long)k * bsize]; };
  const float m00 = __fadd_rn(A(0), B(0)), m01 = __fadd_rn(A(1), B(1)), m02 = __fadd_rn(A(2), B(2));
  const float m11 = __fadd_rn(A(6), B(3)), m12 = __fadd_rn(A(7), B(4)), m22 = __fadd_rn(A(11), B(5));
  // cofactors, each the float difference of two float products (TBB:384-386, 390-398)
  auto cof = [](float p, float q, float r, float s) { return __fsub_rn(__fmul_rn(p, q), __fmul_rn(r, s)); };
  const float c00 = cof(m11, m22, m12, m12);
  const float c01 = cof(m01, m22, m12, m02);  // the (0,1) minor as TBB:384 writes it
  const float c02 = cof(m01, m12, m02, m11);
  const float det_f = __fadd_rn(__fsub_rn(__fmul_rn(m00, c00), __fmul_rn(m01, c01)), __fmul_rn(m02, c02));
  const double invdet = 1.0 / (double)det_f;
  float* o = inv + b * 9LL * bsize + it;
  o[0LL * bsize] = (float)(invdet * cof(m11, m22, m12, m12));
  o[1LL * bsize] = (float)(-1 * invdet * cof(m01, m22, m02, m12));
  o[2LL * bsize] = (float)(invdet * cof(m01, m12, m02, m12));
  o[3LL * bsize] = (float)(-1 * invdet * cof(m01, m22, m12, m02));
  o[4LL * bsize] = (float)(invdet * cof(m00, m22, m02, m02));
  o[5LL * bsize] = (float)(-1 * invdet * cof(m00, m12, m02, m01));
  o[6LL * bsize] = (float)(invdet * cof(m01, m12, m02, m11));
  o[7LL * bsize] = (float)(-1 * invdet * cof(m00, m12, m02, m01));
  o[8LL * bsize] = (float)(invdet * cof(m00, m11, m01, m01));
}

__global__ void gain_kernel(const float* __restrict__ trk, const float* __restrict__ inv, long long nblocks,
                            int bsize, float* __restrict__ gain) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nblocks * bsize) return;
  const long long b = t / bsize;
  const int it = (int)(t - b * bsize);
  const float* a = trk + b * 28LL * bsize + 6LL * bsize + it;
  const float* m = inv + b * 9LL * bsize + it;
  float* g = gain + b * 18LL * bsize + it;
  float w[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) w[k] = m[(long long)k * bsize];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const float x0 = a[(long long)upper6(r, 0) * bsize], x1 = a[(long long)upper6(r, 1) * bsize],
                x2 = a[(long long)upper6(r, 2) * bsize];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      g[(long long)(3 * r + c) * bsize] =
          __fadd_rn(__fadd_rn(__fmul_rn(x0, w[c]), __fmul_rn(x1, w[3 + c])), __fmul_rn(x2, w[6 + c]));
  }
}

int check_gain_args(const p2r_config* cfg, const char* who, long long* nblocks) {
  int rc = p2r_check_config(cfg, who);
  if (rc) return rc;
  *nblocks = (long long)cfg->nevts * cfg->nb;
  return P2R_OK;
}

}  // namespace

extern "C" {

int p2r_kalman_gain_inv(const p2r_config* cfg, const void* trk, const void* hits, int32_t layer, float* inv_out,
                        void* stream) {
  const char* who = "p2r_kalman_gain_inv";
  P2rRange range(who);
  long long nblocks = 0;
  int rc = check_gain_args(cfg, who, &nblocks);
  if (rc) return rc;
  if (layer < 0 || layer >= cfg->nlayer) return p2r_set_errorf(P2R_ERR_INVALID, "%s: layer %d", who, layer);
  if (nblocks == 0) return p2r_clear_error();
  if (!trk || !hits || !inv_out) return p2r_set_errorf(P2R_ERR_INVALID, "%s: null array pointer", who);
  if ((rc = p2r_check_aligned(who, 4, {trk, hits, inv_out}))) return rc;
  const size_t tb = (size_t)nblocks * 28 * cfg->bsize * sizeof(float);
  const size_t hb = (size_t)nblocks * cfg->nlayer * 9 * cfg->bsize * sizeof(float);
  const size_t ib = (size_t)nblocks * 9 * cfg->bsize * sizeof(float);
  if ((rc = p2r_check_spans(who, {{"trk", trk, tb, false}, {"hits", hits, hb, false}, {"inv_out", inv_out, ib, true}})))
    return rc;
  const long long n = nblocks * cfg->bsize;
  gain_inv_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      (const float*)trk, (const float*)hits, layer, cfg->nlayer, nblocks, cfg->bsize, inv_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: launch failed: %s", who, cudaGetErrorString(e));
  return p2r_clear_error();
}

int p2r_kalman_gain(const p2r_config* cfg, const void* trk, const float* inv, float* gain_out, void* stream) {
  const char* who = "p2r_kalman_gain";
  P2rRange range(who);
  long long nblocks = 0;
  int rc = check_gain_args(cfg, who, &nblocks);
  if (rc) return rc;
  if (nblocks == 0) return p2r_clear_error();
  if (!trk || !inv || !gain_out) return p2r_set_errorf(P2R_ERR_INVALID, "%s: null array pointer", who);
  if ((rc = p2r_check_aligned(who, 4, {trk, inv, gain_out}))) return rc;
  const size_t tb = (size_t)nblocks * 28 * cfg->bsize * sizeof(float);
  const size_t ib = (size_t)nblocks * 9 * cfg->bsize * sizeof(float);
  const size_t gb = (size_t)nblocks * 18 * cfg->bsize * sizeof(float);
  if ((rc = p2r_check_spans(who, {{"trk", trk, tb, false}, {"inv", inv, ib, false}, {"gain_out", gain_out, gb, true}})))
    return rc;
  const long long n = nblocks * cfg->bsize;
  gain_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>((const float*)trk, inv, nblocks,
                                                                              cfg->bsize, gain_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: launch failed: %s", who, cudaGetErrorString(e));
  return p2r_clear_error();
}

}  // extern "C"
