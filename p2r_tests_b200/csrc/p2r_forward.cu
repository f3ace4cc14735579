// C-ABI entry points of the forward path: the fused driver (p2r_forward, p2r_forward_masked)
// and the per-layer kernels that mirror the reference's call shape:
//  propagate_kernel  one propagateToR per track for one layer (TBB:894)
//  update_kernel     one KalmanUpdate per track for one layer (TBB:911)
#include <cuda_runtime.h>
#include <stdint.h>

#include "p2r_fwd.cuh"
#include "p2r_fwd_ordered.cuh"
#include "p2r_internal.h"

namespace p2r {

// ---------------------------------------------------------------- per-layer kernels
__global__ void __launch_bounds__(128) propagate_kernel(const float* trk_in, const float* hits, float* trk_out,
                                                        const float* dr, long long nblocks, int bs, int nlayer,
                                                        int layer, float kfact) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = g / bs;
  const int it = (int)(g - b * bs);
  if (b >= nblocks) return;
  // trk_in may alias trk_out: plain loads, all inputs read before any store.
  const float* blk = trk_in + b * (long long)(kTrkWords * bs);
  float par[6], cov[21];
#pragma unroll
  for (int i = 0; i < 6; ++i) par[i] = blk[i * bs + it];
#pragma unroll
  for (int i = 0; i < 21; ++i) cov[i] = blk[(6 + i) * bs + it];
  const float qf = blk[27 * bs + it];
  const float k = (float)__float_as_int(qf) * kfact;
  const float* h = hits + (b * nlayer + layer) * (long long)(kHitWords * bs);
  const float rh = hipo(h[it], h[bs + it]);
  const float rt = dr ? rh + dr[layer] : rh;
  float op[6], oc[21];
  propagate_to_r(par, cov, k, 1.f / k, rt, op, oc);
  float* ob = trk_out + b * (long long)(kTrkWords * bs);
#pragma unroll
  for (int i = 0; i < 6; ++i) ob[i * bs + it] = op[i];
#pragma unroll
  for (int i = 0; i < 21; ++i) ob[(6 + i) * bs + it] = oc[i];
  ob[27 * bs + it] = qf;
}

template <bool FP64DET>
__global__ void __launch_bounds__(128) update_kernel(float* trk, const float* hits, float* chi2_accum, long long nblocks,
                                                     int bs, int nlayer, int layer, int squash) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = g / bs;
  const int it = (int)(g - b * bs);
  if (b >= nblocks) return;
  float* blk = trk + b * (long long)(kTrkWords * bs);
  float par[6], cov[21];
#pragma unroll
  for (int i = 0; i < 6; ++i) par[i] = blk[i * bs + it];
#pragma unroll
  for (int i = 0; i < 21; ++i) cov[i] = blk[(6 + i) * bs + it];
  const float* h = hits + (b * nlayer + layer) * (long long)(kHitWords * bs);
  float hp[3], hc[6];
#pragma unroll
  for (int i = 0; i < 3; ++i) hp[i] = h[i * bs + it];
#pragma unroll
  for (int i = 0; i < 6; ++i) hc[i] = h[(3 + i) * bs + it];
  const float rh = hipo(hp[0], hp[1]);
  float chi2;
  if (chi2_accum)
    chi2 = kalman_update<FP64DET, true>(par, cov, hp, hc, rh);
  else
    chi2 = kalman_update<FP64DET, false>(par, cov, hp, hc, rh);
  if (squash) par[4] = squash_phi(par[4]);
#pragma unroll
  for (int i = 0; i < 6; ++i) blk[i * bs + it] = par[i];
#pragma unroll
  for (int i = 0; i < 21; ++i) blk[(6 + i) * bs + it] = cov[i];
  if (chi2_accum) chi2_accum[b * bs + it] += chi2;
}

__global__ void count_nonfinite_kernel(const float* trk, long long nblocks, int bs, unsigned long long* count) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = g / bs;
  const int it = (int)(g - b * bs);
  bool bad = false;
  if (b < nblocks) {
    const float* blk = trk + b * (long long)(kTrkWords * bs);
#pragma unroll
    for (int i = 0; i < 6; ++i) bad |= !isfinite(blk[i * bs + it]);
  }
  const unsigned m = __ballot_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
}

}  // namespace p2r


using namespace p2r;

static int check_ptr16(const void* ptr) { return ((uintptr_t)ptr & 15u) == 0; }

static int forward_impl(const p2r_config* cfg, const void* trk_in, const void* hits, void* trk_out,
                        const int32_t* nlay, float* chi2_out, const float* dr, void* stream, const char* who) {
  P2rRange range(who);
  int rc = p2r_check_config(cfg, who);
  if (rc) return rc;
  const long long nblocks = (long long)cfg->nevts * cfg->nb;
  if (nblocks == 0) return p2r_clear_error();  // an empty batch is valid (pointers unused)
  if (!trk_in || !hits || !trk_out) return p2r_set_errorf(P2R_ERR_INVALID, "%s: null array pointer", who);
  if (trk_in == trk_out) return p2r_set_errorf(P2R_ERR_INVALID, "%s: trk_out may not alias trk_in", who);
  if ((rc = p2r_check_aligned(who, 4, {trk_in, hits, trk_out, chi2_out, dr, nlay}))) return rc;
  if (cfg->mode != P2R_MODE_RESTART && cfg->mode != P2R_MODE_CHAINED)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: unknown mode %d", who, cfg->mode);
  if (nlay && cfg->mode != P2R_MODE_CHAINED)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: per-lane layer counts need CHAINED mode", who);
  {
    const size_t tb = (size_t)nblocks * 28 * cfg->bsize * sizeof(float);
    const size_t hb = (size_t)nblocks * cfg->nlayer * 9 * cfg->bsize * sizeof(float);
    const size_t lb = (size_t)nblocks * cfg->bsize * sizeof(float);  // chi2 and layer counts
    if ((rc = p2r_check_disjoint(who, "trk_out and trk_in", trk_out, tb, trk_in, tb)) ||
        (rc = p2r_check_disjoint(who, "trk_out and hits", trk_out, tb, hits, hb)) ||
        (rc = p2r_check_disjoint(who, "trk_out and nlay_lane", trk_out, tb, nlay, lb)) ||
        (rc = p2r_check_disjoint(who, "trk_out and dr", trk_out, tb, dr, cfg->nlayer * sizeof(float))) ||
        (rc = p2r_check_disjoint(who, "chi2_out and trk_out", chi2_out, lb, trk_out, tb)) ||
        (rc = p2r_check_disjoint(who, "chi2_out and trk_in", chi2_out, lb, trk_in, tb)) ||
        (rc = p2r_check_disjoint(who, "chi2_out and hits", chi2_out, lb, hits, hb)) ||
        (rc = p2r_check_disjoint(who, "chi2_out and nlay_lane", chi2_out, lb, nlay, lb)) ||
        (rc = p2r_check_disjoint(who, "chi2_out and dr", chi2_out, lb, dr, cfg->nlayer * sizeof(float))))
      return rc;
  }
  FwdParams p;
  p.trk_in = (const float*)trk_in;
  p.hits = (const float*)hits;
  p.trk_out = (float*)trk_out;
  p.chi2 = chi2_out;
  p.dr = dr;
  p.nlay = nlay;
  p.nblocks = nblocks;
  p.bsize = cfg->bsize;
  p.nlayer = cfg->nlayer;
  p.kfact = p2r_kfact_of(cfg->bz);
  p.squash = (cfg->flags & P2R_FLAG_SQUASH_PHI) != 0;
  const int threads = cfg->block_threads > 0 ? cfg->block_threads : 128;
  if (threads % 32 || threads > 128)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: block_threads must be a multiple of 32 up to 128", who);
  const int stages = cfg->stages > 0 ? cfg->stages : 4;
  if (stages != 2 && stages != 4) return p2r_set_errorf(P2R_ERR_INVALID, "%s: stages must be 2 or 4", who);
  const bool staged = !(cfg->flags & P2R_FLAG_NO_STAGING) && cfg->bsize % 32 == 0 && check_ptr16(hits);
  const bool fp64det = !(cfg->flags & P2R_FLAG_FP32_DET);
  if (p.squash && !fp64det)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: P2R_FLAG_SQUASH_PHI is built with the FP64 determinant only", who);
  // ordering by layer count matters only with per-track layer counts (chained)
  const bool ordered = nlay && (cfg->flags & P2R_FLAG_ORDER_BY_LAYERS);
  if (ordered && (!fp64det || cfg->nlayer > kOrdMaxKeys - 1 ||
                  cfg->bsize > (threads == 128 ? 2 * 128 : 2 * 256) || cfg->bsize % 32 != 0))
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED,
                          "%s: P2R_FLAG_ORDER_BY_LAYERS needs the FP64 determinant, nlayer <= %d, a bsize that is a "
                          "multiple of 32 and at most 2 x the CTA size (block_threads 128: 4 warps, else 8)",
                          who, kOrdMaxKeys - 1);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (cfg->mode == P2R_MODE_RESTART)
    e = launch_restart(p, fp64det, threads, stages, st);
  else if (ordered)
    e = launch_ordered(p, fp64det, threads, st);
  else if (nlay)
    e = launch_masked(p, staged, fp64det, threads, stages, st);
  else
    e = launch_chained(p, staged, fp64det, threads, stages, st);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: launch failed: %s", who, cudaGetErrorString(e));
  return p2r_clear_error();
}

extern "C" {

int p2r_forward(const p2r_config* cfg, const void* trk_in, const void* hits, void* trk_out, float* chi2_out,
                const float* dr, void* stream) {
  return forward_impl(cfg, trk_in, hits, trk_out, nullptr, chi2_out, dr, stream, "p2r_forward");
}

int p2r_forward_masked(const p2r_config* cfg, const void* trk_in, const void* hits, void* trk_out,
                       const int32_t* nlay_lane, float* chi2_out, const float* dr, void* stream) {
  if (!nlay_lane) return p2r_set_error(P2R_ERR_INVALID, "p2r_forward_masked: nlay_lane is null");
  return forward_impl(cfg, trk_in, hits, trk_out, nlay_lane, chi2_out, dr, stream, "p2r_forward_masked");
}

int p2r_propagate_to_r(const p2r_config* cfg, const void* trk_in, const void* hits, int32_t layer, void* trk_out,
                       const float* dr, void* stream) {
  P2rRange range("p2r_propagate_to_r");
  int rc = p2r_check_config(cfg, "p2r_propagate_to_r");
  if (rc) return rc;
  if (!trk_in || !hits || !trk_out) return p2r_set_error(P2R_ERR_INVALID, "p2r_propagate_to_r: null array pointer");
  if ((rc = p2r_check_aligned("p2r_propagate_to_r", 4, {trk_in, hits, trk_out, dr}))) return rc;
  if (layer < 0 || layer >= cfg->nlayer)
    return p2r_set_errorf(P2R_ERR_INVALID, "p2r_propagate_to_r: layer %d outside [0, %d)", layer, cfg->nlayer);
  const long long nblocks = (long long)cfg->nevts * cfg->nb;
  if (nblocks == 0) return p2r_clear_error();
  const size_t tb = (size_t)nblocks * 28 * cfg->bsize * sizeof(float);
  const size_t hb = (size_t)nblocks * cfg->nlayer * 9 * cfg->bsize * sizeof(float);
  if ((rc = p2r_check_disjoint("p2r_propagate_to_r", "trk_out and trk_in", trk_out, tb, trk_in, tb, true)) ||
      (rc = p2r_check_disjoint("p2r_propagate_to_r", "trk_out and hits", trk_out, tb, hits, hb)) ||
      (rc = p2r_check_disjoint("p2r_propagate_to_r", "trk_out and dr", trk_out, tb, dr, cfg->nlayer * sizeof(float))))
    return rc;
  const long long ntr = nblocks * cfg->bsize;
  const int threads = 128;
  propagate_kernel<<<(unsigned)((ntr + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(
      (const float*)trk_in, (const float*)hits, (float*)trk_out, dr, nblocks, cfg->bsize, cfg->nlayer, layer,
      p2r_kfact_of(cfg->bz));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_propagate_to_r: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}

int p2r_kalman_update(const p2r_config* cfg, void* trk, const void* hits, int32_t layer, float* chi2_accum,
                      void* stream) {
  P2rRange range("p2r_kalman_update");
  int rc = p2r_check_config(cfg, "p2r_kalman_update");
  if (rc) return rc;
  if (!trk || !hits) return p2r_set_error(P2R_ERR_INVALID, "p2r_kalman_update: null array pointer");
  if ((rc = p2r_check_aligned("p2r_kalman_update", 4, {trk, hits, chi2_accum}))) return rc;
  if (layer < 0 || layer >= cfg->nlayer)
    return p2r_set_errorf(P2R_ERR_INVALID, "p2r_kalman_update: layer %d outside [0, %d)", layer, cfg->nlayer);
  const long long nblocks = (long long)cfg->nevts * cfg->nb;
  if (nblocks == 0) return p2r_clear_error();
  const size_t tb = (size_t)nblocks * 28 * cfg->bsize * sizeof(float);
  const size_t hb = (size_t)nblocks * cfg->nlayer * 9 * cfg->bsize * sizeof(float);
  const size_t lb = (size_t)nblocks * cfg->bsize * sizeof(float);
  if ((rc = p2r_check_disjoint("p2r_kalman_update", "trk and hits", trk, tb, hits, hb)) ||
      (rc = p2r_check_disjoint("p2r_kalman_update", "chi2_accum and trk", chi2_accum, lb, trk, tb)) ||
      (rc = p2r_check_disjoint("p2r_kalman_update", "chi2_accum and hits", chi2_accum, lb, hits, hb)))
    return rc;
  const long long ntr = nblocks * cfg->bsize;
  const int threads = 128;
  const unsigned grid = (unsigned)((ntr + threads - 1) / threads);
  const int squash = (cfg->flags & P2R_FLAG_SQUASH_PHI) != 0;
  if (cfg->flags & P2R_FLAG_FP32_DET)
    update_kernel<false><<<grid, threads, 0, (cudaStream_t)stream>>>((float*)trk, (const float*)hits, chi2_accum,
                                                                      nblocks, cfg->bsize, cfg->nlayer, layer, squash);
  else
    update_kernel<true><<<grid, threads, 0, (cudaStream_t)stream>>>((float*)trk, (const float*)hits, chi2_accum,
                                                                     nblocks, cfg->bsize, cfg->nlayer, layer, squash);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_kalman_update: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}

int p2r_count_nonfinite(const void* trk, int64_t nblocks, int32_t bsize, unsigned long long* count_out, void* stream) {
  if (!trk || !count_out) return p2r_set_error(P2R_ERR_INVALID, "p2r_count_nonfinite: null pointer");
  if (nblocks < 0 || bsize < 1) return p2r_set_error(P2R_ERR_INVALID, "p2r_count_nonfinite: bad sizes");
  if (int rc = p2r_check_aligned("p2r_count_nonfinite", 4, {trk})) return rc;
  if (int rc = p2r_check_aligned("p2r_count_nonfinite", 8, {count_out})) return rc;
  if (nblocks == 0) return p2r_clear_error();
  const long long ntr = nblocks * (long long)bsize;
  const int threads = 256;
  count_nonfinite_kernel<<<(unsigned)((ntr + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(
      (const float*)trk, nblocks, bsize, count_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_count_nonfinite: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}

}  // extern "C"
