// Fused forward + adjoint of the chained layer loop (sm_100a), and its C-ABI entry points.
//
// One thread per track. The forward pass is the production chained forward
// (p2r_math.cuh); it stores the track state every CK layers (thread-local checkpoints).
// The reverse sweep walks the segments backwards: it recomputes the states inside a
// segment from its checkpoint, then for each layer, last to first, recomputes that layer
// with the tape of p2r_adjoint.cuh and runs the hand-written reverse of the update and
// of the propagation. Gradients produced:
//   per track  d/d(initial par, cov), d/d(hit pos, hit cov) for every layer
//   shared     d/d(dr[layer]) and d/d(Bz), summed over tracks, and optionally per event
// of L = sum_tracks (g_par . par_final + g_cov . cov_final + g_chi2 * chi2_total).
// Shared sums: each warp reduces with shuffles (fixed order) into per-warp partials in
// the workspace; a second kernel adds the partials in a fixed order in double, so the
// results are deterministic run to run.
#include <cuda_runtime.h>
#include <stdint.h>

#include "p2r_adjoint.cuh"
#include "p2r_internal.h"
#include "p2r_math.cuh"

namespace p2r {

constexpr int kMaxAdjLayers = 64;
constexpr int kAdjThreads = 128;

struct AdjParams {
  const float* trk_in;
  const float* hits;
  const float* dr;          // nullable, nlayer
  const int32_t* nlay;      // nullable, per-track layer counts
  float* trk_out;           // nullable
  float* chi2_out;          // nullable
  const float* g_trk_out;   // nullable, Matriplex cotangent of trk_out (par and cov rows)
  const float* g_chi2;      // nullable, per-track cotangent of the summed chi2
  float* g_trk_in;          // nullable, Matriplex
  float* g_hits;            // nullable, Matriplex
  float* partials;          // [nwarps][nlayer + 1]
  long long nblocks;
  int bsize;
  int nlayer;
  float kfact;
  float bz;
};

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int CK>
__global__ void __launch_bounds__(kAdjThreads) fwdbwd_kernel(AdjParams p) {
  constexpr int NCK = (kMaxAdjLayers + CK - 1) / CK;
  const int bs = p.bsize;
  const int lane = threadIdx.x & 31;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = g / bs;
  const int it = (int)(g - b * bs);
  const bool valid = b < p.nblocks;
  const long long gwarp = g >> 5;
  float* wpart = p.partials + gwarp * (p.nlayer + 1);

  float par[6] = {0, 0, 0, 1, 0, 1}, cov[21] = {};
  int q = 1;
  int nl = 0;
  const float* tb = p.trk_in + b * (long long)(28 * bs);
  if (valid) {
#pragma unroll
    for (int i = 0; i < 6; ++i) par[i] = tb[i * bs + it];
#pragma unroll
    for (int i = 0; i < 21; ++i) cov[i] = tb[(6 + i) * bs + it];
    q = __float_as_int(tb[27 * bs + it]);
    nl = p.nlay ? min(p.nlayer, max(0, p.nlay[b * bs + it])) : p.nlayer;
  }
  const float k = (float)q * p.kfact;
  const float kinv = 1.f / k;
  int nl_warp = nl;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nl_warp = max(nl_warp, __shfl_xor_sync(0xffffffffu, nl_warp, o));
  const float* hblk = p.hits + b * (long long)p.nlayer * (9 * bs);

  // ---- forward pass with checkpoints every CK layers
  float ck[NCK][27];
  float chi2 = 0.f;
  for (int l = 0; l < nl; ++l) {
    if (l % CK == 0) {
#pragma unroll
      for (int i = 0; i < 6; ++i) ck[l / CK][i] = par[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) ck[l / CK][6 + i] = cov[i];
    }
    const float* h = hblk + (long long)l * (9 * bs);
    float hp[3], hc[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) hp[i] = h[i * bs + it];
#pragma unroll
    for (int i = 0; i < 6; ++i) hc[i] = h[(3 + i) * bs + it];
    const float rh = hipo(hp[0], hp[1]);
    const float rt = p.dr ? rh + p.dr[l] : rh;
    propagate_to_r(par, cov, k, kinv, rt, par, cov);
    chi2 += kalman_update<true, true>(par, cov, hp, hc, rh);
  }
  if (valid) {
    if (p.trk_out) {
      float* ob = p.trk_out + b * (long long)(28 * bs);
#pragma unroll
      for (int i = 0; i < 6; ++i) ob[i * bs + it] = par[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) ob[(6 + i) * bs + it] = cov[i];
      ob[27 * bs + it] = __int_as_float(q);
    }
    if (p.chi2_out) p.chi2_out[b * bs + it] = chi2;
  }

  // ---- reverse sweep
  float pb[6] = {}, cb[21] = {};
  float chi2b = 0.f;
  if (valid) {
    if (p.g_trk_out) {
      const float* gb = p.g_trk_out + b * (long long)(28 * bs);
#pragma unroll
      for (int i = 0; i < 6; ++i) pb[i] = gb[i * bs + it];
#pragma unroll
      for (int i = 0; i < 21; ++i) cb[i] = gb[(6 + i) * bs + it];
    }
    if (p.g_chi2) chi2b = p.g_chi2[b * bs + it];
  }
  float kbar = 0.f, kinvbar = 0.f;
  const int nseg = (nl_warp + CK - 1) / CK;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int a = seg * CK;
    const int e = min(a + CK, nl_warp);
    // states before layers a .. e-1 of this segment, recomputed from the checkpoint
    float st[CK][27];
    if (a < nl) {
#pragma unroll
      for (int i = 0; i < 27; ++i) st[0][i] = ck[seg][i];
    }
    for (int l = a + 1; l < e && l < nl; ++l) {
      float sp[6], sc[21];
#pragma unroll
      for (int i = 0; i < 6; ++i) sp[i] = st[l - 1 - a][i];
#pragma unroll
      for (int i = 0; i < 21; ++i) sc[i] = st[l - 1 - a][6 + i];
      const float* h = hblk + (long long)(l - 1) * (9 * bs);
      float hp[3], hc[6];
#pragma unroll
      for (int i = 0; i < 3; ++i) hp[i] = h[i * bs + it];
#pragma unroll
      for (int i = 0; i < 6; ++i) hc[i] = h[(3 + i) * bs + it];
      const float rh = hipo(hp[0], hp[1]);
      const float rt = p.dr ? rh + p.dr[l - 1] : rh;
      propagate_to_r(sp, sc, k, kinv, rt, sp, sc);
      kalman_update<true, false>(sp, sc, hp, hc, rh);
#pragma unroll
      for (int i = 0; i < 6; ++i) st[l - a][i] = sp[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) st[l - a][6 + i] = sc[i];
    }
    for (int l = e - 1; l >= a; --l) {
      float drb = 0.f;
      if (l < nl) {
        float sp[6], sc[21];
#pragma unroll
        for (int i = 0; i < 6; ++i) sp[i] = st[l - a][i];
#pragma unroll
        for (int i = 0; i < 21; ++i) sc[i] = st[l - a][6 + i];
        const float* h = hblk + (long long)l * (9 * bs);
        float hp[3], hc[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) hp[i] = h[i * bs + it];
#pragma unroll
        for (int i = 0; i < 6; ++i) hc[i] = h[(3 + i) * bs + it];
        const float drl = p.dr ? p.dr[l] : 0.f;
        float hpb[3], hcb[6];
        adj::layer_rev(sp, sc, k, kinv, hp, hc, drl, pb, cb, chi2b, hpb, hcb, drb, kbar, kinvbar);
        if (p.g_hits) {
          float* gh = p.g_hits + (b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
          for (int i = 0; i < 3; ++i) gh[i * bs + it] = hpb[i];
#pragma unroll
          for (int i = 0; i < 6; ++i) gh[(3 + i) * bs + it] = hcb[i];
        }
      } else if (valid && p.g_hits) {
        float* gh = p.g_hits + (b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
        for (int i = 0; i < 9; ++i) gh[i * bs + it] = 0.f;
      }
      drb = warp_sum(drb);
      if (lane == 0) wpart[l] = drb;
    }
  }
  // layers the whole warp skipped have zero gradient
  if (lane == 0)
    for (int l = nl_warp; l < p.nlayer; ++l) wpart[l] = 0.f;
  if (valid && p.g_hits)
    for (int l = nl_warp; l < p.nlayer; ++l) {
      float* gh = p.g_hits + (b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
      for (int i = 0; i < 9; ++i) gh[i * bs + it] = 0.f;
    }
  // k = q * kfact(Bz): dk/dBz = -k / Bz
  float bzb = valid ? (kbar - kinvbar * kinv * kinv) * (-k / p.bz) : 0.f;
  bzb = warp_sum(bzb);
  if (lane == 0) wpart[p.nlayer] = bzb;
  if (valid && p.g_trk_in) {
    float* gb = p.g_trk_in + b * (long long)(28 * bs);
#pragma unroll
    for (int i = 0; i < 6; ++i) gb[i * bs + it] = pb[i];
#pragma unroll
    for (int i = 0; i < 21; ++i) gb[(6 + i) * bs + it] = cb[i];
    gb[27 * bs + it] = 0.f;
  }
}

// Sums per-warp partials [nwarps][nout] in a fixed order, in double. Block (e, j) sums
// warps [e*wpe, min((e+1)*wpe, nwarps)) of column j into out[e*nout + j].
__global__ void __launch_bounds__(256) sum_partials_kernel(const float* partials, long long nwarps, int nout,
                                                           long long wpe, double* out) {
  __shared__ double red[256];
  const long long e = blockIdx.x;
  const int j = blockIdx.y;
  const long long w0 = e * wpe, w1 = min(w0 + wpe, nwarps);
  double s = 0.0;
  for (long long w = w0 + threadIdx.x; w < w1; w += blockDim.x) s += (double)partials[w * nout + j];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[e * nout + j] = red[0];
}

// out[j] = sum over rows of in[rows][nout], fixed order.
__global__ void sum_rows_kernel(const double* in, long long rows, int nout, double* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nout) return;
  double s = 0.0;
  for (long long r = 0; r < rows; ++r) s += in[r * nout + j];
  out[j] = s;
}

__global__ void split_kernel(const double* src, long long rows, int nlayer, double* g_dr, double* g_bz) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * (nlayer + 1)) return;
  const long long r = i / (nlayer + 1);
  const int j = (int)(i - r * (nlayer + 1));
  if (j < nlayer) {
    if (g_dr) g_dr[r * nlayer + j] = src[i];
  } else if (g_bz) {
    g_bz[r] = src[i];
  }
}

}  // namespace p2r

using namespace p2r;

namespace {

// workspace: float partials[nwarps][nlayer+1], then (8-byte aligned) double
// event_sums[nevts][nlayer+1] and double totals[nlayer+1]
struct WsLayout {
  long long nwarps;
  size_t partial_bytes, event_off, total_off, total_bytes;
};

WsLayout layout_of(const p2r_config* cfg) {
  WsLayout w;
  const long long ntr = (long long)cfg->nevts * cfg->nb * cfg->bsize;
  const long long nthreads = (ntr + kAdjThreads - 1) / kAdjThreads * kAdjThreads;
  w.nwarps = nthreads / 32;
  w.partial_bytes = (size_t)w.nwarps * (cfg->nlayer + 1) * sizeof(float);
  w.event_off = (w.partial_bytes + 255) & ~(size_t)255;
  w.total_off = w.event_off + (((size_t)cfg->nevts * (cfg->nlayer + 1) * sizeof(double) + 255) & ~(size_t)255);
  w.total_bytes = w.total_off + (size_t)(cfg->nlayer + 1) * sizeof(double);
  return w;
}

template <int CK>
cudaError_t launch_fwdbwd(const AdjParams& p, long long ntr, cudaStream_t st) {
  const long long grid = (ntr + kAdjThreads - 1) / kAdjThreads;
  fwdbwd_kernel<CK><<<(unsigned)grid, kAdjThreads, 0, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

extern "C" {

size_t p2r_forward_backward_workspace_size(const p2r_config* cfg) {
  if (p2r_check_config(cfg, "p2r_forward_backward_workspace_size")) return 0;
  return layout_of(cfg).total_bytes;
}

int p2r_forward_backward(const p2r_config* cfg, const void* trk_in, const void* hits, const float* dr,
                         const int32_t* nlay_lane, void* trk_out, float* chi2_out, const void* grad_trk_out,
                         const float* grad_chi2, void* grad_trk_in, void* grad_hits, double* grad_dr, double* grad_bz,
                         double* grad_dr_event, double* grad_bz_event, int32_t ckpt_stride, void* workspace,
                         size_t workspace_bytes, void* stream) {
  const char* who = "p2r_forward_backward";
  int rc = p2r_check_config(cfg, who);
  if (rc) return rc;
  if (cfg->mode != P2R_MODE_CHAINED) return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: only CHAINED mode has an adjoint", who);
  if (cfg->nlayer > kMaxAdjLayers)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: nlayer %d exceeds %d", who, cfg->nlayer, kMaxAdjLayers);
  const long long nblocks = (long long)cfg->nevts * cfg->nb;
  if (nblocks == 0) return p2r_clear_error();
  if (!trk_in || !hits) return p2r_set_errorf(P2R_ERR_INVALID, "%s: null input array", who);
  if ((grad_dr_event || grad_bz_event) && cfg->bsize % 32 != 0)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: per-event gradients need bsize %% 32 == 0", who);
  const WsLayout w = layout_of(cfg);
  if (!workspace || workspace_bytes < w.total_bytes)
    return p2r_set_errorf(P2R_ERR_WORKSPACE, "%s: workspace of %zu bytes needed", who, w.total_bytes);
  if (((uintptr_t)workspace & 255u) != 0) return p2r_set_errorf(P2R_ERR_INVALID, "%s: workspace must be 256-byte aligned", who);
  AdjParams p;
  p.trk_in = (const float*)trk_in;
  p.hits = (const float*)hits;
  p.dr = dr;
  p.nlay = nlay_lane;
  p.trk_out = (float*)trk_out;
  p.chi2_out = chi2_out;
  p.g_trk_out = (const float*)grad_trk_out;
  p.g_chi2 = grad_chi2;
  p.g_trk_in = (float*)grad_trk_in;
  p.g_hits = (float*)grad_hits;
  p.partials = (float*)workspace;
  p.nblocks = nblocks;
  p.bsize = cfg->bsize;
  p.nlayer = cfg->nlayer;
  p.kfact = p2r_kfact_of(cfg->bz);
  p.bz = (float)(cfg->bz == 0.0 ? 3.8112 : cfg->bz);
  const long long ntr = nblocks * cfg->bsize;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch (ckpt_stride) {
    case 1: e = launch_fwdbwd<1>(p, ntr, st); break;
    case 2: e = launch_fwdbwd<2>(p, ntr, st); break;
    case 4: e = launch_fwdbwd<4>(p, ntr, st); break;
    case 0:
    case 5: e = launch_fwdbwd<5>(p, ntr, st); break;
    case 10: e = launch_fwdbwd<10>(p, ntr, st); break;
    default:
      return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: checkpoint stride %d (use 1, 2, 4, 5 or 10)", who, ckpt_stride);
  }
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: launch failed: %s", who, cudaGetErrorString(e));
  const int nout = cfg->nlayer + 1;
  double* ev = (double*)((char*)workspace + w.event_off);
  double* tot = (double*)((char*)workspace + w.total_off);
  // per-event sums (warps of an event are contiguous when bsize % 32 == 0), then totals
  const bool per_event = cfg->bsize % 32 == 0;
  const long long wpe = per_event ? cfg->nb * cfg->bsize / 32 : w.nwarps;
  const long long rows = per_event ? cfg->nevts : 1;
  sum_partials_kernel<<<dim3((unsigned)rows, (unsigned)nout), 256, 0, st>>>(p.partials, w.nwarps, nout, wpe, ev);
  sum_rows_kernel<<<(nout + 63) / 64, 64, 0, st>>>(ev, rows, nout, tot);
  if (grad_dr || grad_bz) split_kernel<<<(nout + 63) / 64, 64, 0, st>>>(tot, 1, cfg->nlayer, grad_dr, grad_bz);
  if (grad_dr_event || grad_bz_event)
    split_kernel<<<(unsigned)((rows * nout + 255) / 256), 256, 0, st>>>(ev, rows, cfg->nlayer, grad_dr_event,
                                                                        grad_bz_event);
  e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: reduction launch failed: %s", who, cudaGetErrorString(e));
  return p2r_clear_error();
}

}  // extern "C"
