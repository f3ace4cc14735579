// Fused forward + adjoint of the chained layer loop (sm_100a), and its C-ABI entry points.
//
// One thread per track. The forward pass stores the track state every CK layers
// (thread-local checkpoints). The reverse sweep walks the segments backwards: it recomputes
// the states inside a segment from its checkpoint, then for each layer, last to first,
// recomputes that layer with the tape of p2r_adjoint.cuh and runs the hand-written reverse
// of the update and of the propagation. Gradients produced:
//   per track  d/d(initial par, cov), d/d(hit pos, hit cov) for every layer
//   shared     d/d(dr[layer]) and d/d(Bz), summed over tracks, and optionally per event
// of L = sum_tracks (g_par . par_final + g_cov . cov_final + g_chi2 * chi2_total).
//
// Precision: by default the whole kernel (carried state, trajectory, tape and reverse)
// runs in FP64. Measured on the synthetic-helix workload: the FP32 chain leaves 0.7 % (p99)
// of rounding in chi2 (an FP32 position at 100 cm carries ~8e-6 cm, ~1 % of a 10 um
// residual) and 16-46 % (p99) in d/d(initial parameters) (the filtered state depends on
// the seed through small differences of large terms); FP64 arithmetic with the state
// rounded to FP32 between layers still leaves 2e-3 on d chi2/d dr. P2R_FLAG_ADJ_FP32 selects
// the FP32 kernel (the same code instantiated in float) where that accuracy suffices.
//
// Shared sums: each warp reduces with shuffles (fixed order) into per-warp double partials in
// the workspace; a second kernel adds the partials in a fixed order in double, so the
// results are deterministic run to run.
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
#include <new>

#include "p2r_adjoint.cuh"
#include "p2r_internal.h"
#include "p2r_queue_check.cuh"

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
  double* partials;         // [nwarps][nlayer + 1]
  const uint32_t* order;    // nullable: the track at each position (each event's tracks by layer count)
  long long nblocks;
  int bsize;
  int nlayer;
  float kfact;
  double bz;
};

template <class T>
__device__ __forceinline__ T warp_sum_t(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class T>
__device__ __forceinline__ void load_hit_t(const float* h, int bs, int it, T (&hp)[3], T (&hc)[6]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) hp[i] = (T)h[i * bs + it];
#pragma unroll
  for (int i = 0; i < 6; ++i) hc[i] = (T)h[(3 + i) * bs + it];
}

// T: arithmetic type of the whole kernel (float or double). CK: checkpoint stride.
template <class T, int CK>
__global__ void __launch_bounds__(kAdjThreads) fwdbwd_kernel(AdjParams p) {
  constexpr int NCK = (kMaxAdjLayers + CK - 1) / CK;
  const int bs = p.bsize;
  const int lane = threadIdx.x & 31;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long b = g / bs;
  int it = (int)(g - b * bs);
  bool valid = b < p.nblocks;
  if (valid && p.order) {  // position g holds track order[g]
    const long long t = p.order[g];
    valid = t < p.nblocks * bs;
    b = valid ? t / bs : 0;
    it = valid ? (int)(t - b * bs) : 0;
  }
  const long long gwarp = g >> 5;
  double* wpart = p.partials + gwarp * (p.nlayer + 1);

  T par[6] = {0, 0, 0, 1, 0, 1}, cov[21] = {};
  int q = 1;
  int nl = 0;
  const float* tb = p.trk_in + b * (long long)(28 * bs);
  if (valid) {
#pragma unroll
    for (int i = 0; i < 6; ++i) par[i] = (T)tb[i * bs + it];
#pragma unroll
    for (int i = 0; i < 21; ++i) cov[i] = (T)tb[(6 + i) * bs + it];
    q = __float_as_int(tb[27 * bs + it]);
    nl = p.nlay ? min(p.nlayer, max(0, p.nlay[b * bs + it])) : p.nlayer;
  }
  // k = q * kfact(Bz) in the kernel's precision (kfact evaluated in double, TBB:654)
  const T kfact = (sizeof(T) == sizeof(float)) ? (T)p.kfact : (T)(100.0 / (-0.299792458 * p.bz));
  const T k = (T)q * kfact;
  const T kinv = T(1) / k;
  int nl_warp = nl;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nl_warp = max(nl_warp, __shfl_xor_sync(0xffffffffu, nl_warp, o));
  const float* hblk = p.hits + b * (long long)p.nlayer * (9 * bs);

  // ---- forward pass with checkpoints every CK layers
  T ck[NCK][27];
  T chi2 = 0;
  for (int l = 0; l < nl; ++l) {
    if (l % CK == 0) {
#pragma unroll
      for (int i = 0; i < 6; ++i) ck[l / CK][i] = par[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) ck[l / CK][6 + i] = cov[i];
    }
    T hp[3], hc[6];
    load_hit_t(hblk + (long long)l * (9 * bs), bs, it, hp, hc);
    chi2 += adj::layer_fwd(par, cov, k, kinv, hp, hc, p.dr ? (T)p.dr[l] : T(0));
  }
  if (valid) {
    if (p.trk_out) {
      float* ob = p.trk_out + b * (long long)(28 * bs);
#pragma unroll
      for (int i = 0; i < 6; ++i) ob[i * bs + it] = (float)par[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) ob[(6 + i) * bs + it] = (float)cov[i];
      ob[27 * bs + it] = __int_as_float(q);
    }
    if (p.chi2_out) p.chi2_out[b * bs + it] = (float)chi2;
  }

  // ---- reverse sweep
  T pb[6] = {}, cb[21] = {};
  T chi2b = 0;
  if (valid) {
    if (p.g_trk_out) {
      const float* gb = p.g_trk_out + b * (long long)(28 * bs);
#pragma unroll
      for (int i = 0; i < 6; ++i) pb[i] = (T)gb[i * bs + it];
#pragma unroll
      for (int i = 0; i < 21; ++i) cb[i] = (T)gb[(6 + i) * bs + it];
    }
    if (p.g_chi2) chi2b = (T)p.g_chi2[b * bs + it];
  }
  T kbar = 0, kinvbar = 0;
  const int nseg = (nl_warp + CK - 1) / CK;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int a = seg * CK;
    const int e = min(a + CK, nl_warp);
    // states before layers a .. e-1 of this segment, recomputed from the checkpoint
    T st[CK][27];
    if (a < nl) {
#pragma unroll
      for (int i = 0; i < 27; ++i) st[0][i] = ck[seg][i];
    }
    for (int l = a + 1; l < e && l < nl; ++l) {
      T sp[6], sc[21];
#pragma unroll
      for (int i = 0; i < 6; ++i) sp[i] = st[l - 1 - a][i];
#pragma unroll
      for (int i = 0; i < 21; ++i) sc[i] = st[l - 1 - a][6 + i];
      T hp[3], hc[6];
      load_hit_t(hblk + (long long)(l - 1) * (9 * bs), bs, it, hp, hc);
      adj::layer_fwd(sp, sc, k, kinv, hp, hc, p.dr ? (T)p.dr[l - 1] : T(0));
#pragma unroll
      for (int i = 0; i < 6; ++i) st[l - a][i] = sp[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) st[l - a][6 + i] = sc[i];
    }
    for (int l = e - 1; l >= a; --l) {
      T drb = 0;
      if (l < nl) {
        T sp[6], sc[21];
#pragma unroll
        for (int i = 0; i < 6; ++i) sp[i] = st[l - a][i];
#pragma unroll
        for (int i = 0; i < 21; ++i) sc[i] = st[l - a][6 + i];
        T hp[3], hc[6], hpb[3], hcb[6];
        load_hit_t(hblk + (long long)l * (9 * bs), bs, it, hp, hc);
        adj::layer_rev(sp, sc, k, kinv, hp, hc, p.dr ? (T)p.dr[l] : T(0), pb, cb, chi2b, hpb, hcb, drb, kbar,
                       kinvbar);
        if (p.g_hits) {
          float* gh = p.g_hits + (b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
          for (int i = 0; i < 3; ++i) gh[i * bs + it] = (float)hpb[i];
#pragma unroll
          for (int i = 0; i < 6; ++i) gh[(3 + i) * bs + it] = (float)hcb[i];
        }
      } else if (valid && p.g_hits) {
        float* gh = p.g_hits + (b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
        for (int i = 0; i < 9; ++i) gh[i * bs + it] = 0.f;
      }
      drb = warp_sum_t(drb);
      if (lane == 0) wpart[l] = (double)drb;
    }
  }
  // layers the whole warp skipped have zero gradient
  if (lane == 0)
    for (int l = nl_warp; l < p.nlayer; ++l) wpart[l] = 0.0;
  if (valid && p.g_hits)
    for (int l = nl_warp; l < p.nlayer; ++l) {
      float* gh = p.g_hits + (b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
      for (int i = 0; i < 9; ++i) gh[i * bs + it] = 0.f;
    }
  // k = q * kfact(Bz): dk/dBz = -k / Bz
  T bzb = valid ? (kbar - kinvbar * kinv * kinv) * (-k / (T)p.bz) : T(0);
  bzb = warp_sum_t(bzb);
  if (lane == 0) wpart[p.nlayer] = (double)bzb;
  if (valid && p.g_trk_in) {
    float* gb = p.g_trk_in + b * (long long)(28 * bs);
#pragma unroll
    for (int i = 0; i < 6; ++i) gb[i * bs + it] = (float)pb[i];
#pragma unroll
    for (int i = 0; i < 21; ++i) gb[(6 + i) * bs + it] = (float)cb[i];
    gb[27 * bs + it] = 0.f;
  }
}

// ---------------------------------------------------------------- tape path
// The same computation as fwdbwd_kernel split in two kernels, with the checkpoints and the
// recomputed segment states in a tape in device memory instead of thread-local arrays:
// fwd_tape_kernel runs the forward and stores the state every CK layers; rev_tape_kernel
// walks the segments backwards, recomputes each segment's states once into a segment
// buffer, and reverses the layers. At CK = 1 every layer has a slot, and the slot holds the
// propagated state entering the layer's update instead: the reverse starts each layer from it
// and rebuilds the layer's input with one update of the previous slot. Layout of both:
// [slot][27 components][thread], so a warp's 32 lanes read and write one 256-byte (double) or
// 128-byte (float) line per component. Used when the caller's workspace holds the tape
// (p2r_forward_backward_workspace_size_tape).
struct TapeParams {
  void* tape;      // [nslots][27][nthreads] of T: the state before layers 0, CK, 2 CK, ...;
                   // for CK = 1 the state after each layer's propagation, entering its update
  void* segbuf;    // [CK - 1][27][nthreads] of T: the state before layers a+1 .. a+CK-1
  long long nthreads;
};

// One track's column of a tape: slot l, component i at base[l * slot + i * comp + idx].
template <class T>
struct TapeRef {
  T* base;
  long long slot, comp, idx;
  __device__ __forceinline__ void store(long long l, const T (&par)[6], const T (&cov)[21]) const {
    T* q = base + l * slot + idx;
#pragma unroll
    for (int i = 0; i < 6; ++i) q[i * comp] = par[i];
#pragma unroll
    for (int i = 0; i < 21; ++i) q[(6 + i) * comp] = cov[i];
  }
  __device__ __forceinline__ void load(long long l, T (&par)[6], T (&cov)[21]) const {
    const T* q = base + l * slot + idx;
#pragma unroll
    for (int i = 0; i < 6; ++i) par[i] = q[i * comp];
#pragma unroll
    for (int i = 0; i < 21; ++i) cov[i] = q[(6 + i) * comp];
  }
};

// Per-track set-up shared by the tape kernels and the queue kernel: track (block b, lane it)
// of the Matriplex arrays, its initial state, layer count and k = q kfact.
template <class T>
struct TrackCtx {
  long long b;
  int it, lane, nl, nl_warp, q;
  bool valid;
  T k, kinv;
  const float* hblk;
  __device__ TrackCtx(const AdjParams& p, T (&par)[6], T (&cov)[21], long long b_, int it_, bool valid_) {
    const int bs = p.bsize;
    lane = threadIdx.x & 31;
    b = b_;
    it = it_;
    valid = valid_;
    q = 1;
    nl = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) par[i] = (i == 3 || i == 5) ? T(1) : T(0);
#pragma unroll
    for (int i = 0; i < 21; ++i) cov[i] = 0;
    if (valid) {
      const float* tb = p.trk_in + b * (long long)(28 * bs);
#pragma unroll
      for (int i = 0; i < 6; ++i) par[i] = (T)tb[i * bs + it];
#pragma unroll
      for (int i = 0; i < 21; ++i) cov[i] = (T)tb[(6 + i) * bs + it];
      q = __float_as_int(tb[27 * bs + it]);
      nl = p.nlay ? min(p.nlayer, max(0, p.nlay[b * bs + it])) : p.nlayer;
    }
    const T kfact = (sizeof(T) == sizeof(float)) ? (T)p.kfact : (T)(100.0 / (-0.299792458 * p.bz));
    k = (T)q * kfact;
    kinv = T(1) / k;
    nl_warp = nl;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nl_warp = max(nl_warp, __shfl_xor_sync(0xffffffffu, nl_warp, o));
    hblk = p.hits + b * (long long)p.nlayer * (9 * bs);
  }
};

// The grid kernels' track: global thread g is lane it of block b.
template <class T>
__device__ __forceinline__ TrackCtx<T> grid_track(const AdjParams& p, T (&par)[6], T (&cov)[21], long long& g) {
  g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long b = g / p.bsize;
  int it = (int)(g - b * p.bsize);
  bool valid = b < p.nblocks;
  if (valid && p.order) {  // position g holds track order[g]; the tape stays indexed by position
    const long long t = p.order[g];
    valid = t < p.nblocks * p.bsize;
    b = valid ? t / p.bsize : 0;
    it = valid ? (int)(t - b * p.bsize) : 0;
  }
  return TrackCtx<T>(p, par, cov, b, it, valid);
}

template <class T>
__device__ __forceinline__ void write_forward_outputs(const AdjParams& p, const TrackCtx<T>& c, const T (&par)[6],
                                                      const T (&cov)[21], T chi2) {
  if (!c.valid) return;
  const int bs = p.bsize;
  if (p.trk_out) {
    float* ob = p.trk_out + c.b * (long long)(28 * bs);
#pragma unroll
    for (int i = 0; i < 6; ++i) ob[i * bs + c.it] = (float)par[i];
#pragma unroll
    for (int i = 0; i < 21; ++i) ob[(6 + i) * bs + c.it] = (float)cov[i];
    ob[27 * bs + c.it] = __int_as_float(c.q);
  }
  if (p.chi2_out) p.chi2_out[c.b * bs + c.it] = (float)chi2;
}

// CK = 1 forward of one track: the state after each layer's propagation (entering its update)
// goes to tape slot l; the final state and chi2 to the outputs.
template <class T>
__device__ __forceinline__ void fwd_track_ck1(const AdjParams& p, const TrackCtx<T>& c, T (&par)[6], T (&cov)[21],
                                              const TapeRef<T>& tr) {
  const int bs = p.bsize;
  T chi2 = 0;
  for (int l = 0; l < c.nl; ++l) {
    T hp[3], hc[6];
    load_hit_t(c.hblk + (long long)l * (9 * bs), bs, c.it, hp, hc);
    adj::PropTape<T> t;
    const T r = adj::hipo(hp[0], hp[1]) + (p.dr ? (T)p.dr[l] : T(0));
    adj::prop_fwd(par, cov, c.k, c.kinv, r, t, par, cov);
    tr.store(l, par, cov);
    chi2 += adj::upd_fwd(par, cov, hp, hc);
  }
  write_forward_outputs(p, c, par, cov, chi2);
}

// The cotangents of one track's final state and chi2.
template <class T>
__device__ __forceinline__ void load_seeds(const AdjParams& p, const TrackCtx<T>& c, T (&pb)[6], T (&cb)[21], T& chi2b) {
  const int bs = p.bsize;
#pragma unroll
  for (int i = 0; i < 6; ++i) pb[i] = 0;
#pragma unroll
  for (int i = 0; i < 21; ++i) cb[i] = 0;
  chi2b = 0;
  if (!c.valid) return;
  if (p.g_trk_out) {
    const float* gb = p.g_trk_out + c.b * (long long)(28 * bs);
#pragma unroll
    for (int i = 0; i < 6; ++i) pb[i] = (T)gb[i * bs + c.it];
#pragma unroll
    for (int i = 0; i < 21; ++i) cb[i] = (T)gb[(6 + i) * bs + c.it];
  }
  if (p.g_chi2) chi2b = (T)p.g_chi2[c.b * bs + c.it];
}

template <class T>
__device__ __forceinline__ void write_hit_grads(const AdjParams& p, const TrackCtx<T>& c, int l, const T (&hpb)[3],
                                                const T (&hcb)[6]) {
  if (!p.g_hits) return;
  const int bs = p.bsize;
  float* gh = p.g_hits + (c.b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
  for (int i = 0; i < 3; ++i) gh[i * bs + c.it] = (float)hpb[i];
#pragma unroll
  for (int i = 0; i < 6; ++i) gh[(3 + i) * bs + c.it] = (float)hcb[i];
}

template <class T>
__device__ __forceinline__ void zero_hit_grads(const AdjParams& p, const TrackCtx<T>& c, int l) {
  if (!c.valid || !p.g_hits) return;
  const int bs = p.bsize;
  float* gh = p.g_hits + (c.b * (long long)p.nlayer + l) * (9 * bs);
#pragma unroll
  for (int i = 0; i < 9; ++i) gh[i * bs + c.it] = 0.f;
}

// End of one track's reverse sweep: zero gradients of layers the whole warp skipped, the warp's
// Bz partial (lane 0 writes wpart[nlayer]) and the initial-state gradient.
template <class T>
__device__ __forceinline__ void finish_track(const AdjParams& p, const TrackCtx<T>& c, const T (&pb)[6],
                                             const T (&cb)[21], T kbar, T kinvbar, double* wpart) {
  const int bs = p.bsize;
  if (c.lane == 0)
    for (int l = c.nl_warp; l < p.nlayer; ++l) wpart[l] = 0.0;
  for (int l = c.nl_warp; l < p.nlayer; ++l) zero_hit_grads(p, c, l);
  // k = q * kfact(Bz): dk/dBz = -k / Bz
  T bzb = c.valid ? (kbar - kinvbar * c.kinv * c.kinv) * (-c.k / (T)p.bz) : T(0);
  bzb = warp_sum_t(bzb);
  if (c.lane == 0) wpart[p.nlayer] = (double)bzb;
  if (c.valid && p.g_trk_in) {
    float* gb = p.g_trk_in + c.b * (long long)(28 * bs);
#pragma unroll
    for (int i = 0; i < 6; ++i) gb[i * bs + c.it] = (float)pb[i];
#pragma unroll
    for (int i = 0; i < 21; ++i) gb[(6 + i) * bs + c.it] = (float)cb[i];
    gb[27 * bs + c.it] = 0.f;
  }
}

// CK = 1 reverse of one track from its tape. Layer l, last to first: the update's reverse
// straight from the tape (the propagated state entering it), then the state entering the layer
// (the input track for l = 0, else the update of layer l-1 applied to its tape entry, as the
// forward did), the propagation's tape (its output covariance is not needed, so J C J^T is not
// recomputed) and its reverse. Lane 0 writes the warp's dr and Bz partials to wpart.
template <class T>
__device__ __forceinline__ void rev_track_ck1(const AdjParams& p, const TrackCtx<T>& c, const TapeRef<T>& tr,
                                              double* wpart) {
  const int bs = p.bsize;
  T pb[6], cb[21], chi2b;
  load_seeds(p, c, pb, cb, chi2b);
  T kbar = 0, kinvbar = 0;
  for (int l = c.nl_warp - 1; l >= 0; --l) {
    T drb = 0;
    if (l < c.nl) {
      T hp[3], hc[6], hpb[3], hcb[6];
      load_hit_t(c.hblk + (long long)l * (9 * bs), bs, c.it, hp, hc);
      {
        T up[6], uc[21];
        tr.load(l, up, uc);
        adj::upd_rev(up, uc, hp, hc, pb, cb, chi2b, hpb, hcb);
      }
      T sp[6], sc[21];
      if (l == 0) {
        const float* tb = p.trk_in + c.b * (long long)(28 * bs);
#pragma unroll
        for (int i = 0; i < 6; ++i) sp[i] = (T)tb[i * bs + c.it];
#pragma unroll
        for (int i = 0; i < 21; ++i) sc[i] = (T)tb[(6 + i) * bs + c.it];
      } else {
        T hq[3], hqc[6];
        tr.load(l - 1, sp, sc);
        load_hit_t(c.hblk + (long long)(l - 1) * (9 * bs), bs, c.it, hq, hqc);
        adj::upd_fwd(sp, sc, hq, hqc);
      }
      const T rh = adj::hipo(hp[0], hp[1]);
      const T r = rh + (p.dr ? (T)p.dr[l] : T(0));
      adj::PropTape<T> t;
      T pp[6], pc[21];
      adj::prop_fwd(sp, sc, c.k, c.kinv, r, t, pp, pc);
      T pin[6], cin[21], rbar = 0;
      adj::prop_rev(t, sp, sc, c.k, c.kinv, r, pb, cb, pin, cin, rbar, kbar, kinvbar);
#pragma unroll
      for (int i = 0; i < 6; ++i) pb[i] = pin[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) cb[i] = cin[i];
      drb = rbar;
      if (rh > T(0)) {
        const T irh = T(1) / rh;
        hpb[0] += rbar * hp[0] * irh;
        hpb[1] += rbar * hp[1] * irh;
      }
      write_hit_grads(p, c, l, hpb, hcb);
    } else {
      zero_hit_grads(p, c, l);
    }
    drb = warp_sum_t(drb);
    if (c.lane == 0) wpart[l] = (double)drb;
  }
  finish_track(p, c, pb, cb, kbar, kinvbar, wpart);
}

template <class T, int CK>
__global__ void __launch_bounds__(kAdjThreads) fwd_tape_kernel(AdjParams p, TapeParams tp) {
  T par[6], cov[21];
  long long g;
  const TrackCtx<T> c = grid_track(p, par, cov, g);
  const int bs = p.bsize;
  const TapeRef<T> tr{(T*)tp.tape, 27 * tp.nthreads, tp.nthreads, g};
  if constexpr (CK == 1) {
    fwd_track_ck1(p, c, par, cov, tr);
  } else {
    T chi2 = 0;
    for (int l = 0; l < c.nl; ++l) {
      T hp[3], hc[6];
      load_hit_t(c.hblk + (long long)l * (9 * bs), bs, c.it, hp, hc);
      if (l % CK == 0) tr.store(l / CK, par, cov);
      chi2 += adj::layer_fwd(par, cov, c.k, c.kinv, hp, hc, p.dr ? (T)p.dr[l] : T(0));
    }
    write_forward_outputs(p, c, par, cov, chi2);
  }
}

template <class T, int CK>
__global__ void __launch_bounds__(kAdjThreads) rev_tape_kernel(AdjParams p, TapeParams tp) {
  T par[6], cov[21];
  long long g;
  const TrackCtx<T> c = grid_track(p, par, cov, g);
  const int bs = p.bsize;
  const TapeRef<T> tr{(T*)tp.tape, 27 * tp.nthreads, tp.nthreads, g};
  double* wpart = p.partials + (g >> 5) * (p.nlayer + 1);
  if constexpr (CK == 1) {
    rev_track_ck1(p, c, tr, wpart);
  } else {
    const TapeRef<T> sr{(T*)tp.segbuf, 27 * tp.nthreads, tp.nthreads, g};
    T pb[6], cb[21], chi2b;
    load_seeds(p, c, pb, cb, chi2b);
    T kbar = 0, kinvbar = 0;
    const int nseg = (c.nl_warp + CK - 1) / CK;
    for (int seg = nseg - 1; seg >= 0; --seg) {
      const int a = seg * CK;
      const int e = min(a + CK, c.nl_warp);
      if (a + 1 < min(e, c.nl)) {
        // states before layers a+1 .. e-1, recomputed once from the checkpoint
        T sp[6], sc[21];
        tr.load(seg, sp, sc);
        for (int l = a + 1; l < e && l < c.nl; ++l) {
          T hp[3], hc[6];
          load_hit_t(c.hblk + (long long)(l - 1) * (9 * bs), bs, c.it, hp, hc);
          adj::layer_fwd(sp, sc, c.k, c.kinv, hp, hc, p.dr ? (T)p.dr[l - 1] : T(0));
          sr.store(l - a - 1, sp, sc);
        }
      }
      for (int l = e - 1; l >= a; --l) {
        T drb = 0;
        if (l < c.nl) {
          T sp[6], sc[21];
          if (l == a)
            tr.load(seg, sp, sc);
          else
            sr.load(l - a - 1, sp, sc);
          T hp[3], hc[6], hpb[3], hcb[6];
          load_hit_t(c.hblk + (long long)l * (9 * bs), bs, c.it, hp, hc);
          adj::layer_rev(sp, sc, c.k, c.kinv, hp, hc, p.dr ? (T)p.dr[l] : T(0), pb, cb, chi2b, hpb, hcb, drb, kbar,
                         kinvbar);
          write_hit_grads(p, c, l, hpb, hcb);
        } else {
          zero_hit_grads(p, c, l);
        }
        drb = warp_sum_t(drb);
        if (c.lane == 0) wpart[l] = (double)drb;
      }
    }
    finish_track(p, c, pb, cb, kbar, kinvbar, wpart);
  }
}

// ---------------------------------------------------------------- persistent queue path
// Forward + adjoint of an uneven batch in ONE persistent launch: CTAs pull (event, block range)
// items from the queue's atomic counter (the items are checked on the device first, as in the
// forward queue kernel); each warp takes 32-lane slices of an item's blocks and runs, per lane,
// the CK = 1 forward (FP64, propagated states to the warp's own tape) and then the reverse from
// that tape. A warp's tape is [nlayer][27][32] doubles in the workspace, reused slice after
// slice, so the memory is bounded by the resident warps (not by the batch) and the reverse reads
// back the most recently written entries first, while they are still in L2. Shared-gradient
// partials go to a per-slice row (slice = block * (bsize / 32) + 32-lane group), summed per event
// and then in total in a fixed order: deterministic, and the same per-slice order as the
// per-warp partials of the grid kernels.
struct QAdjParams {
  const p2r_queue_item* items;
  long long n_items;
  const int64_t* ev_off;
  long long nevts;
  int* counter;
  unsigned* error;
  double* tapes;          // [tape_warps][nlayer][27][32]
  double* slice_partials; // [nblocks * bsize / 32][nlayer + 1]
  const uint32_t* order;  // nullable: track at each position, each event's tracks by layer count
};

__global__ void __launch_bounds__(kAdjThreads) queue_adj_kernel(AdjParams p, QAdjParams q) {
  __shared__ long long s_item;
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const int spb = p.bsize / 32;
  const long long tstride = (long long)p.nlayer * 27 * 32;
  double* tape = q.tapes + ((long long)blockIdx.x * nwarps + warp) * tstride;
  const TapeRef<double> tr{tape, 27 * 32, 32, lane};
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(q.counter, 1);
    __syncthreads();
    const long long item = s_item;
    __syncthreads();  // every thread has read s_item before thread 0 claims the next one
    if (item >= q.n_items) break;
    const p2r_queue_item qi = q.items[item];
    const unsigned bad = queue_item_error(qi, q.nevts, p.nblocks, q.ev_off);
    if (bad) {
      if (threadIdx.x == 0) atomicOr(q.error, bad);
      continue;
    }
    const int nslices = qi.nblk * spb;
    const long long ntr = p.nblocks * p.bsize;
    for (int s = warp; s < nslices; s += nwarps) {
      // position (block b, lane it) of the batch; with an order, the track placed there
      long long b = qi.block0 + s / spb;
      int it = (s % spb) * 32 + lane;
      const long long slice = b * spb + s % spb;
      bool valid = true;
      if (q.order) {
        const long long t = q.order[b * p.bsize + it];
        valid = t < ntr;  // written by the ordering kernel for every position of a valid item
        if (!valid) atomicOr(q.error, kQerrOrder);
        b = valid ? t / p.bsize : 0;
        it = valid ? (int)(t - b * p.bsize) : 0;
      }
      double par[6], cov[21];
      const TrackCtx<double> c(p, par, cov, b, it, valid);
      fwd_track_ck1(p, c, par, cov, tr);
      rev_track_ck1(p, c, tr, q.slice_partials + slice * (p.nlayer + 1));
    }
  }
}

// Tracks ordered by layer count, longest first, ties in track order, within windows of
// win_blocks blocks of each event (win_blocks <= 0: whole events): order[pos] = the track placed
// at position pos, always a track of the same window. Small windows keep a warp's 32 tracks
// within a few neighbouring blocks, so the hits the lanes read one by one share cache lines with
// the other warps of the window; whole events give the most uniform lengths per warp. Measured on
// the 40-layer calibration workload: the grid adjoint is faster with windows of 512 tracks
// (kOrderWindow), the persistent queue adjoint with whole events. Stable counting sort, one CTA
// per window: keys nlayer - clamp(nlay, 0, nlayer) ascending; each lane's rank among equal keys
// comes from its warp (__match_any_sync) and the warps before it. Grid (nevts, Y): CTA (e, y)
// sorts windows y, y + Y, ... of event e.
constexpr int kOrderThreads = 512;
constexpr int kOrderWindow = 512;
__global__ void __launch_bounds__(kOrderThreads) order_by_layers_kernel(const int32_t* nlay, const int64_t* ev_off,
                                                                       long long nb_event, long long nblocks, int bsize,
                                                                       int nlayer, long long win_blocks,
                                                                       uint32_t* order) {
  constexpr int kW = kOrderThreads / 32;
  __shared__ int base[kMaxAdjLayers + 1];
  __shared__ int wcount[kW][kMaxAdjLayers + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nkeys = nlayer + 1;
  const long long e = blockIdx.x;
  // event e's blocks: [ev_off[e], ev_off[e+1]), or [e nb_event, (e+1) nb_event) without offsets
  long long b0 = ev_off ? ev_off[e] : e * nb_event, b1 = ev_off ? ev_off[e + 1] : (e + 1) * nb_event;
  b0 = b0 < 0 ? 0 : (b0 > nblocks ? nblocks : b0);
  b1 = b1 < b0 ? b0 : (b1 > nblocks ? nblocks : b1);
  // blocks per window (win_blocks <= 0: the whole event is one window)
  const long long wb = win_blocks > 0 ? win_blocks : (b1 - b0 > 0 ? b1 - b0 : 1);
  const long long nwin = (b1 - b0 + wb - 1) / wb;
  const unsigned lt = (1u << lane) - 1u;
  for (long long wi = blockIdx.y; wi < nwin; wi += gridDim.y) {
    const long long t0 = (b0 + wi * wb) * bsize;
    const long long t1 = (b0 + wi * wb + wb < b1 ? b0 + wi * wb + wb : b1) * bsize;
    // the window holds at most kOrderThreads tracks when bsize <= kOrderWindow; larger blocks
    // make a one-block window sorted in several chunks
    for (int k = tid; k < nkeys; k += kOrderThreads) base[k] = 0;
    __syncthreads();
    for (long long t = t0 + tid; t < t1; t += kOrderThreads) {
      const int v = nlay[t];
      atomicAdd(&base[nlayer - (v < 0 ? 0 : (v > nlayer ? nlayer : v))], 1);
    }
    __syncthreads();
    if (tid == 0) {
      int run = 0;
      for (int k = 0; k < nkeys; ++k) {
        const int c = base[k];
        base[k] = run;
        run += c;
      }
    }
    __syncthreads();
    for (long long c = t0; c < t1; c += kOrderThreads) {
      const long long t = c + tid;
      const bool valid = t < t1;
      int k = -1;
      if (valid) {
        const int v = nlay[t];
        k = nlayer - (v < 0 ? 0 : (v > nlayer ? nlayer : v));
      }
      const unsigned same = __match_any_sync(0xffffffffu, k);
      const int rank = __popc(same & lt);
      for (int j = lane; j < nkeys; j += 32) wcount[warp][j] = 0;
      __syncwarp();
      if (valid && rank == 0) wcount[warp][k] = __popc(same);
      __syncthreads();
      if (valid) {
        long long pre = t0 + base[k] + rank;
        for (int w = 0; w < warp; ++w) pre += wcount[w][k];
        order[pre] = (uint32_t)t;
      }
      __syncthreads();
      for (int j = tid; j < nkeys; j += kOrderThreads) {
        int add = 0;
        for (int w = 0; w < kW; ++w) add += wcount[w][j];
        base[j] += add;
      }
      __syncthreads();
    }
  }
}

// Grid of order_by_layers_kernel: one row per event, enough CTAs per event to cover ~4 per SM.
inline dim3 order_grid(long long nevts) {
  const long long y = nevts >= 1184 ? 1 : (1184 + nevts - 1) / nevts;
  return dim3((unsigned)nevts, (unsigned)(y > 65535 ? 65535 : y));
}

// Sums per-warp partials [nwarps][nout] in a fixed order, in double. Block (e, j) sums
// warps [e*wpe, min((e+1)*wpe, nwarps)) of column j into out[e*nout + j].
__global__ void __launch_bounds__(256) sum_partials_kernel(const double* partials, long long nwarps, int nout,
                                                           long long wpe, double* out) {
  __shared__ double red[256];
  const long long e = blockIdx.x;
  const int j = blockIdx.y;
  const long long w0 = e * wpe, w1 = min(w0 + wpe, nwarps);
  double s = 0.0;
  for (long long w = w0 + threadIdx.x; w < w1; w += blockDim.x) s += partials[w * nout + j];
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

// workspace: double partials[nwarps][nlayer+1], then (256-byte aligned) double
// event_sums[nevts][nlayer+1] and double totals[nlayer+1]
struct WsLayout {
  long long nwarps;
  size_t partial_bytes, event_off, total_off, order_off, total_bytes;
};

// With P2R_FLAG_ORDER_BY_LAYERS the track order (uint32 per track) follows the totals.
WsLayout layout_of(const p2r_config* cfg) {
  WsLayout w;
  const long long ntr = (long long)cfg->nevts * cfg->nb * cfg->bsize;
  const long long nthreads = (ntr + kAdjThreads - 1) / kAdjThreads * kAdjThreads;
  w.nwarps = nthreads / 32;
  w.partial_bytes = (size_t)w.nwarps * (cfg->nlayer + 1) * sizeof(double);
  w.event_off = (w.partial_bytes + 255) & ~(size_t)255;
  w.total_off = w.event_off + (((size_t)cfg->nevts * (cfg->nlayer + 1) * sizeof(double) + 255) & ~(size_t)255);
  w.total_bytes = w.total_off + (size_t)(cfg->nlayer + 1) * sizeof(double);
  w.order_off = (w.total_bytes + 255) & ~(size_t)255;
  if (cfg->flags & P2R_FLAG_ORDER_BY_LAYERS) w.total_bytes = w.order_off + (size_t)ntr * sizeof(uint32_t);
  return w;
}

// Tape region after the partial sums: [nslots][27][nthreads] checkpoints, then
// [CK - 1][27][nthreads] segment states, in the kernel's arithmetic type.
struct TapeLayout {
  long long nthreads;
  size_t tape_off, seg_off, end;
};

TapeLayout tape_layout_of(const p2r_config* cfg, int ck, size_t elem) {
  TapeLayout t;
  const long long ntr = (long long)cfg->nevts * cfg->nb * cfg->bsize;
  t.nthreads = (ntr + kAdjThreads - 1) / kAdjThreads * kAdjThreads;
  const long long nslots = (cfg->nlayer + ck - 1) / ck;
  const size_t per_slot = (size_t)27 * t.nthreads * elem;
  t.tape_off = (layout_of(cfg).total_bytes + 255) & ~(size_t)255;
  t.seg_off = t.tape_off + (((size_t)nslots * per_slot + 255) & ~(size_t)255);
  t.end = t.seg_off + (size_t)(ck - 1) * per_slot;
  return t;
}

int normal_ckpt(int ckpt_stride) { return ckpt_stride == 0 ? 5 : ckpt_stride; }

template <class T, int CK>
cudaError_t launch_tape(const AdjParams& p, const TapeParams& tp, cudaStream_t st) {
  const unsigned grid = (unsigned)(tp.nthreads / kAdjThreads);
  fwd_tape_kernel<T, CK><<<grid, kAdjThreads, 0, st>>>(p, tp);
  rev_tape_kernel<T, CK><<<grid, kAdjThreads, 0, st>>>(p, tp);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_tape_ck(const AdjParams& p, const TapeParams& tp, int ck, cudaStream_t st) {
  switch (ck) {
    case 1: return launch_tape<T, 1>(p, tp, st);
    case 2: return launch_tape<T, 2>(p, tp, st);
    case 4: return launch_tape<T, 4>(p, tp, st);
    case 10: return launch_tape<T, 10>(p, tp, st);
    default: return launch_tape<T, 5>(p, tp, st);
  }
}

template <class T, int CK>
cudaError_t launch_fwdbwd(const AdjParams& p, long long ntr, cudaStream_t st) {
  const long long grid = (ntr + kAdjThreads - 1) / kAdjThreads;
  fwdbwd_kernel<T, CK><<<(unsigned)grid, kAdjThreads, 0, st>>>(p);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_fwdbwd_ck(const AdjParams& p, long long ntr, int ck, cudaStream_t st) {
  switch (ck) {
    case 1: return launch_fwdbwd<T, 1>(p, ntr, st);
    case 2: return launch_fwdbwd<T, 2>(p, ntr, st);
    case 4: return launch_fwdbwd<T, 4>(p, ntr, st);
    case 10: return launch_fwdbwd<T, 10>(p, ntr, st);
    default: return launch_fwdbwd<T, 5>(p, ntr, st);
  }
}

}  // namespace

extern "C" {

size_t p2r_forward_backward_workspace_size(const p2r_config* cfg) {
  if (p2r_check_config(cfg, "p2r_forward_backward_workspace_size")) return 0;
  return layout_of(cfg).total_bytes;
}

size_t p2r_forward_backward_workspace_size_tape(const p2r_config* cfg, int32_t ckpt_stride) {
  if (p2r_check_config(cfg, "p2r_forward_backward_workspace_size_tape")) return 0;
  const int ck = normal_ckpt(ckpt_stride);
  if (ck != 1 && ck != 2 && ck != 4 && ck != 5 && ck != 10) return 0;
  return tape_layout_of(cfg, ck, (cfg->flags & P2R_FLAG_ADJ_FP32) ? sizeof(float) : sizeof(double)).end;
}

int p2r_forward_backward(const p2r_config* cfg, const void* trk_in, const void* hits, const float* dr,
                         const int32_t* nlay_lane, void* trk_out, float* chi2_out, const void* grad_trk_out,
                         const float* grad_chi2, void* grad_trk_in, void* grad_hits, double* grad_dr, double* grad_bz,
                         double* grad_dr_event, double* grad_bz_event, int32_t ckpt_stride, void* workspace,
                         size_t workspace_bytes, void* stream) {
  const char* who = "p2r_forward_backward";
  P2rRange range(who);
  int rc = p2r_check_config(cfg, who);
  if (rc) return rc;
  if (cfg->mode != P2R_MODE_CHAINED) return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: only CHAINED mode has an adjoint", who);
  if (cfg->flags & P2R_FLAG_SQUASH_PHI)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: P2R_FLAG_SQUASH_PHI is a forward-only option", who);
  if ((cfg->flags & P2R_FLAG_ORDER_BY_LAYERS) && (long long)cfg->nevts * cfg->nb * cfg->bsize > (long long)UINT32_MAX)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: ordering needs fewer than 2^32 tracks", who);
  if (cfg->nlayer > kMaxAdjLayers)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: nlayer %d exceeds %d", who, cfg->nlayer, kMaxAdjLayers);
  const long long nblocks = (long long)cfg->nevts * cfg->nb;
  if (nblocks == 0) return p2r_clear_error();
  if (!trk_in || !hits) return p2r_set_errorf(P2R_ERR_INVALID, "%s: null input array", who);
  if ((rc = p2r_check_aligned(who, 4, {trk_in, hits, dr, nlay_lane, trk_out, chi2_out, grad_trk_out, grad_chi2,
                                       grad_trk_in, grad_hits})) ||
      (rc = p2r_check_aligned(who, 8, {grad_dr, grad_bz, grad_dr_event, grad_bz_event})))
    return rc;
  if ((grad_dr_event || grad_bz_event) && cfg->bsize % 32 != 0)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: per-event gradients need bsize %% 32 == 0", who);
  const WsLayout w = layout_of(cfg);
  if (!workspace || workspace_bytes < w.total_bytes)
    return p2r_set_errorf(P2R_ERR_WORKSPACE, "%s: workspace of %zu bytes needed", who, w.total_bytes);
  if (((uintptr_t)workspace & 255u) != 0) return p2r_set_errorf(P2R_ERR_INVALID, "%s: workspace must be 256-byte aligned", who);
  {
    // no written array may share a byte with another array of the call (the kernels read
    // inputs after other tracks' outputs are written)
    const size_t tb = (size_t)nblocks * 28 * cfg->bsize * sizeof(float);
    const size_t hb = (size_t)nblocks * cfg->nlayer * 9 * cfg->bsize * sizeof(float);
    const size_t lb = (size_t)nblocks * cfg->bsize * sizeof(float);
    const size_t nl = (size_t)cfg->nlayer;
    if ((rc = p2r_check_spans(
             who, {{"trk_in", trk_in, tb, false},
                   {"hits", hits, hb, false},
                   {"dr", dr, nl * sizeof(float), false},
                   {"nlay_lane", nlay_lane, lb, false},
                   {"grad_trk_out", grad_trk_out, tb, false},
                   {"grad_chi2", grad_chi2, lb, false},
                   {"trk_out", trk_out, tb, true},
                   {"chi2_out", chi2_out, lb, true},
                   {"grad_trk_in", grad_trk_in, tb, true},
                   {"grad_hits", grad_hits, hb, true},
                   {"grad_dr", grad_dr, nl * sizeof(double), true},
                   {"grad_bz", grad_bz, sizeof(double), true},
                   {"grad_dr_event", grad_dr_event, (size_t)cfg->nevts * nl * sizeof(double), true},
                   {"grad_bz_event", grad_bz_event, (size_t)cfg->nevts * sizeof(double), true},
                   {"workspace", workspace, workspace_bytes, true}})))
      return rc;
  }
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
  p.partials = (double*)workspace;
  // ordering only matters (and only runs) with per-track layer counts
  const bool ordered = (cfg->flags & P2R_FLAG_ORDER_BY_LAYERS) && nlay_lane;
  p.order = ordered ? (const uint32_t*)((char*)workspace + w.order_off) : nullptr;
  p.nblocks = nblocks;
  p.bsize = cfg->bsize;
  p.nlayer = cfg->nlayer;
  p.kfact = p2r_kfact_of(cfg->bz);
  p.bz = cfg->bz == 0.0 ? 3.8112 : cfg->bz;
  const long long ntr = nblocks * cfg->bsize;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (ckpt_stride != 0 && ckpt_stride != 1 && ckpt_stride != 2 && ckpt_stride != 4 && ckpt_stride != 5 &&
      ckpt_stride != 10)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: checkpoint stride %d (use 1, 2, 4, 5 or 10)", who, ckpt_stride);
  if (ordered) {
    const long long win = kOrderWindow / cfg->bsize > 0 ? kOrderWindow / cfg->bsize : 1;
    order_by_layers_kernel<<<order_grid(cfg->nevts), kOrderThreads, 0, st>>>(nlay_lane, nullptr, cfg->nb, nblocks,
                                                                           cfg->bsize, cfg->nlayer, win,
                                                                           (uint32_t*)p.order);
    e = cudaGetLastError();
    if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: launch failed: %s", who, cudaGetErrorString(e));
  }
  const bool fp32 = (cfg->flags & P2R_FLAG_ADJ_FP32) != 0;
  const int ck = normal_ckpt(ckpt_stride);
  const TapeLayout tl = tape_layout_of(cfg, ck, fp32 ? sizeof(float) : sizeof(double));
  if (workspace_bytes >= tl.end) {
    // the workspace holds the tape: two kernels, checkpoints and segment states in memory
    TapeParams tp;
    tp.tape = (char*)workspace + tl.tape_off;
    tp.segbuf = (char*)workspace + tl.seg_off;
    tp.nthreads = tl.nthreads;
    e = fp32 ? launch_tape_ck<float>(p, tp, ck, st) : launch_tape_ck<double>(p, tp, ck, st);
  } else if (fp32) {
    e = launch_fwdbwd_ck<float>(p, ntr, ck, st);
  } else {
    e = launch_fwdbwd_ck<double>(p, ntr, ck, st);
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

// ---------------------------------------------------------------- allocation-free variant
// Some callers cannot allocate device memory at the point where they need gradients:
// code running while another framework captures a CUDA graph (cudaMalloc is not allowed
// during stream capture), online / trigger-style event loops that forbid allocation after
// start-up (unbounded latency and pool fragmentation), and plugin hosts whose device
// memory is entirely owned by the host framework's pool. For them the workspace of
// p2r_forward_backward lives in this fixed device array instead. Every GPU that loads the
// library holds the array until the process exits.
#include <cuda.h>  // driver-API types only; the functions are reached through the runtime

#include <mutex>

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB per GPU
static __device__ __align__(256) unsigned char g_fwdbwd_scratch[kNoAllocScratchBytes];

// The array has its own address in every CUDA context: the runtime's primary context of
// each device, and any context a plugin host creates with the driver API and makes current.
// The address is therefore cached per context, keyed by the context's process-unique id
// (cuCtxGetId), so a context created after another was destroyed (cudaDeviceReset, a
// host's own cuCtxDestroy / cuCtxCreate) never sees a stale address.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

struct ScratchCache {
  std::mutex mu;
  bool resolved = false;
  CtxGetCurrentFn ctx_current = nullptr;
  CtxGetIdFn ctx_id = nullptr;
  static constexpr int kSlots = 64;
  unsigned long long ids[kSlots] = {};
  void* ptrs[kSlots] = {};
  int used = 0;
};
ScratchCache g_scratch;

void resolve_driver_entry_points(ScratchCache& c) {
  if (c.resolved) return;
  c.resolved = true;
  void* f = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    c.ctx_current = (CtxGetCurrentFn)f;
  f = nullptr;
  if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    c.ctx_id = (CtxGetIdFn)f;
  cudaGetLastError();  // a failed query leaves no sticky error for the caller's next check
}

// Unique id of the calling thread's current context, or 0 if none is current (or the driver
// cannot say).
unsigned long long current_context_id(const ScratchCache& c) {
  if (!c.ctx_current || !c.ctx_id) return 0;
  CUcontext ctx = nullptr;
  if (c.ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  unsigned long long id = 0;
  return c.ctx_id(ctx, &id) == CUDA_SUCCESS ? id : 0;
}

// Device address of g_fwdbwd_scratch in the current context. In host code the array's name
// is only a host-side stand-in, so its address is looked up with cudaGetSymbolAddress, with
// the caller's context current, on the first call in each context, and cached.
int scratch_address(void** out) {
  std::lock_guard<std::mutex> lk(g_scratch.mu);
  resolve_driver_entry_points(g_scratch);
  unsigned long long id = current_context_id(g_scratch);
  if (id != 0)
    for (int i = 0; i < g_scratch.used; ++i)
      if (g_scratch.ids[i] == id) {
        *out = g_scratch.ptrs[i];
        return P2R_OK;
      }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_fwdbwd_scratch);
  if (e != cudaSuccess || !p)
    return p2r_set_errorf(P2R_ERR_CUDA, "p2r_forward_backward_noalloc: scratch address: %s", cudaGetErrorString(e));
  // the lookup makes the device's primary context current if no context was
  if (id == 0) id = current_context_id(g_scratch);
  if (id != 0 && g_scratch.used < ScratchCache::kSlots) {  // otherwise: looked up again on every call
    g_scratch.ids[g_scratch.used] = id;
    g_scratch.ptrs[g_scratch.used] = p;
    ++g_scratch.used;
  }
  *out = p;
  return P2R_OK;
}

}  // namespace

extern "C" int p2r_forward_backward_noalloc(const p2r_config* cfg, const void* trk_in, const void* hits,
                                            const float* dr, const int32_t* nlay_lane, void* trk_out,
                                            float* chi2_out, const void* grad_trk_out, const float* grad_chi2,
                                            void* grad_trk_in, void* grad_hits, double* grad_dr, double* grad_bz,
                                            double* grad_dr_event, double* grad_bz_event, int32_t ckpt_stride,
                                            void* stream) {
  int rc = p2r_check_config(cfg, "p2r_forward_backward_noalloc");
  if (rc) return rc;
  const size_t need = layout_of(cfg).total_bytes;
  if (need > kNoAllocScratchBytes)
    return p2r_set_errorf(P2R_ERR_WORKSPACE,
                          "p2r_forward_backward_noalloc: this batch needs %zu bytes of scratch; the allocation-free "
                          "entry point has a fixed %zu bytes per GPU (about (tracks/32)*(nlayer+1)*8 + "
                          "nevts*(nlayer+1)*8 bytes are used): split the batch or pass a workspace to "
                          "p2r_forward_backward",
                          need, kNoAllocScratchBytes);
  void* ws = nullptr;
  if ((rc = scratch_address(&ws))) return rc;
  // Nothing in the scratch must start at zero: the kernel writes every partial it reads
  // and the reductions write every sum. Calls that overlap on the GPU (other streams or
  // threads) share the array and race.
  return p2r_forward_backward(cfg, trk_in, hits, dr, nlay_lane, trk_out, chi2_out, grad_trk_out, grad_chi2,
                              grad_trk_in, grad_hits, grad_dr, grad_bz, grad_dr_event, grad_bz_event, ckpt_stride,
                              ws, kNoAllocScratchBytes, stream);
}

// ---------------------------------------------------------------- persistent queue entry points
namespace p2r {

// Per-event sums of the per-slice partials: block (e, j) adds slices [b0 * spb, b1 * spb) of
// column j, [b0, b1) = event e's block range (clamped to [0, nblocks]; bad offsets are reported
// by the queue checks), in the same fixed order as sum_partials_kernel.
__global__ void __launch_bounds__(256) sum_slices_kernel(const double* partials, const int64_t* ev_off,
                                                         long long nblocks, int spb, int nout, double* out) {
  __shared__ double red[256];
  const long long e = blockIdx.x;
  const int j = blockIdx.y;
  long long b0 = ev_off[e], b1 = ev_off[e + 1];
  b0 = b0 < 0 ? 0 : (b0 > nblocks ? nblocks : b0);
  b1 = b1 < b0 ? b0 : (b1 > nblocks ? nblocks : b1);
  const long long w0 = b0 * spb, w1 = b1 * spb;
  double s = 0.0;
  for (long long w = w0 + threadIdx.x; w < w1; w += blockDim.x) s += partials[w * nout + j];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[e * nout + j] = red[0];
}

}  // namespace p2r

namespace {

// Queue-adjoint workspace: item counter (0) and error word (128) as every queue workspace, then
// double slice partials [nslices][nlayer+1], event sums [nevts][nlayer+1], totals [nlayer+1],
// with P2R_FLAG_ORDER_BY_LAYERS the track order [nblocks * bsize] (uint32), then the warps'
// tapes [tape_warps][nlayer][27][32] doubles.
struct QAdjWs {
  long long nslices;
  size_t partial_off, event_off, total_off, order_off, tape_off, per_warp_tape;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

QAdjWs qadj_ws(const p2r_queue* q) {
  QAdjWs w;
  const size_t nout = (size_t)q->nlayer + 1;
  w.nslices = q->nblocks * (q->bsize / 32);
  w.partial_off = 256;
  w.event_off = align256(w.partial_off + (size_t)w.nslices * nout * sizeof(double));
  w.total_off = align256(w.event_off + (size_t)q->nevts * nout * sizeof(double));
  w.order_off = align256(w.total_off + nout * sizeof(double));
  const bool ordered = (q->flags & P2R_FLAG_ORDER_BY_LAYERS) != 0;
  w.tape_off = align256(w.order_off + (ordered ? (size_t)q->nblocks * q->bsize * sizeof(uint32_t) : 0));
  w.per_warp_tape = (size_t)q->nlayer * 27 * 32 * sizeof(double);
  return w;
}

// Resident CTAs of the queue-adjoint kernel on the current device (the persistent grid).
int qadj_resident_ctas(const p2r_queue* q, int threads, int* out) {
  int dev = 0, sms = 0, occ = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, queue_adj_kernel, threads, 0);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "queue adjoint: %s", cudaGetErrorString(e));
  const int per_sm = q->ctas_per_sm > 0 ? (q->ctas_per_sm < occ ? q->ctas_per_sm : occ) : occ;
  *out = sms * (per_sm > 0 ? per_sm : 1);
  return P2R_OK;
}

int qadj_threads(const p2r_queue* q) { return q->block_threads > 0 ? q->block_threads : kAdjThreads; }

int check_queue_adjoint(const p2r_queue* q, const char* who) {
  int rc = p2r_check_queue(q, who);
  if (rc) return rc;
  if (q->flags & ~(uint32_t)P2R_FLAG_ORDER_BY_LAYERS)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED,
                          "%s: the queue adjoint runs in FP64; P2R_FLAG_ORDER_BY_LAYERS is its only option", who);
  if ((q->flags & P2R_FLAG_ORDER_BY_LAYERS) && q->nblocks * (long long)q->bsize > (long long)UINT32_MAX)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: ordering needs fewer than 2^32 tracks", who);
  if (q->nlayer > kMaxAdjLayers)
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: nlayer %d exceeds %d", who, q->nlayer, kMaxAdjLayers);
  return P2R_OK;
}

int enqueue_queue_adjoint(const p2r_queue* q, const void* trk_in, const void* hits, const float* dr, void* trk_out,
                          float* chi2_out, const void* grad_trk_out, const float* grad_chi2, void* grad_trk_in,
                          void* grad_hits, double* grad_dr, double* grad_bz, double* grad_dr_event,
                          double* grad_bz_event, void* workspace, size_t ws_bytes, cudaStream_t st, const char* who) {
  P2rRange range(who);
  int rc = check_queue_adjoint(q, who);
  if (rc) return rc;
  const QAdjWs w = qadj_ws(q);
  const int threads = qadj_threads(q);
  const int wpc = threads / 32;
  if (!workspace || ws_bytes < w.tape_off + w.per_warp_tape * wpc)
    return p2r_set_errorf(P2R_ERR_WORKSPACE, "%s: workspace of at least %zu bytes needed (%zu for full occupancy: "
                          "p2r_queue_adjoint_workspace_size)", who, w.tape_off + w.per_warp_tape * wpc,
                          p2r_queue_adjoint_workspace_size(q));
  if (((uintptr_t)workspace & 255u) != 0) return p2r_set_errorf(P2R_ERR_INVALID, "%s: workspace must be 256-byte aligned", who);
  if (q->nevts == 0) return p2r_clear_error();
  if (!trk_in || !hits) return p2r_set_errorf(P2R_ERR_INVALID, "%s: null input array", who);
  if ((rc = p2r_check_aligned(who, 4, {trk_in, hits, dr, q->nlay_lane, trk_out, chi2_out, grad_trk_out, grad_chi2,
                                       grad_trk_in, grad_hits})) ||
      (rc = p2r_check_aligned(who, 8, {grad_dr, grad_bz, grad_dr_event, grad_bz_event, q->event_block_offset,
                                       q->items})))
    return rc;
  {
    const size_t tb = (size_t)q->nblocks * 28 * q->bsize * sizeof(float);
    const size_t hb = (size_t)q->nblocks * q->nlayer * 9 * q->bsize * sizeof(float);
    const size_t lb = (size_t)q->nblocks * q->bsize * sizeof(float);
    const size_t nl = (size_t)q->nlayer, ne = (size_t)q->nevts;
    if ((rc = p2r_check_spans(
             who, {{"trk_in", trk_in, tb, false},
                   {"hits", hits, hb, false},
                   {"dr", dr, nl * sizeof(float), false},
                   {"nlay_lane", q->nlay_lane, lb, false},
                   {"event_block_offset", q->event_block_offset, (ne + 1) * sizeof(int64_t), false},
                   {"items", q->items, (size_t)q->n_items * sizeof(p2r_queue_item), false},
                   {"grad_trk_out", grad_trk_out, tb, false},
                   {"grad_chi2", grad_chi2, lb, false},
                   {"trk_out", trk_out, tb, true},
                   {"chi2_out", chi2_out, lb, true},
                   {"grad_trk_in", grad_trk_in, tb, true},
                   {"grad_hits", grad_hits, hb, true},
                   {"grad_dr", grad_dr, nl * sizeof(double), true},
                   {"grad_bz", grad_bz, sizeof(double), true},
                   {"grad_dr_event", grad_dr_event, ne * nl * sizeof(double), true},
                   {"grad_bz_event", grad_bz_event, ne * sizeof(double), true},
                   {"workspace", workspace, ws_bytes, true}})))
      return rc;
  }
  int resident = 0;
  if ((rc = qadj_resident_ctas(q, threads, &resident))) return rc;
  const long long tape_ctas = (long long)((ws_bytes - w.tape_off) / (w.per_warp_tape * wpc));
  long long grid = resident < tape_ctas ? resident : tape_ctas;
  if (grid > q->n_items) grid = q->n_items;
  if (grid < 1) grid = 1;
  AdjParams p;
  p.trk_in = (const float*)trk_in;
  p.hits = (const float*)hits;
  p.dr = dr;
  p.nlay = q->nlay_lane;
  p.trk_out = (float*)trk_out;
  p.chi2_out = chi2_out;
  p.g_trk_out = (const float*)grad_trk_out;
  p.g_chi2 = grad_chi2;
  p.g_trk_in = (float*)grad_trk_in;
  p.g_hits = (float*)grad_hits;
  p.partials = nullptr;
  p.order = nullptr;  // the queue kernel reads its own order (QAdjParams)
  p.nblocks = q->nblocks;
  p.bsize = q->bsize;
  p.nlayer = q->nlayer;
  p.kfact = p2r_kfact_of(q->bz);
  p.bz = q->bz == 0.0 ? 3.8112 : q->bz;
  QAdjParams qp;
  qp.items = q->items;
  qp.n_items = q->n_items;
  qp.ev_off = q->event_block_offset;
  qp.nevts = q->nevts;
  qp.counter = (int*)((char*)workspace + kQueueCounterOff);
  qp.error = (unsigned*)((char*)workspace + kQueueErrorOff);
  qp.slice_partials = (double*)((char*)workspace + w.partial_off);
  qp.tapes = (double*)((char*)workspace + w.tape_off);
  qp.order = (q->flags & P2R_FLAG_ORDER_BY_LAYERS) ? (const uint32_t*)((char*)workspace + w.order_off) : nullptr;
  // counter and error word cleared; slice partials zeroed (slices of skipped items add nothing)
  cudaError_t e = cudaMemsetAsync(workspace, 0, 256, st);
  if (e == cudaSuccess && w.nslices > 0)
    e = cudaMemsetAsync(qp.slice_partials, 0, (size_t)w.nslices * (q->nlayer + 1) * sizeof(double), st);
  if (e == cudaSuccess && qp.order && q->nblocks > 0) {
    order_by_layers_kernel<<<order_grid(q->nevts), kOrderThreads, 0, st>>>(
        q->nlay_lane, q->event_block_offset, 0, q->nblocks, q->bsize, q->nlayer, 0, (uint32_t*)qp.order);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && q->n_items > 0) {
    queue_adj_kernel<<<(unsigned)grid, threads, 0, st>>>(p, qp);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: launch failed: %s", who, cudaGetErrorString(e));
  const int nout = q->nlayer + 1;
  double* ev = (double*)((char*)workspace + w.event_off);
  double* tot = (double*)((char*)workspace + w.total_off);
  sum_slices_kernel<<<dim3((unsigned)q->nevts, (unsigned)nout), 256, 0, st>>>(
      qp.slice_partials, q->event_block_offset, q->nblocks, q->bsize / 32, nout, ev);
  sum_rows_kernel<<<(nout + 63) / 64, 64, 0, st>>>(ev, q->nevts, nout, tot);
  if (grad_dr || grad_bz) split_kernel<<<(nout + 63) / 64, 64, 0, st>>>(tot, 1, q->nlayer, grad_dr, grad_bz);
  if (grad_dr_event || grad_bz_event)
    split_kernel<<<(unsigned)((q->nevts * nout + 255) / 256), 256, 0, st>>>(ev, q->nevts, q->nlayer, grad_dr_event,
                                                                            grad_bz_event);
  e = cudaGetLastError();
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: reduction launch failed: %s", who, cudaGetErrorString(e));
  return p2r_clear_error();
}

}  // namespace

extern "C" {

size_t p2r_queue_adjoint_workspace_size(const p2r_queue* q) {
  const char* who = "p2r_queue_adjoint_workspace_size";
  if (check_queue_adjoint(q, who)) return 0;
  const QAdjWs w = qadj_ws(q);
  const int threads = qadj_threads(q);
  int resident = 0;
  if (qadj_resident_ctas(q, threads, &resident)) return 0;
  long long ctas = resident < q->n_items ? resident : q->n_items;
  if (ctas < 1) ctas = 1;
  p2r_clear_error();
  return w.tape_off + (size_t)ctas * (threads / 32) * w.per_warp_tape;
}

int p2r_run_queue_adjoint(const p2r_queue* q, const void* trk_in, const void* hits, const float* dr, void* trk_out,
                          float* chi2_out, const void* grad_trk_out, const float* grad_chi2, void* grad_trk_in,
                          void* grad_hits, double* grad_dr, double* grad_bz, double* grad_dr_event,
                          double* grad_bz_event, void* workspace, size_t workspace_bytes, void* stream) {
  return enqueue_queue_adjoint(q, trk_in, hits, dr, trk_out, chi2_out, grad_trk_out, grad_chi2, grad_trk_in,
                               grad_hits, grad_dr, grad_bz, grad_dr_event, grad_bz_event, workspace, workspace_bytes,
                               (cudaStream_t)stream, "p2r_run_queue_adjoint");
}

int p2r_queue_adjoint_graph_create(const p2r_queue* q, const void* trk_in, const void* hits, const float* dr,
                                   void* trk_out, float* chi2_out, const void* grad_trk_out, const float* grad_chi2,
                                   void* grad_trk_in, void* grad_hits, double* grad_dr, double* grad_bz,
                                   double* grad_dr_event, double* grad_bz_event, void* workspace,
                                   size_t workspace_bytes, p2r_graph** out) {
  const char* who = "p2r_queue_adjoint_graph_create";
  if (!out) return p2r_set_errorf(P2R_ERR_INVALID, "%s: out is null", who);
  *out = nullptr;
  int rc = check_queue_adjoint(q, who);
  if (rc) return rc;
  cudaStream_t cs;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
  p2r_graph* g = new (std::nothrow) p2r_graph();
  if (!g) {
    cudaStreamDestroy(cs);
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: out of host memory", who);
  }
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = enqueue_queue_adjoint(q, trk_in, hits, dr, trk_out, chi2_out, grad_trk_out, grad_chi2, grad_trk_in,
                               grad_hits, grad_dr, grad_bz, grad_dr_event, grad_bz_event, workspace, workspace_bytes,
                               cs, who);
    cudaError_t e2 = cudaStreamEndCapture(cs, &g->graph);
    if (!rc && e2 != cudaSuccess) e = e2;
  }
  if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  cudaStreamDestroy(cs);
  if (rc || e != cudaSuccess) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return rc ? rc : p2r_set_errorf(P2R_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
  }
  *out = g;
  return p2r_clear_error();
}

}  // extern "C"
