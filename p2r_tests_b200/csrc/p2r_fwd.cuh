// Fused forward kernel template of the p2r hot path for sm_100a (see p2r_forward.cu for the
// C-ABI entry points). Instantiated by p2r_fwd_restart.cu, p2r_fwd_chained.cu and
// p2r_fwd_masked.cu so the variants compile in parallel.
//
//  fwd_kernel  the fused driver loop (TBB:873-926 for one iteration): one thread per track
//              runs every layer with its state in registers. Hits are staged per warp
//              through a shared-memory ring filled by 16-byte cp.async copies (the 32-lane
//              slice of one MPHIT block is 9 rows of 128 B), so the next layers' hits are in
//              flight while the current layer computes.
//
// Layout: MPTRK block = 28*bsize 32-bit words (par 6, cov 21, q 1 rows of bsize lanes),
// MPHIT block = 9*bsize words (pos 3, cov 6), TBB:56-125. Track block b = ib + nb*ev,
// hit block lay + b*nlayer (TBB:147-153, 212-217).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "p2r_internal.h"
#include "p2r_math.cuh"

namespace p2r {

struct FwdParams {
  const float* trk_in;
  const float* hits;
  float* trk_out;
  float* chi2;            // nullable, one per track
  const float* dr;        // nullable, nlayer
  const int32_t* nlay;    // nullable, one per track (masked mode)
  long long nblocks;
  int bsize;
  int nlayer;
  float kfact;
  int squash;             // wrap phi after every update (P2R_FLAG_SQUASH_PHI)
};

constexpr int kTrkWords = 28;
constexpr int kHitWords = 9;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Copies the warp's 32-lane slice of one MPHIT block (9 rows x 128 B) into a 288-float
// smem stage: 72 chunks of 16 B, lane j takes chunks j, j+32 and (j < 8) j+64.
__device__ __forceinline__ void stage_hit_slice(float* stage, const float* hit_slice, int bs, int lane) {
#pragma unroll
  for (int rep = 0; rep < 3; ++rep) {
    const int q = lane + 32 * rep;
    if (q < 72) {
      const int comp = q >> 3, sub = q & 7;
      cp_async16(stage + comp * 32 + sub * 4, hit_slice + (size_t)comp * bs + sub * 4);
    }
  }
}

__device__ __forceinline__ void load_track(const float* blk, int bs, int it, float (&par)[6], float (&cov)[21], int& q) {
#pragma unroll
  for (int i = 0; i < 6; ++i) par[i] = __ldg(blk + i * bs + it);
#pragma unroll
  for (int i = 0; i < 21; ++i) cov[i] = __ldg(blk + (6 + i) * bs + it);
  q = __float_as_int(__ldg(blk + 27 * bs + it));
}

__device__ __forceinline__ void store_track(float* blk, int bs, int it, const float (&par)[6], const float (&cov)[21], int q) {
#pragma unroll
  for (int i = 0; i < 6; ++i) __stcs(blk + i * bs + it, par[i]);
#pragma unroll
  for (int i = 0; i < 21; ++i) __stcs(blk + (6 + i) * bs + it, cov[i]);
  __stcs(blk + 27 * bs + it, __int_as_float(q));
}

// One warp's 32-lane slice of one Matriplex block through its layers, chained, with the
// hits staged per warp through the cp.async ring `ring` (STAGES x 288 floats of shared
// memory). Lane `lane` owns lane `it` of block `b`; lanes run layers [0, nlay) (MASK: the
// per-track count, else p.nlayer) and the warp iterates to its largest count. All 32 lanes
// must call it together (bs % 32 == 0).
template <int BS, int STAGES, bool CHI2, bool DR, bool MASK, bool FP64DET, bool SQUASH>
__device__ __forceinline__ void chained_slice_staged(const FwdParams& p, long long b, int it, int lane, float* ring) {
  const int bs = BS > 0 ? BS : p.bsize;
  float par[6], cov[21];
  int q;
  load_track(p.trk_in + b * (long long)(kTrkWords * bs), bs, it, par, cov, q);
  const float k = (float)q * p.kfact;
  const float kinv = 1.f / k;
  int nl = p.nlayer;
  if (MASK) nl = min(nl, max(0, p.nlay[b * bs + it]));
  const int nl_warp = MASK ? __reduce_max_sync(0xffffffffu, nl) : nl;
  const float* slice = p.hits + b * (long long)p.nlayer * (kHitWords * bs) + (it - lane);
  const long long lstride = (long long)kHitWords * bs;
  float chi2 = 0.f;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nl_warp) stage_hit_slice(ring + s * 288, slice + s * lstride, bs, lane);
    cp_async_commit();
  }
  for (int l = 0; l < nl_warp; ++l) {
    const int ln = l + STAGES - 1;
    if (ln < nl_warp) stage_hit_slice(ring + (ln % STAGES) * 288, slice + ln * lstride, bs, lane);
    cp_async_commit();
    cp_async_wait<STAGES - 1>();
    __syncwarp();
    const float* st = ring + (l % STAGES) * 288;
    float hp[3], hc[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) hp[i] = st[i * 32 + lane];
#pragma unroll
    for (int i = 0; i < 6; ++i) hc[i] = st[(3 + i) * 32 + lane];
    __syncwarp();  // the stage may be refilled from the next iteration on
    if (!MASK || l < nl) {
      const float rh = hipo(hp[0], hp[1]);
      const float rt = DR ? rh + __ldg(p.dr + l) : rh;
      propagate_to_r(par, cov, k, kinv, rt, par, cov);
      chi2 += kalman_update<FP64DET, CHI2>(par, cov, hp, hc, rh);
      if (SQUASH) par[4] = squash_phi(par[4]);
    }
  }
  cp_async_wait<0>();
  __syncwarp();  // no lane reuses the ring before every lane's copies have landed
  store_track(p.trk_out + b * (long long)(kTrkWords * bs), bs, it, par, cov, q);
  if (CHI2) p.chi2[b * bs + it] = chi2;
}

// BS: compile-time bsize (0 = run-time p.bsize). STAGED requires bsize % 32 == 0.
template <int BS, int STAGES, bool STAGED, bool RESTART, bool CHI2, bool DR, bool MASK, bool FP64DET, bool SQUASH>
__global__ void __launch_bounds__(128) fwd_kernel(FwdParams p) {
  extern __shared__ __align__(16) float smem[];
  const int bs = BS > 0 ? BS : p.bsize;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long b = g / bs;
  const int it = (int)(g - b * bs);
  if (b >= p.nblocks) return;  // with STAGED whole warps leave together (bs % 32 == 0)

  float par[6], cov[21];
  int q;
  load_track(p.trk_in + b * (long long)(kTrkWords * bs), bs, it, par, cov, q);
  const float k = (float)q * p.kfact;
  const float kinv = 1.f / k;
  int nl = p.nlayer;
  if (MASK) nl = min(nl, max(0, p.nlay[b * bs + it]));
  int nl_warp = nl;
  if (MASK && STAGED) nl_warp = __reduce_max_sync(0xffffffffu, nl);
  const float* hblk = p.hits + b * (long long)p.nlayer * (kHitWords * bs);
  float chi2 = 0.f;

  if (RESTART) {
    // Only the last layer reaches the output (TBB:894 rewrites the output each layer).
    if (nl > 0) {
      const int l = nl - 1;
      const float* h = hblk + (long long)l * (kHitWords * bs);
      float hp[3], hc[6];
#pragma unroll
      for (int i = 0; i < 3; ++i) hp[i] = __ldcs(h + i * bs + it);
#pragma unroll
      for (int i = 0; i < 6; ++i) hc[i] = __ldcs(h + (3 + i) * bs + it);
      const float rh = hipo(hp[0], hp[1]);
      const float rt = DR ? rh + __ldg(p.dr + l) : rh;
      float op[6], oc[21];
      propagate_to_r(par, cov, k, kinv, rt, op, oc);
      chi2 += kalman_update<FP64DET, CHI2>(op, oc, hp, hc, rh);
      if (SQUASH) op[4] = squash_phi(op[4]);
#pragma unroll
      for (int i = 0; i < 6; ++i) par[i] = op[i];
#pragma unroll
      for (int i = 0; i < 21; ++i) cov[i] = oc[i];
    }
  } else if (STAGED) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float* ring = smem + warp * (STAGES * 288);
    const float* slice = hblk + (it - lane);  // first lane of this warp within the block
    const long long lstride = (long long)kHitWords * bs;
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < nl_warp) stage_hit_slice(ring + s * 288, slice + s * lstride, bs, lane);
      cp_async_commit();
    }
    for (int l = 0; l < nl_warp; ++l) {
      const int ln = l + STAGES - 1;
      if (ln < nl_warp) stage_hit_slice(ring + (ln % STAGES) * 288, slice + ln * lstride, bs, lane);
      cp_async_commit();
      cp_async_wait<STAGES - 1>();
      __syncwarp();
      const float* st = ring + (l % STAGES) * 288;
      float hp[3], hc[6];
#pragma unroll
      for (int i = 0; i < 3; ++i) hp[i] = st[i * 32 + lane];
#pragma unroll
      for (int i = 0; i < 6; ++i) hc[i] = st[(3 + i) * 32 + lane];
      __syncwarp();  // the stage may be refilled from the next iteration on
      if (!MASK || l < nl) {
        const float rh = hipo(hp[0], hp[1]);
        const float rt = DR ? rh + __ldg(p.dr + l) : rh;
        propagate_to_r(par, cov, k, kinv, rt, par, cov);
        chi2 += kalman_update<FP64DET, CHI2>(par, cov, hp, hc, rh);
        if (SQUASH) par[4] = squash_phi(par[4]);
      }
    }
    cp_async_wait<0>();
  } else {
    for (int l = 0; l < nl; ++l) {
      const float* h = hblk + (long long)l * (kHitWords * bs);
      float hp[3], hc[6];
#pragma unroll
      for (int i = 0; i < 3; ++i) hp[i] = __ldcs(h + i * bs + it);
#pragma unroll
      for (int i = 0; i < 6; ++i) hc[i] = __ldcs(h + (3 + i) * bs + it);
      const float rh = hipo(hp[0], hp[1]);
      const float rt = DR ? rh + __ldg(p.dr + l) : rh;
      propagate_to_r(par, cov, k, kinv, rt, par, cov);
      chi2 += kalman_update<FP64DET, CHI2>(par, cov, hp, hc, rh);
      if (SQUASH) par[4] = squash_phi(par[4]);
    }
  }
  store_track(p.trk_out + b * (long long)(kTrkWords * bs), bs, it, par, cov, q);
  if (CHI2) p.chi2[b * bs + it] = chi2;
}

// ---------------------------------------------------------------- launch plumbing
template <int BS, int STAGES, bool STAGED, bool RESTART, bool CHI2, bool DR, bool MASK, bool FP64DET, bool SQUASH>
inline cudaError_t launch_fwd(const FwdParams& p, int threads, cudaStream_t st) {
  const long long ntr = p.nblocks * (long long)p.bsize;
  const long long grid = (ntr + threads - 1) / threads;
  const size_t smem = STAGED ? (size_t)(threads / 32) * STAGES * 288 * sizeof(float) : 0;
  auto kern = fwd_kernel<BS, STAGES, STAGED, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<(unsigned)grid, threads, smem, st>>>(p);
  return cudaGetLastError();
}

// compile-time bsize dispatch
template <int STAGES, bool STAGED, bool RESTART, bool CHI2, bool DR, bool MASK, bool FP64DET, bool SQUASH>
inline cudaError_t dispatch_bs(const FwdParams& p, int threads, cudaStream_t st) {
  switch (p.bsize) {
    case 32: return launch_fwd<32, STAGES, STAGED, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>(p, threads, st);
    case 64: return launch_fwd<64, STAGES, STAGED, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>(p, threads, st);
    case 128: return launch_fwd<128, STAGES, STAGED, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>(p, threads, st);
    default: return launch_fwd<0, STAGES, STAGED, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>(p, threads, st);
  }
}

template <bool STAGED, bool RESTART, bool CHI2, bool DR, bool MASK, bool FP64DET, bool SQUASH>
inline cudaError_t dispatch_stages(const FwdParams& p, int threads, int stages, cudaStream_t st) {
  if (!STAGED) return dispatch_bs<2, false, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>(p, threads, st);
  if (stages <= 2) return dispatch_bs<2, STAGED, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>(p, threads, st);
  return dispatch_bs<4, STAGED, RESTART, CHI2, DR, MASK, FP64DET, SQUASH>(p, threads, st);
}

// p.squash selects the SQUASH instances (compiled for the FP64 determinant only: a run-time
// branch in the layer loop costs ~4 % of the chained forward).
template <bool STAGED, bool RESTART, bool MASK>
inline cudaError_t dispatch_flags(const FwdParams& p, bool fp64det, int threads, int stages, cudaStream_t st) {
  const bool chi2 = p.chi2 != nullptr, dr = p.dr != nullptr, sq = p.squash != 0;
#define P2R_D(C, D, F, S)                        \
  if (chi2 == C && dr == D && fp64det == F && sq == S) \
    return dispatch_stages<STAGED, RESTART, C, D, MASK, F, S>(p, threads, stages, st);
  P2R_D(false, false, true, false)
  P2R_D(true, false, true, false)
  P2R_D(false, true, true, false)
  P2R_D(true, true, true, false)
  P2R_D(false, false, false, false)
  P2R_D(true, false, false, false)
  P2R_D(false, true, false, false)
  P2R_D(true, true, false, false)
  P2R_D(false, false, true, true)
  P2R_D(true, false, true, true)
  P2R_D(false, true, true, true)
  P2R_D(true, true, true, true)
#undef P2R_D
  return cudaErrorNotSupported;
}

// Launchers, one per translation unit.
cudaError_t launch_restart(const FwdParams& p, bool fp64det, int threads, int stages, cudaStream_t st);
cudaError_t launch_chained(const FwdParams& p, bool staged, bool fp64det, int threads, int stages, cudaStream_t st);
cudaError_t launch_masked(const FwdParams& p, bool staged, bool fp64det, int threads, int stages, cudaStream_t st);

}  // namespace p2r
