// The fused chained forward over a chunk of blocks with the chunk's tracks ordered by layer
// count (P2R_FLAG_ORDER_BY_LAYERS), shared by the persistent queue (p2r_queue.cu, one chunk of
// an item at a time) and the masked fused forward (p2r_fwd_ordered.cu, one chunk per CTA).
//
// A CTA of NW warps (4 or 8) takes floor(64 NW / bsize) blocks, at most 64 NW tracks, and orders
// them by layer count (a stable counting sort in shared memory), so the 32 lanes of a warp run
// tracks of similar length and few lanes idle while a warp's longest track runs. The ordered
// tracks form 2 NW groups of 32; warp w runs group w and then group 2NW-1-w, one long and one
// short group, so the warps finish the chunk at about the same time and the CTA rarely holds a
// lone warp. A lane reads its own track's hits straight from the Matriplex rows (the chunk's
// blocks are shared by the CTA's warps through L1), the next layer's hits loaded while the
// current one computes; warps synchronise only at chunk boundaries. Per track the arithmetic is
// the masked forward's, in the same order: bit-identical results. nlayer <= 64 (the ordering
// keys), bsize <= 64 NW.
#pragma once

#include "p2r_fwd.cuh"

namespace p2r {

constexpr int kOrdMaxKeys = 65;

// Resident warps per SM the ordered kernels are compiled for (__launch_bounds__): 16, so a
// thread may hold 128 registers. A lane's next-layer hit loads are scattered (its track sits
// anywhere in the chunk) and come from DRAM more often than the staged rows of the unordered
// kernels; with registers to keep them in flight across a whole layer the launch runs faster
// than at 24 warps of 80 registers (measured on one B200, same results bit for bit: 1000-event
// uneven batch 1.297 -> 1.255 ms, 40-layer masked forward 7.86 -> 6.87 ms).
constexpr int kOrdWarpsPerSm = 16;

template <int NW>
struct OrdSmem {
  int order[2 * NW * 32];
  int wcount[NW][kOrdMaxKeys];
  int base[kOrdMaxKeys];
  int cnt[2][kOrdMaxKeys];
};

// Blocks per chunk for a CTA of NW warps.
template <int NW>
__host__ __device__ __forceinline__ int ordered_chunk_blocks(int bsize) {
  return (2 * NW * 32) / bsize;
}

// Runs blocks [b0, b0 + nblk) (nblk <= ordered_chunk_blocks<NW>(bsize)) with all NW warps of the
// CTA; returns after a barrier, when the shared memory may be reused.
template <int BS, int NW, bool CHI2, bool DR, bool FP64DET, bool SQUASH>
__device__ __forceinline__ void ordered_chunk(const FwdParams& p, long long b0, int nblk, OrdSmem<NW>& sm) {
  constexpr int kThreads = NW * 32;
  const int bs = BS > 0 ? BS : p.bsize;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nkeys = p.nlayer + 1;
  const unsigned lt = (1u << lane) - 1u;
  const long long lstride = (long long)kHitWords * bs;
  const int ntrk = nblk * bs;
  // ---- order the chunk's tracks: stable counting sort on key = nlayer - layers, over two passes
  // of NW*32 tracks (track t = pass * NW*32 + tid); a track's rank among equal keys comes from its
  // warp (__match_any_sync) and the warps before it, pass 1 after all of pass 0
  int keyv[2], rankv[2];
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    const int t = pass * kThreads + tid;
    int key = -1;
    if (t < ntrk) {
      const int v = p.nlay[(b0 + t / bs) * bs + t % bs];
      key = p.nlayer - min(p.nlayer, max(0, v));
    }
    const unsigned same = __match_any_sync(0xffffffffu, key);
    int r = __popc(same & lt);
    for (int j = lane; j < nkeys; j += 32) sm.wcount[warp][j] = 0;
    __syncwarp();
    if (key >= 0 && r == 0) sm.wcount[warp][key] = __popc(same);
    __syncthreads();
    if (key >= 0)
      for (int w = 0; w < warp; ++w) r += sm.wcount[w][key];
    if (tid < nkeys) {
      int tot = 0;
      for (int w = 0; w < NW; ++w) tot += sm.wcount[w][tid];
      sm.cnt[pass][tid] = tot;
    }
    keyv[pass] = key;
    rankv[pass] = r;
    __syncthreads();  // wcount is reused by the next pass
  }
  if (tid == 0) {  // first position of each key
    int run = 0;
    for (int k = 0; k < nkeys; ++k) {
      sm.base[k] = run;
      run += sm.cnt[0][k] + sm.cnt[1][k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    const int key = keyv[pass];
    if (key >= 0) sm.order[sm.base[key] + (pass ? sm.cnt[0][key] : 0) + rankv[pass]] = pass * kThreads + tid;
  }
  __syncthreads();
  // ---- two ordered groups per warp: group w (long tracks), then group 2NW-1-w (short)
  for (int half = 0; half < 2; ++half) {
    const int grp = half == 0 ? warp : 2 * NW - 1 - warp;
    const int pos = grp * 32 + lane;
    const bool mine = pos < ntrk;
    const int li = mine ? sm.order[pos] : 0;
    const int jb = li / bs, it = li - jb * bs;
    const long long b = b0 + jb;
    float par[6], cov[21];
    int qq = 1, nl = 0;
    if (mine) {
      load_track(p.trk_in + b * (long long)(kTrkWords * bs), bs, it, par, cov, qq);
      nl = min(p.nlayer, max(0, p.nlay[b * bs + it]));
    }
    const float k = (float)qq * p.kfact;
    const float kinv = 1.f / k;
    float chi2 = 0.f;
    const float* hb = p.hits + b * (long long)p.nlayer * lstride + it;
    float hn[9];
    if (nl > 0) {
#pragma unroll
      for (int i = 0; i < 9; ++i) hn[i] = __ldg(hb + i * bs);
    }
    for (int l = 0; l < nl; ++l) {
      float hp[3], hc[6];
#pragma unroll
      for (int i = 0; i < 3; ++i) hp[i] = hn[i];
#pragma unroll
      for (int i = 0; i < 6; ++i) hc[i] = hn[3 + i];
      if (l + 1 < nl) {  // the next layer's hit, in flight while this layer computes
#pragma unroll
        for (int i = 0; i < 9; ++i) hn[i] = __ldg(hb + (l + 1) * lstride + i * bs);
      }
      const float rh = hipo(hp[0], hp[1]);
      const float rt = DR ? rh + __ldg(p.dr + l) : rh;
      propagate_to_r(par, cov, k, kinv, rt, par, cov);
      chi2 += kalman_update<FP64DET, CHI2>(par, cov, hp, hc, rh);
      if (SQUASH) par[4] = squash_phi(par[4]);
    }
    if (mine) {
      store_track(p.trk_out + b * (long long)(kTrkWords * bs), bs, it, par, cov, qq);
      if (CHI2) p.chi2[b * bs + it] = chi2;
    }
  }
  __syncthreads();  // the order may be reused by the next chunk
}

// Launcher of the masked fused forward with in-launch ordering (p2r_fwd_ordered.cu): one chunk
// per CTA, ctas = ceil(nblocks / chunk). block_threads 128 -> 4 warps, else 8.
cudaError_t launch_ordered(const FwdParams& p, bool fp64det, int threads, cudaStream_t st);

}  // namespace p2r
