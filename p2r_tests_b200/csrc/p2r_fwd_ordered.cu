// Masked fused forward with the tracks of each CTA's chunk ordered by layer count
// (P2R_FLAG_ORDER_BY_LAYERS with per-track layer counts): one chunk of floor(64 NW / bsize)
// blocks per CTA, see p2r_fwd_ordered.cuh. The FP64 determinant build only.
#include "p2r_fwd_ordered.cuh"

namespace p2r {

template <int BS, int NW, bool CHI2, bool DR, bool SQUASH>
__global__ void __launch_bounds__(NW * 32, kOrdWarpsPerSm / NW) fwd_ordered_kernel(FwdParams p) {
  __shared__ OrdSmem<NW> sm;
  const int bs = BS > 0 ? BS : p.bsize;
  const int cb = ordered_chunk_blocks<NW>(bs);
  const long long b0 = (long long)blockIdx.x * cb;
  const int nblk = (int)(p.nblocks - b0 < cb ? p.nblocks - b0 : cb);
  ordered_chunk<BS, NW, CHI2, DR, true, SQUASH>(p, b0, nblk, sm);
}

template <int BS, int NW, bool CHI2, bool DR, bool SQUASH>
cudaError_t launch_ordered_t(const FwdParams& p, cudaStream_t st) {
  const int cb = ordered_chunk_blocks<NW>(p.bsize);
  const long long grid = (p.nblocks + cb - 1) / cb;
  fwd_ordered_kernel<BS, NW, CHI2, DR, SQUASH><<<(unsigned)grid, NW * 32, 0, st>>>(p);
  return cudaGetLastError();
}

template <int NW, bool CHI2, bool DR, bool SQUASH>
cudaError_t launch_ordered_bs(const FwdParams& p, cudaStream_t st) {
  return p.bsize == 32 ? launch_ordered_t<32, NW, CHI2, DR, SQUASH>(p, st)
                       : launch_ordered_t<0, NW, CHI2, DR, SQUASH>(p, st);
}

template <int NW>
cudaError_t launch_ordered_nw(const FwdParams& p, cudaStream_t st) {
  const bool chi2 = p.chi2 != nullptr, dr = p.dr != nullptr, sq = p.squash != 0;
#define P2R_D(C, D, S) \
  if (chi2 == C && dr == D && sq == S) return launch_ordered_bs<NW, C, D, S>(p, st);
  P2R_D(false, false, false)
  P2R_D(true, false, false)
  P2R_D(false, true, false)
  P2R_D(true, true, false)
  P2R_D(false, false, true)
  P2R_D(true, false, true)
  P2R_D(false, true, true)
  P2R_D(true, true, true)
#undef P2R_D
  return cudaErrorNotSupported;
}

cudaError_t launch_ordered(const FwdParams& p, bool fp64det, int threads, cudaStream_t st) {
  if (!fp64det) return cudaErrorNotSupported;  // rejected on the host before the launch
  return threads == 128 ? launch_ordered_nw<4>(p, st) : launch_ordered_nw<8>(p, st);
}

}  // namespace p2r
