// Instantiations of the fused forward kernel: restart mode.
#include "p2r_fwd.cuh"

namespace p2r {

cudaError_t launch_restart(const FwdParams& p, bool fp64det, int threads, int stages, cudaStream_t st) {
  return dispatch_flags<false, true, false>(p, fp64det, threads, stages, st);
}

}  // namespace p2r
