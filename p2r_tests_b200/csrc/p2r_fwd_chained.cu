// Instantiations of the fused forward kernel: chained mode.
#include "p2r_fwd.cuh"

namespace p2r {

cudaError_t launch_chained(const FwdParams& p, bool staged, bool fp64det, int threads, int stages, cudaStream_t st) {
  return staged ? dispatch_flags<true, false, false>(p, fp64det, threads, stages, st)
                : dispatch_flags<false, false, false>(p, fp64det, threads, stages, st);
}

}  // namespace p2r
