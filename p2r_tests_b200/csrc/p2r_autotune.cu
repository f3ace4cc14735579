// Native timing core of the autotuner: runs p2r_forward over candidate launch shapes
// (threads per CTA x hit-staging depth) on the caller's arrays and returns the fastest.
// Timing: CUDA events on the caller's stream, one warm-up launch per candidate, then
// `reps` launches; the reported time is the mean. Allocates no device memory.
#include <cuda_runtime.h>

#include <cfloat>

#include "p2r_internal.h"

extern "C" int p2r_autotune_forward(const p2r_config* cfg, const void* trk_in, const void* hits, void* trk_out,
                                    const int32_t* threads, int32_t n_threads, const int32_t* stages,
                                    int32_t n_stages, int32_t reps, p2r_tune_result* out, void* stream) {
  if (!cfg || !threads || !stages || !out || n_threads < 1 || n_stages < 1 || reps < 1)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_autotune_forward: bad arguments");
  P2rRange range("p2r_autotune_forward");
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return p2r_set_errorf(P2R_ERR_CUDA, "p2r_autotune_forward: %s", cudaGetErrorString(e));
  }
  out->best_ms = FLT_MAX;
  out->block_threads = 0;
  out->stages = 0;
  out->n_tried = 0;
  int rc = P2R_OK;
  for (int i = 0; i < n_threads && rc == P2R_OK; ++i)
    for (int j = 0; j < n_stages && rc == P2R_OK; ++j) {
      p2r_config c = *cfg;
      c.block_threads = threads[i];
      c.stages = stages[j];
      rc = p2r_forward(&c, trk_in, hits, trk_out, nullptr, nullptr, stream);
      if (rc) break;
      if ((e = cudaEventRecord(e0, st)) != cudaSuccess) {
        rc = p2r_set_errorf(P2R_ERR_CUDA, "p2r_autotune_forward: %s", cudaGetErrorString(e));
        break;
      }
      for (int r = 0; r < reps && rc == P2R_OK; ++r) rc = p2r_forward(&c, trk_in, hits, trk_out, nullptr, nullptr, stream);
      if (rc) break;
      float ms = 0.f;
      if ((e = cudaEventRecord(e1, st)) != cudaSuccess || (e = cudaEventSynchronize(e1)) != cudaSuccess ||
          (e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) {
        rc = p2r_set_errorf(P2R_ERR_CUDA, "p2r_autotune_forward: %s", cudaGetErrorString(e));
        break;
      }
      ms /= reps;
      if (out->n_tried < 64) {
        out->tried_threads[out->n_tried] = threads[i];
        out->tried_stages[out->n_tried] = stages[j];
        out->tried_ms[out->n_tried] = ms;
      }
      out->n_tried++;
      if (ms < out->best_ms) {
        out->best_ms = ms;
        out->block_threads = threads[i];
        out->stages = stages[j];
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc ? rc : p2r_clear_error();
}
