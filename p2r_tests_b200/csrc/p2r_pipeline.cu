// Host-buffer driver: events split into chunks whose host->device copy, fused forward and
// device->host copy run on a small pool of streams, so the copies of one chunk overlap the
// kernel of another. This is the transfer pipeline of the reference's multi-stream CUDA
// driver (cuda_v4.cu:912-1010: per-stream cudaMemcpyAsync H2D, kernel, D2H), over the same
// Matriplex arrays. Events are contiguous in both arrays (track block ib + nb*ev, hit block
// lay + nlayer*(ib + nb*ev)), so a chunk of events is one contiguous byte range of each.
// In restart mode only the last layer reaches the output (the reference's restart loop
// rewrites it at every layer from the same input track), so only that layer's hit block of
// each track block is copied: one strided 2-D copy per chunk, a 1/nlayer share of the hits.
#include <cuda_runtime.h>

#include <mutex>

#include "p2r_internal.h"

namespace {

constexpr int kMaxDevices = 64;
constexpr int kPoolStreams = 3;

struct StreamPool {
  std::mutex mu;  // one call at a time enqueues on the pool (the fork / join events are shared)
  bool ready = false;
  cudaStream_t s[kPoolStreams];
  cudaEvent_t fork;
  cudaEvent_t join[kPoolStreams];
};

StreamPool g_pools[kMaxDevices];
std::mutex g_pool_mu;

int get_pool(StreamPool** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_forward_host: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return p2r_set_error(P2R_ERR_UNSUPPORTED, "p2r_forward_host: device index");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  StreamPool& p = g_pools[dev];
  if (!p.ready) {
    for (int i = 0; i < kPoolStreams; ++i) p.s[i] = nullptr, p.join[i] = nullptr;
    p.fork = nullptr;
    for (int i = 0; i < kPoolStreams && e == cudaSuccess; ++i) {
      e = cudaStreamCreateWithFlags(&p.s[i], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming);
    if (e != cudaSuccess) {  // release what was created, so a later call starts from nothing
      for (int i = 0; i < kPoolStreams; ++i) {
        if (p.join[i]) cudaEventDestroy(p.join[i]);
        if (p.s[i]) cudaStreamDestroy(p.s[i]);
      }
      if (p.fork) cudaEventDestroy(p.fork);
      return p2r_set_errorf(P2R_ERR_CUDA, "p2r_forward_host: %s", cudaGetErrorString(e));
    }
    p.ready = true;
  }
  *out = &p;
  return P2R_OK;
}

}  // namespace

extern "C" int p2r_forward_host(const p2r_config* cfg, const void* host_trk_in, const void* host_hits,
                                void* host_trk_out, void* dev_trk_in, void* dev_hits, void* dev_trk_out,
                                int32_t nchunks, void* stream) {
  P2rRange range("p2r_forward_host");
  int rc = p2r_check_config(cfg, "p2r_forward_host");
  if (rc) return rc;
  if (!host_trk_in || !host_hits || !host_trk_out || !dev_trk_in || !dev_hits || !dev_trk_out)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_forward_host: null pointer");
  if (nchunks < 1) return p2r_set_error(P2R_ERR_INVALID, "p2r_forward_host: nchunks must be >= 1");
  if ((rc = p2r_check_aligned("p2r_forward_host", 4, {dev_trk_in, dev_hits, dev_trk_out}))) return rc;
  if (cfg->nevts == 0 || cfg->nb == 0) return p2r_clear_error();
  {  // the copies write dev_trk_in and dev_hits, the kernels dev_trk_out: all three disjoint
    const size_t tb = (size_t)cfg->nevts * cfg->nb * 28 * cfg->bsize * sizeof(float);
    const size_t hb = (size_t)cfg->nevts * cfg->nb * cfg->nlayer * 9 * cfg->bsize * sizeof(float);
    if ((rc = p2r_check_disjoint("p2r_forward_host", "dev_trk_in and dev_trk_out", dev_trk_in, tb, dev_trk_out, tb)) ||
        (rc = p2r_check_disjoint("p2r_forward_host", "dev_hits and dev_trk_out", dev_hits, hb, dev_trk_out, tb)) ||
        (rc = p2r_check_disjoint("p2r_forward_host", "dev_trk_in and dev_hits", dev_trk_in, tb, dev_hits, hb)))
      return rc;
  }
  StreamPool* pool = nullptr;
  if ((rc = get_pool(&pool))) return rc;
  std::lock_guard<std::mutex> lk(pool->mu);
  const int64_t chunks = nchunks > cfg->nevts ? cfg->nevts : nchunks;
  const size_t trk_ev = (size_t)cfg->nb * 28 * cfg->bsize * sizeof(float);
  const size_t hit_ev = (size_t)cfg->nb * cfg->nlayer * 9 * cfg->bsize * sizeof(float);
  const size_t hit_blk = (size_t)9 * cfg->bsize * sizeof(float);  // one layer of one track block
  const size_t last = (size_t)(cfg->nlayer - 1) * hit_blk;          // offset of the last layer's block
  const bool restart = cfg->mode == P2R_MODE_RESTART;
  cudaStream_t caller = (cudaStream_t)stream;
  cudaError_t e = cudaEventRecord(pool->fork, caller);
  for (int i = 0; i < kPoolStreams && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(pool->s[i], pool->fork, 0);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_forward_host: %s", cudaGetErrorString(e));
  // the caller's stream waits for everything queued on the pool, also when a step fails
  auto join = [&]() {
    cudaError_t je = cudaSuccess;
    for (int i = 0; i < kPoolStreams && je == cudaSuccess; ++i) {
      je = cudaEventRecord(pool->join[i], pool->s[i]);
      if (je == cudaSuccess) je = cudaStreamWaitEvent(caller, pool->join[i], 0);
    }
    return je;
  };
  for (int64_t c = 0; c < chunks; ++c) {
    const int64_t ev0 = cfg->nevts * c / chunks, ev1 = cfg->nevts * (c + 1) / chunks;
    if (ev1 == ev0) continue;
    cudaStream_t s = pool->s[c % kPoolStreams];
    char* dti = (char*)dev_trk_in + ev0 * trk_ev;
    char* dh = (char*)dev_hits + ev0 * hit_ev;
    char* dto = (char*)dev_trk_out + ev0 * trk_ev;
    if ((e = cudaMemcpyAsync(dti, (const char*)host_trk_in + ev0 * trk_ev, (ev1 - ev0) * trk_ev,
                             cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = restart ? cudaMemcpy2DAsync(dh + last, (size_t)cfg->nlayer * hit_blk,
                                         (const char*)host_hits + ev0 * hit_ev + last, (size_t)cfg->nlayer * hit_blk,
                                         hit_blk, (size_t)(ev1 - ev0) * cfg->nb, cudaMemcpyHostToDevice, s)
                     : cudaMemcpyAsync(dh, (const char*)host_hits + ev0 * hit_ev, (ev1 - ev0) * hit_ev,
                                       cudaMemcpyHostToDevice, s)) != cudaSuccess)
    {
      join();
      return p2r_set_errorf(P2R_ERR_CUDA, "p2r_forward_host: H2D: %s", cudaGetErrorString(e));
    }
    p2r_config sub = *cfg;
    sub.nevts = ev1 - ev0;
    if ((rc = p2r_forward(&sub, dti, dh, dto, nullptr, nullptr, s))) {
      join();
      return rc;
    }
    if ((e = cudaMemcpyAsync((char*)host_trk_out + ev0 * trk_ev, dto, (ev1 - ev0) * trk_ev, cudaMemcpyDeviceToHost,
                             s)) != cudaSuccess) {
      join();
      return p2r_set_errorf(P2R_ERR_CUDA, "p2r_forward_host: D2H: %s", cudaGetErrorString(e));
    }
  }
  if ((e = join()) != cudaSuccess)
    return p2r_set_errorf(P2R_ERR_CUDA, "p2r_forward_host: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}
