// Persistent work-queue launch for uneven batches: events with different track counts
// (blocks padded to bsize, padding lanes carry zero layers) and tracks with different layer
// counts run in ONE launch. The reference has no such mode: it runs a fixed ntrks x nevts
// grid (TBB:870-926) and silently drops ntrks % bsize tracks (nb = ntrks/bsize, TBB:22).
//
// Work items are (event, first block, block count) ranges planned on the host. A grid of
// (SMs x resident CTAs) CTAs pulls items from an atomic counter; each warp of a CTA takes
// 32-lane slices of the item's blocks and runs them with the chained staged body of the
// fused forward. When the last slice of an event finishes, its warp records %globaltimer
// into event_done_ns[event], giving per-event completion times. No thread waits on another
// (items are claimed with one atomicAdd), so there is no spin loop to bound. Items and event
// offsets are device data: each is range-checked on the device before use, and a bad one is
// skipped and recorded in an error word of the workspace (read by p2r_queue_error).
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <new>

#include "p2r_fwd.cuh"
#include "p2r_fwd_ordered.cuh"
#include "p2r_internal.h"
#include "p2r_queue_check.cuh"

namespace p2r {

struct QueueParams {
  FwdParams f;  // arrays, bsize, nlayer (= layer slots per block), kfact; f.nlay per lane
  const p2r_queue_item* items;
  long long n_items;
  int* counter;                 // next item
  int* ev_remaining;            // slices left per event
  const int64_t* ev_off;        // event block offsets (nevts + 1)
  long long nevts;
  unsigned* error;              // P2R_QERR_* bits of items that were skipped
  unsigned long long* ev_done;  // nullable
  unsigned long long* t_start;  // nullable
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void queue_init_kernel(const int64_t* ev_off, long long nevts, long long nblocks, int slices_per_block,
                                  int* counter, int* ev_remaining, unsigned* error, unsigned long long* t_start) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e == 0) {
    *counter = 0;
    if (t_start) *t_start = ULLONG_MAX;
  }
  if (e < nevts) {
    const long long b0 = ev_off[e], b1 = ev_off[e + 1];
    const long long n = (b1 - b0) * slices_per_block;
    if (b0 < 0 || b1 < b0 || b1 > nblocks || n > INT_MAX) {
      atomicOr(error, kQerrOffsets);
      ev_remaining[e] = 0;
    } else {
      ev_remaining[e] = (int)n;
    }
  }
}

template <int BS, int STAGES, bool CHI2, bool FP64DET, bool SQUASH>
__global__ void __launch_bounds__(128) queue_kernel(QueueParams q) {
  extern __shared__ __align__(16) float smem[];
  __shared__ int s_item;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int bs = BS > 0 ? BS : q.f.bsize;
  const int spb = bs / 32;  // 32-lane slices per block
  float* ring = smem + warp * (STAGES * 288);
  if (threadIdx.x == 0 && q.t_start) atomicMin(q.t_start, globaltimer_ns());
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(q.counter, 1);
    __syncthreads();
    const long long item = s_item;
    __syncthreads();  // every thread has read s_item before thread 0 claims the next one
    if (item >= q.n_items) break;
    const p2r_queue_item qi = q.items[item];
    // the items are device data the host did not re-read: an item outside the arrays is
    // skipped and reported (p2r_queue_error), never indexed
    const unsigned bad = queue_item_error(qi, q.nevts, q.f.nblocks, q.ev_off);
    if (bad) {
      if (threadIdx.x == 0) atomicOr(q.error, bad);
      continue;
    }
    const int nslices = qi.nblk * spb;
    for (int s = warp; s < nslices; s += nwarps) {
      const long long b = qi.block0 + s / spb;
      const int it = (s % spb) * 32 + lane;
      chained_slice_staged<BS, STAGES, CHI2, false, true, FP64DET, SQUASH>(q.f, b, it, lane, ring);
      if (lane == 0) {
        __threadfence();
        if (atomicSub(&q.ev_remaining[qi.event], 1) == 1 && q.ev_done) q.ev_done[qi.event] = globaltimer_ns();
      }
    }
  }
}

// ---------------------------------------------------------------- ordered variant
// The same queue with each item's blocks run in chunks whose tracks are ordered by layer count
// (P2R_FLAG_ORDER_BY_LAYERS; ordered_chunk in p2r_fwd_ordered.cuh).
template <int BS, int NW, bool CHI2, bool FP64DET, bool SQUASH>
__global__ void __launch_bounds__(NW * 32, kOrdWarpsPerSm / NW) queue_ordered_kernel(QueueParams q) {
  __shared__ OrdSmem<NW> sm;
  __shared__ long long s_item;
  const FwdParams& p = q.f;
  const int bs = BS > 0 ? BS : p.bsize;
  const int spb = bs / 32;
  const int cb = ordered_chunk_blocks<NW>(bs);
  const int tid = threadIdx.x;
  if (tid == 0 && q.t_start) atomicMin(q.t_start, globaltimer_ns());
  for (;;) {
    if (tid == 0) s_item = atomicAdd(q.counter, 1);
    __syncthreads();
    const long long item = s_item;
    __syncthreads();  // every thread has read s_item before thread 0 claims the next one
    if (item >= q.n_items) break;
    const p2r_queue_item qi = q.items[item];
    const unsigned bad = queue_item_error(qi, q.nevts, p.nblocks, q.ev_off);
    if (bad) {
      if (tid == 0) atomicOr(q.error, bad);
      continue;
    }
    for (int c0 = 0; c0 < qi.nblk; c0 += cb) {
      const int nblk = min(cb, qi.nblk - c0);
      ordered_chunk<BS, NW, CHI2, false, FP64DET, SQUASH>(p, qi.block0 + c0, nblk, sm);
      if (tid == 0) {
        __threadfence();
        if (atomicSub(&q.ev_remaining[qi.event], nblk * spb) == nblk * spb && q.ev_done)
          q.ev_done[qi.event] = globaltimer_ns();
      }
    }
  }
}

template <int BS, int NW, bool CHI2, bool FP64DET, bool SQUASH>
cudaError_t launch_queue_ordered_t(const QueueParams& q, int ctas_per_sm, cudaStream_t st) {
  constexpr int kOrdThreads = NW * 32;
  auto kern = queue_ordered_kernel<BS, NW, CHI2, FP64DET, SQUASH>;
  int dev = 0, sms = 0, occ = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kOrdThreads, 0);
  if (e != cudaSuccess) return e;
  const int per_sm = ctas_per_sm > 0 ? (ctas_per_sm < occ ? ctas_per_sm : occ) : occ;
  const long long want = (long long)sms * (per_sm > 0 ? per_sm : 1);
  const long long grid = want < q.n_items ? want : (q.n_items > 0 ? q.n_items : 1);
  kern<<<(unsigned)grid, kOrdThreads, 0, st>>>(q);
  return cudaGetLastError();
}

template <int NW, bool CHI2, bool FP64DET, bool SQUASH>
cudaError_t launch_queue_ordered_bs(const QueueParams& q, int ctas, cudaStream_t st) {
  switch (q.f.bsize) {
    case 32: return launch_queue_ordered_t<32, NW, CHI2, FP64DET, SQUASH>(q, ctas, st);
    case 64: return launch_queue_ordered_t<64, NW, CHI2, FP64DET, SQUASH>(q, ctas, st);
    case 128: return launch_queue_ordered_t<128, NW, CHI2, FP64DET, SQUASH>(q, ctas, st);
    default: return launch_queue_ordered_t<0, NW, CHI2, FP64DET, SQUASH>(q, ctas, st);
  }
}

template <int BS, int STAGES, bool CHI2, bool FP64DET, bool SQUASH>
cudaError_t launch_queue_t(const QueueParams& q, int threads, int ctas_per_sm, cudaStream_t st) {
  auto kern = queue_kernel<BS, STAGES, CHI2, FP64DET, SQUASH>;
  const size_t smem = (size_t)(threads / 32) * STAGES * 288 * sizeof(float);
  int dev = 0, sms = 0, occ = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
  if (e != cudaSuccess) return e;
  const int per_sm = ctas_per_sm > 0 ? (ctas_per_sm < occ ? ctas_per_sm : occ) : occ;
  const long long want = (long long)sms * (per_sm > 0 ? per_sm : 1);
  const long long grid = want < q.n_items ? want : (q.n_items > 0 ? q.n_items : 1);
  kern<<<(unsigned)grid, threads, smem, st>>>(q);
  return cudaGetLastError();
}

template <int STAGES, bool CHI2, bool FP64DET, bool SQUASH>
cudaError_t launch_queue_bs(const QueueParams& q, int threads, int ctas, cudaStream_t st) {
  switch (q.f.bsize) {
    case 32: return launch_queue_t<32, STAGES, CHI2, FP64DET, SQUASH>(q, threads, ctas, st);
    case 64: return launch_queue_t<64, STAGES, CHI2, FP64DET, SQUASH>(q, threads, ctas, st);
    case 128: return launch_queue_t<128, STAGES, CHI2, FP64DET, SQUASH>(q, threads, ctas, st);
    default: return launch_queue_t<0, STAGES, CHI2, FP64DET, SQUASH>(q, threads, ctas, st);
  }
}

}  // namespace p2r

using namespace p2r;

namespace {

struct QueueWs {
  size_t counter_off, error_off, start_off, remaining_off, bytes;
};

QueueWs queue_ws(int64_t nevts) {
  QueueWs w;
  w.counter_off = kQueueCounterOff;
  w.error_off = kQueueErrorOff;
  w.start_off = 256;
  w.remaining_off = 512;
  w.bytes = 512 + (((size_t)nevts * sizeof(int) + 255) & ~(size_t)255);
  return w;
}

}  // namespace

int p2r_check_queue(const p2r_queue* q, const char* who) {
  if (!q) return p2r_set_errorf(P2R_ERR_INVALID, "%s: queue is null", who);
  if (q->bsize < 32 || q->bsize % 32 != 0 || q->bsize > 4096)
    return p2r_set_errorf(P2R_ERR_QUEUE, "%s: bsize %d must be a multiple of 32", who, q->bsize);
  if (q->nlayer < 1 || q->nlayer > 4096) return p2r_set_errorf(P2R_ERR_QUEUE, "%s: nlayer %d", who, q->nlayer);
  if (q->nevts < 0 || q->nblocks < 0 || q->n_items < 0 || q->nevts > INT_MAX)
    return p2r_set_errorf(P2R_ERR_QUEUE, "%s: negative or too large sizes", who);
  if (q->n_items > INT_MAX - 65536) return p2r_set_errorf(P2R_ERR_QUEUE, "%s: too many work items", who);
  if (q->nblocks > 0 && (!q->event_block_offset || !q->items || !q->nlay_lane))
    return p2r_set_errorf(P2R_ERR_QUEUE, "%s: event offsets, items and layer counts are required", who);
  if (q->block_threads != 0 && (q->block_threads % 32 || q->block_threads > 128))
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: block_threads must be a multiple of 32 up to 128", who);
  if (q->stages != 0 && q->stages != 2 && q->stages != 4)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: stages must be 2 or 4", who);
  if (!std::isfinite(q->bz)) return p2r_set_errorf(P2R_ERR_INVALID, "%s: bz is not finite", who);
  if ((q->flags & P2R_FLAG_SQUASH_PHI) && (q->flags & P2R_FLAG_FP32_DET))
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED, "%s: P2R_FLAG_SQUASH_PHI is built with the FP64 determinant only", who);
  return P2R_OK;
}

namespace {

int enqueue_queue(const p2r_queue* q, const void* trk_in, const void* hits, void* trk_out, float* chi2_out,
                  unsigned long long* event_done_ns, unsigned long long* start_ns, void* workspace, size_t ws_bytes,
                  cudaStream_t st, const char* who) {
  P2rRange range(who);
  int rc = p2r_check_queue(q, who);
  if (rc) return rc;
  const bool ordered = (q->flags & P2R_FLAG_ORDER_BY_LAYERS) != 0;
  // ordered launches: 8 warps per CTA (block_threads 0) or 4 (block_threads 128)
  const int ord_warps = q->block_threads == 128 ? 4 : 8;
  if (ordered && (q->nlayer > kOrdMaxKeys - 1 || q->bsize > 64 * ord_warps ||
                  (q->block_threads != 0 && q->block_threads != 128)))
    return p2r_set_errorf(P2R_ERR_UNSUPPORTED,
                          "%s: P2R_FLAG_ORDER_BY_LAYERS needs nlayer <= %d, block_threads 0 (8 warps per CTA) or 128 "
                          "(4 warps), and bsize <= 64 x warps per CTA",
                          who, kOrdMaxKeys - 1);
  const QueueWs w = queue_ws(q->nevts);
  if (!workspace || ws_bytes < w.bytes)
    return p2r_set_errorf(P2R_ERR_WORKSPACE, "%s: workspace of %zu bytes needed", who, w.bytes);
  if (((uintptr_t)workspace & 255u) != 0) return p2r_set_errorf(P2R_ERR_INVALID, "%s: workspace must be 256-byte aligned", who);
  if (q->nevts == 0 || q->n_items == 0) return p2r_clear_error();
  if (!trk_in || !hits || !trk_out) return p2r_set_errorf(P2R_ERR_INVALID, "%s: null array pointer", who);
  if (((uintptr_t)hits & 15u) != 0) return p2r_set_errorf(P2R_ERR_INVALID, "%s: hits must be 16-byte aligned", who);
  if ((rc = p2r_check_aligned(who, 4, {trk_in, trk_out, chi2_out, q->nlay_lane})) ||
      (rc = p2r_check_aligned(who, 8, {event_done_ns, start_ns, q->event_block_offset, q->items})))
    return rc;
  {
    const size_t tb = (size_t)q->nblocks * 28 * q->bsize * sizeof(float);
    const size_t hb = (size_t)q->nblocks * q->nlayer * 9 * q->bsize * sizeof(float);
    const size_t lb = (size_t)q->nblocks * q->bsize * sizeof(float);
    const size_t ne = (size_t)q->nevts;
    if ((rc = p2r_check_spans(
             who, {{"trk_in", trk_in, tb, false},
                   {"hits", hits, hb, false},
                   {"nlay_lane", q->nlay_lane, lb, false},
                   {"event_block_offset", q->event_block_offset, (ne + 1) * sizeof(int64_t), false},
                   {"items", q->items, (size_t)q->n_items * sizeof(p2r_queue_item), false},
                   {"trk_out", trk_out, tb, true},
                   {"chi2_out", chi2_out, lb, true},
                   {"event_done_ns", event_done_ns, ne * sizeof(unsigned long long), true},
                   {"start_ns", start_ns, sizeof(unsigned long long), true},
                   {"workspace", workspace, ws_bytes, true}})))
      return rc;
  }
  QueueParams qp;
  qp.f.trk_in = (const float*)trk_in;
  qp.f.hits = (const float*)hits;
  qp.f.trk_out = (float*)trk_out;
  qp.f.chi2 = chi2_out;
  qp.f.dr = nullptr;
  qp.f.nlay = q->nlay_lane;
  qp.f.nblocks = q->nblocks;
  qp.f.bsize = q->bsize;
  qp.f.nlayer = q->nlayer;
  qp.f.kfact = p2r_kfact_of(q->bz);
  qp.f.squash = (q->flags & P2R_FLAG_SQUASH_PHI) != 0;
  qp.items = q->items;
  qp.n_items = q->n_items;
  qp.counter = (int*)((char*)workspace + w.counter_off);
  qp.t_start = start_ns;
  qp.ev_remaining = (int*)((char*)workspace + w.remaining_off);
  qp.ev_off = q->event_block_offset;
  qp.nevts = q->nevts;
  qp.error = (unsigned*)((char*)workspace + w.error_off);
  qp.ev_done = event_done_ns;
  // the error word is cleared before any kernel of this launch can set a bit
  cudaError_t e = cudaMemsetAsync(qp.error, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
  queue_init_kernel<<<(unsigned)((q->nevts + 255) / 256), 256, 0, st>>>(
      q->event_block_offset, q->nevts, q->nblocks, q->bsize / 32, qp.counter, qp.ev_remaining, qp.error, start_ns);
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    const int threads = q->block_threads > 0 ? q->block_threads : 128;
    const int stages = q->stages > 0 ? q->stages : 4;
    const bool fp64 = !(q->flags & P2R_FLAG_FP32_DET);
    const bool chi2 = chi2_out != nullptr;
    const int c = q->ctas_per_sm;
    if (qp.f.squash && !fp64) {
      e = cudaErrorNotSupported;  // rejected before launch in p2r_run_queue's checks
    } else if (ordered) {
#define P2R_O(W, C, F, Q) launch_queue_ordered_bs<W, C, F, Q>(qp, c, st)
      if (qp.f.squash)
        e = ord_warps == 4 ? (chi2 ? P2R_O(4, true, true, true) : P2R_O(4, false, true, true))
                           : (chi2 ? P2R_O(8, true, true, true) : P2R_O(8, false, true, true));
      else if (ord_warps == 4)
        e = chi2 ? (fp64 ? P2R_O(4, true, true, false) : P2R_O(4, true, false, false))
                 : (fp64 ? P2R_O(4, false, true, false) : P2R_O(4, false, false, false));
      else
        e = chi2 ? (fp64 ? P2R_O(8, true, true, false) : P2R_O(8, true, false, false))
                 : (fp64 ? P2R_O(8, false, true, false) : P2R_O(8, false, false, false));
#undef P2R_O
    } else if (qp.f.squash) {
      e = stages == 2 ? (chi2 ? launch_queue_bs<2, true, true, true>(qp, threads, c, st)
                              : launch_queue_bs<2, false, true, true>(qp, threads, c, st))
                      : (chi2 ? launch_queue_bs<4, true, true, true>(qp, threads, c, st)
                              : launch_queue_bs<4, false, true, true>(qp, threads, c, st));
    } else if (stages == 2) {
      e = chi2 ? (fp64 ? launch_queue_bs<2, true, true, false>(qp, threads, c, st)
                       : launch_queue_bs<2, true, false, false>(qp, threads, c, st))
               : (fp64 ? launch_queue_bs<2, false, true, false>(qp, threads, c, st)
                       : launch_queue_bs<2, false, false, false>(qp, threads, c, st));
    } else {
      e = chi2 ? (fp64 ? launch_queue_bs<4, true, true, false>(qp, threads, c, st)
                       : launch_queue_bs<4, true, false, false>(qp, threads, c, st))
               : (fp64 ? launch_queue_bs<4, false, true, false>(qp, threads, c, st)
                       : launch_queue_bs<4, false, false, false>(qp, threads, c, st));
    }
  }
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "%s: launch failed: %s", who, cudaGetErrorString(e));
  return p2r_clear_error();
}

}  // namespace

extern "C" {

int64_t p2r_queue_plan(const int64_t* host_event_block_offset, int64_t nevts, int32_t blocks_per_item,
                       p2r_queue_item* host_items, int64_t capacity) {
  if (!host_event_block_offset || nevts < 0 || blocks_per_item < 1)
    return -p2r_set_error(P2R_ERR_INVALID, "p2r_queue_plan: bad arguments");
  int64_t n = 0;
  for (int64_t e = 0; e < nevts; ++e) {
    const int64_t b0 = host_event_block_offset[e], b1 = host_event_block_offset[e + 1];
    if (b1 < b0) return -p2r_set_error(P2R_ERR_QUEUE, "p2r_queue_plan: event offsets must not decrease");
    for (int64_t b = b0; b < b1; b += blocks_per_item) {
      if (host_items) {
        if (n >= capacity) return -p2r_set_error(P2R_ERR_QUEUE, "p2r_queue_plan: item capacity exceeded");
        host_items[n].event = (int32_t)e;
        host_items[n].nblk = (int32_t)((b1 - b < blocks_per_item) ? (b1 - b) : blocks_per_item);
        host_items[n].block0 = b;
      }
      ++n;
    }
  }
  p2r_clear_error();
  return n;
}

size_t p2r_queue_workspace_size(const p2r_queue* q) {
  if (!q || q->nevts < 0) return 0;
  return queue_ws(q->nevts).bytes;
}

int p2r_queue_error(const void* workspace, uint32_t* host_bits, void* stream) {
  if (!workspace || !host_bits) return p2r_set_error(P2R_ERR_INVALID, "p2r_queue_error: null pointer");
  if (((uintptr_t)workspace & 255u) != 0)
    return p2r_set_error(P2R_ERR_INVALID, "p2r_queue_error: workspace must be 256-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  unsigned bits = 0u;
  cudaError_t e = cudaMemcpyAsync(&bits, (const char*)workspace + queue_ws(0).error_off, sizeof(bits),
                                  cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_queue_error: %s", cudaGetErrorString(e));
  *host_bits = bits;
  if (bits)
    return p2r_set_errorf(P2R_ERR_QUEUE,
                          "p2r_queue_error: work items were skipped (bits 0x%x: 1 event out of range, 2 blocks out "
                          "of range, 4 blocks outside the event's range, 8 bad event offsets)",
                          bits);
  return p2r_clear_error();
}

int p2r_run_queue(const p2r_queue* q, const void* trk_in, const void* hits, void* trk_out, float* chi2_out,
                  unsigned long long* event_done_ns, unsigned long long* start_ns, void* workspace, size_t ws_bytes,
                  void* stream) {
  return enqueue_queue(q, trk_in, hits, trk_out, chi2_out, event_done_ns, start_ns, workspace, ws_bytes,
                       (cudaStream_t)stream, "p2r_run_queue");
}

int p2r_queue_graph_create(const p2r_queue* q, const void* trk_in, const void* hits, void* trk_out, float* chi2_out,
                           unsigned long long* event_done_ns, unsigned long long* start_ns, void* workspace,
                           size_t ws_bytes, p2r_graph** out) {
  if (!out) return p2r_set_error(P2R_ERR_INVALID, "p2r_queue_graph_create: out is null");
  *out = nullptr;
  int rc = p2r_check_queue(q, "p2r_queue_graph_create");
  if (rc) return rc;
  cudaStream_t cs;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_queue_graph_create: %s", cudaGetErrorString(e));
  p2r_graph* g = new (std::nothrow) p2r_graph();
  if (!g) {
    cudaStreamDestroy(cs);
    return p2r_set_error(P2R_ERR_INVALID, "p2r_queue_graph_create: out of host memory");
  }
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = enqueue_queue(q, trk_in, hits, trk_out, chi2_out, event_done_ns, start_ns, workspace, ws_bytes, cs,
                       "p2r_queue_graph_create");
    cudaError_t e2 = cudaStreamEndCapture(cs, &g->graph);
    if (!rc && e2 != cudaSuccess) e = e2;
  }
  if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  cudaStreamDestroy(cs);
  if (rc || e != cudaSuccess) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return rc ? rc : p2r_set_errorf(P2R_ERR_CUDA, "p2r_queue_graph_create: %s", cudaGetErrorString(e));
  }
  *out = g;
  return p2r_clear_error();
}

int p2r_graph_launch(p2r_graph* g, void* stream) {
  if (!g || !g->exec) return p2r_set_error(P2R_ERR_INVALID, "p2r_graph_launch: null graph");
  cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  if (e != cudaSuccess) return p2r_set_errorf(P2R_ERR_CUDA, "p2r_graph_launch: %s", cudaGetErrorString(e));
  return p2r_clear_error();
}

int p2r_graph_destroy(p2r_graph* g) {
  if (!g) return P2R_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return p2r_clear_error();
}

}  // extern "C"
