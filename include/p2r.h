/*
 * p2r-b200: C ABI of the B200-native (sm_100a) track-propagation and Kalman-update path.
 *
 * Reference: cerati/p2r-tests, src/propagate-tor-test_tbb.cpp ("TBB" below). The
 * reference has no library interface: its per-block functions propagateToR (TBB:656-657)
 * and KalmanUpdate (TBB:433) are called by a driver loop (TBB:870-926) over caller-owned
 * Matriplex arrays. This header exposes the same arithmetic over the same arrays.
 *
 * Data layout (identical to the reference's structs, TBB:56-125, with bsize a run-time
 * value instead of a macro):
 *   MPTRK block = { float par[6*bsize]; float cov[21*bsize]; int32 q[bsize]; }  112*bsize B
 *   MPHIT block = { float pos[3*bsize]; float cov[6*bsize]; }                    36*bsize B
 *   element (lane it, component ip) of a block is data[it + ip*bsize].
 *   par = (x, y, z, 1/pT, phi, theta); symmetric matrices are packed lower-triangle
 *   row-major, (i >= j) -> i*(i+1)/2 + j (TBB:46-54).
 *   Track block of event ev, block ib:  tracks[ib + nb*ev]                (TBB:147-153)
 *   Hit block of layer lay:             hits[lay + ib*nlayer + ev*nlayer*nb] (TBB:215-217)
 *
 * Conventions: every pointer is a device pointer unless its name starts with host_;
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream); calls are
 * asynchronous and stream-ordered; nothing allocates device memory except where a
 * function says so. Device arrays must be aligned to their element size (4 bytes for the
 * float / int32 arrays, 8 for double and 64-bit ones; the hit array of the persistent queue to
 * 16): a misaligned pointer is rejected with P2R_ERR_INVALID before anything is launched.
 * Every function returns a p2r_status; p2r_last_error_string() gives
 * the message of the calling thread's last failure. No function aborts the process
 * (the reference aborts on CUDA errors, include/cudaCheck.h:17-58).
 */
#ifndef P2R_B200_H
#define P2R_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P2R_ABI_VERSION 1

typedef enum p2r_status {
  P2R_OK = 0,
  P2R_ERR_INVALID = 1,     /* bad argument: null pointer, size, alignment, mode */
  P2R_ERR_CUDA = 2,        /* a CUDA runtime call failed (message has the CUDA error) */
  P2R_ERR_TIMEOUT = 3,     /* a bounded device-side wait ran out */
  P2R_ERR_UNSUPPORTED = 4, /* valid request this build does not implement */
  P2R_ERR_WORKSPACE = 5,   /* workspace missing or too small */
  P2R_ERR_QUEUE = 6        /* malformed work-queue description */
} p2r_status;

/* Layer-loop semantics (both drive the same per-layer arithmetic):
 *  RESTART: every layer propagates the INPUT track to that layer's hit and updates the
 *           output, so only the last layer determines the result (TBB:880-911).
 *  CHAINED: the state is carried from layer to layer (a Kalman filter; the chained GPU
 *           variants, cuda_v4.cu:840-846). */
typedef enum p2r_mode { P2R_MODE_RESTART = 0, P2R_MODE_CHAINED = 1 } p2r_mode;

/* Option bits for p2r_config.flags. */
#define P2R_FLAG_FP32_DET 0x1u   /* 2x2 residual-covariance determinant in FP32 (default FP64, TBB:457) */
#define P2R_FLAG_NO_STAGING 0x2u /* read hits with plain loads instead of cp.async staging */
#define P2R_FLAG_ADJ_FP32 0x4u   /* p2r_forward_backward in FP32 instead of FP64 (faster, ~1e-2 gradients) */
#define P2R_FLAG_SQUASH_PHI 0x8u /* wrap phi into [-pi, pi] after every update: the step the reference
                                    leaves commented out (squashPhiMPlex, TBB:635); forward entry points,
                                    with the FP64 determinant (not with P2R_FLAG_FP32_DET) */
#define P2R_FLAG_ORDER_BY_LAYERS 0x10u /* with per-track layer counts: inside the launch, order the
                                    tracks by layer count (longest first, ties in track order) so a
                                    warp's lanes run tracks of similar length; outputs stay at each
                                    track's own position and every track's result is the same
                                    arithmetic (shared gradient sums are added in the new grouping).
                                    p2r_forward_masked (cfg.flags): within each CTA's chunk of 256 or
                                    512 tracks (FP64 determinant, nlayer <= 64, bsize <= 512); the
                                    forward queue (p2r_queue.flags): the same per chunk of an item;
                                    p2r_forward_backward (cfg.flags): within windows of 512 tracks of
                                    each event, 4 bytes of workspace per track; the queue adjoint
                                    (p2r_queue.flags): over whole events */

typedef struct p2r_config {
  int32_t bsize;         /* Matriplex lanes per block (TBB:15-17); >= 1 */
  int32_t nlayer;        /* hit blocks per track block (TBB:32-34); >= 1 */
  int64_t nevts;         /* events (TBB:24-26) */
  int64_t nb;            /* track blocks per event, ntrks/bsize (TBB:22) */
  double bz;             /* field [T]; kfact = float(100/(-0.299792458*bz)) (TBB:654); 0 -> 3.8112 */
  int32_t mode;          /* p2r_mode */
  uint32_t flags;        /* P2R_FLAG_* */
  int32_t block_threads; /* threads per CTA, multiple of 32 (0 = library default) */
  int32_t stages;        /* hit-staging pipeline depth, 2 or 4 (0 = library default, 4) */
} p2r_config;

/* Returns P2R_ABI_VERSION. */
int p2r_abi_version(void);

/* Message of the calling thread's last error ("" if none). */
const char* p2r_last_error_string(void);

/* kfact for a field of bz tesla, rounded to float as TBB:654 rounds its constant. */
float p2r_kfact(double bz);

/* ---------------------------------------------------------------- per-layer (drop-in)
 * Replaces one call of propagateToR(&in->cov, &in->par, &in->q, &hit->pos, &out->cov,
 * &out->par) (TBB:656-812, called at TBB:894) for EVERY block b in [0, nevts*nb):
 * in = trk_in[b], hit = hits[layer + b*nlayer], out = trk_out[b]. trk_out's q is copied
 * from trk_in. trk_in may equal trk_out (the chained drivers' in-place call,
 * cuda_v4.cu:843), but may not partly overlap it; trk_out may not overlap hits or dr.
 * dr (nullable, nlayer floats) adds dr[layer] cm to the target radius. */
int p2r_propagate_to_r(const p2r_config* cfg, const void* trk_in, const void* hits, int32_t layer,
                       void* trk_out, const float* dr, void* stream);

/* Replaces one call of KalmanUpdate(&trk->cov, &trk->par, &hit->cov, &hit->pos)
 * (TBB:433-642, called at TBB:911) for every block b: trk[b] updated in place with
 * hits[layer + b*nlayer]. chi2_accum (nullable, one float per track, track index
 * b*bsize + lane) gets the update's chi2 added (the reference's commented-out
 * Chi2Similarity, TBB:631). trk, hits and chi2_accum may not overlap. */
int p2r_kalman_update(const p2r_config* cfg, void* trk, const void* hits, int32_t layer, float* chi2_accum,
                      void* stream);

/* The reference's 3x3 gain routines, which it defines but never calls (its KalmanUpdate
 * measures two coordinates and inverts a 2x2):
 *   p2r_kalman_gain_inv replaces KalmanGainInv(&trk->cov, &hit->cov, &inv) (TBB:376-404) for
 *     every block b, hit = hits[layer + b*nlayer], writing one MP3x3 block (9*bsize floats,
 *     row-major 3x3 per lane) per track block to inv_out. Determinant and its reciprocal in
 *     double, as TBB:383-388.
 *   p2r_kalman_gain replaces KalmanGain(&trk->cov, &inv, &gain) (TBB:405-426), writing one
 *     MP3x6 block (18*bsize floats, row-major 6x3 per lane) per track block to gain_out.
 * Both read the packed covariances with the reference's own element choice: as if they were
 * packed upper-triangle row-major, whereas the arrays are packed lower-triangle (TBB:46-54),
 * so the 3x3 they invert is not the position block. The written array may not overlap the
 * others. */
int p2r_kalman_gain_inv(const p2r_config* cfg, const void* trk, const void* hits, int32_t layer, float* inv_out,
                        void* stream);
int p2r_kalman_gain(const p2r_config* cfg, const void* trk, const float* inv, float* gain_out, void* stream);

/* ---------------------------------------------------------------- fused driver
 * The whole driver loop (TBB:873-926 for one iteration) in one launch: every track runs
 * all nlayer (propagate, update) pairs with its state in registers, reading each hit once.
 * trk_out may not alias or overlap trk_in, and no written array (trk_out, chi2_out) may
 * overlap any other array of the call. chi2_out (nullable) receives the summed chi2 per track.
 * dr (nullable, nlayer floats) as in p2r_propagate_to_r. In RESTART mode only the last
 * layer determines the result (TBB:894 overwrites the output each layer), and only that
 * layer is computed. */
int p2r_forward(const p2r_config* cfg, const void* trk_in, const void* hits, void* trk_out, float* chi2_out,
                const float* dr, void* stream);

/* Chained forward over blocks whose lanes carry their own layer counts: lane `it` of
 * block b runs layers [0, nlay_lane[b*bsize + it]) (values 0..cfg->nlayer), then keeps
 * its state. The reference has no uneven-layer form; at nlay_lane[] == nlayer this equals
 * p2r_forward in CHAINED mode. */
int p2r_forward_masked(const p2r_config* cfg, const void* trk_in, const void* hits, void* trk_out,
                       const int32_t* nlay_lane, float* chi2_out, const float* dr, void* stream);

/* Number of tracks with a non-finite x, y, z, 1/pT, phi or theta among nblocks blocks
 * of trk (the reference's nnans, TBB:952-960), written to *count_out (device int64,
 * accumulated with atomics: zero it first). */
int p2r_count_nonfinite(const void* trk, int64_t nblocks, int32_t bsize, unsigned long long* count_out,
                        void* stream);

/* Host-buffer driver: p2r_forward over HOST arrays (host_trk_in, host_hits -> host_trk_out)
 * through caller-provided device arrays of the full size. Events are split into nchunks
 * contiguous chunks; each chunk's H2D copy, fused forward and D2H copy are queued on a
 * library-owned pool of three streams so copies overlap kernels (the reference's
 * multi-stream driver, cuda_v4.cu:912-1010). Ordered after prior work on `stream`, and
 * `stream` waits for all of it. Host arrays should be pinned for the copies to overlap.
 * The first call on a device creates the pool (streams and events, no device memory).
 * Calls from several host threads are serialised while they queue their work (the pool's
 * streams are shared), and the caller's stream waits for everything queued, also when a step
 * fails and an error is returned. In restart mode only the last layer's hit blocks are copied
 * (the only layer whose result reaches the output); the other layers' part of dev_hits is left
 * as it was. The three device arrays may not overlap. */
int p2r_forward_host(const p2r_config* cfg, const void* host_trk_in, const void* host_hits, void* host_trk_out,
                     void* dev_trk_in, void* dev_hits, void* dev_trk_out, int32_t nchunks, void* stream);

/* ---------------------------------------------------------------- uneven batches
 * Persistent work-queue launch (no counterpart in the reference, which runs a fixed
 * ntrks x nevts grid and drops ntrks % bsize tracks, TBB:22). Events own contiguous block
 * ranges [event_block_offset[e], event_block_offset[e+1]) of the MPTRK array; hits are
 * MPHIT blocks lay + b*nlayer as usual (nlayer = layer slots per block, the largest layer
 * count). Lane `it` of block b runs nlay_lane[b*bsize + it] layers (0 for padding lanes),
 * CHAINED. Work items (host-planned by p2r_queue_plan, copied to the device) are claimed
 * by a persistent grid with one atomic counter; no thread waits on another.
 * The items and event offsets are device data and are not re-read on the host: each item
 * must cover blocks [block0, block0 + nblk) inside [0, nblocks) and inside its event's range,
 * which p2r_queue_plan guarantees for non-decreasing offsets from 0 to nblocks. The kernels
 * check every item and offset on the device before using it: a bad item is skipped (its event
 * never completes) and recorded in the workspace, which p2r_queue_error reports. Layer counts
 * are clamped to [0, nlayer] on the device. */
typedef struct p2r_queue_item {
  int32_t event; /* event of the range */
  int32_t nblk;  /* blocks in the range */
  int64_t block0; /* first block */
} p2r_queue_item;

typedef struct p2r_queue {
  int32_t bsize;                     /* multiple of 32 */
  int32_t nlayer;                    /* layer slots per block (hit blocks per track block) */
  int64_t nevts;
  int64_t nblocks;                   /* total MPTRK blocks */
  double bz;                         /* field [T]; 0 -> 3.8112 */
  uint32_t flags;                    /* P2R_FLAG_FP32_DET */
  int32_t block_threads;             /* threads per CTA, 32..128 (0 = 128) */
  int32_t stages;                    /* hit-staging depth 2 or 4 (0 = 4) */
  int32_t ctas_per_sm;               /* resident CTAs per SM to launch (0 = occupancy limit) */
  const int64_t* event_block_offset; /* device, nevts + 1 */
  const p2r_queue_item* items;       /* device, n_items */
  int64_t n_items;
  const int32_t* nlay_lane;          /* device, nblocks * bsize */
} p2r_queue;

/* Splits every event's blocks into items of at most blocks_per_item blocks, in event order,
 * into host_items (capacity entries; NULL to only count). Returns the item count, or the
 * negated p2r_status on error. */
int64_t p2r_queue_plan(const int64_t* host_event_block_offset, int64_t nevts, int32_t blocks_per_item,
                       p2r_queue_item* host_items, int64_t capacity);

/* Device workspace for p2r_run_queue (item counter, per-event slice counters). */
size_t p2r_queue_workspace_size(const p2r_queue* q);

/* After a p2r_run_queue (or graph launch) on `stream` with this workspace: synchronises the
 * stream and returns P2R_ERR_QUEUE if the device skipped malformed work items or event offsets
 * (host_bits receives the reasons: 1 event outside [0, nevts), 2 blocks outside [0, nblocks),
 * 4 blocks outside the item's event range, 8 event offsets decreasing or outside [0, nblocks],
 * 16 a queue-adjoint track-order entry outside the batch),
 * P2R_OK otherwise. */
int p2r_queue_error(const void* workspace, uint32_t* host_bits, void* stream);

/* One persistent launch over all items (plus a small initialisation kernel). chi2_out
 * (nullable) per lane; event_done_ns (nullable, nevts) receives the %globaltimer value at
 * which each event's last slice finished; start_ns (nullable, 1) the earliest CTA start. */
int p2r_run_queue(const p2r_queue* q, const void* trk_in, const void* hits, void* trk_out, float* chi2_out,
                  unsigned long long* event_done_ns, unsigned long long* start_ns, void* workspace,
                  size_t workspace_bytes, void* stream);

/* The same launch sequence captured once into a CUDA graph (all pointers are baked in). */
typedef struct p2r_graph p2r_graph;
int p2r_queue_graph_create(const p2r_queue* q, const void* trk_in, const void* hits, void* trk_out, float* chi2_out,
                           unsigned long long* event_done_ns, unsigned long long* start_ns, void* workspace,
                           size_t workspace_bytes, p2r_graph** out);
int p2r_graph_launch(p2r_graph* g, void* stream);
int p2r_graph_destroy(p2r_graph* g);

/* ---------------------------------------------------------------- adjoint
 * Fused forward + hand-written adjoint of the CHAINED layer loop (no counterpart in the
 * reference, which has no derivatives). For the scalar
 *   L = sum over tracks of  g_out . out  +  g_chi2 * chi2,
 * out = the final parameters and covariance, chi2 = the summed chi2 of the track's updates
 * (the reference's commented-out Chi2Similarity, TBB:631), it writes:
 *   grad_trk_in   dL/d(initial par, cov)  (MPTRK layout, q row zero)       nullable
 *   grad_hits     dL/d(hit pos, hit cov)  (MPHIT layout, every layer)      nullable
 *   grad_dr       dL/d dr[layer], summed over tracks (nlayer doubles)     nullable
 *   grad_bz       dL/d Bz, summed over tracks (1 double)                 nullable
 *   grad_dr_event / grad_bz_event: the same per event ([nevts][nlayer], [nevts];
 *                 needs bsize % 32 == 0)                                    nullable
 * plus the forward outputs trk_out and chi2_out (nullable). grad_trk_out: cotangent of the
 * final state (MPTRK layout, par and cov rows; nullable = 0); grad_chi2: one per track
 * (nullable = 0). dr: radius offsets (nullable = 0); nlay_lane: per-track layer counts as
 * in p2r_forward_masked (nullable). The state is stored every ckpt_stride layers (1, 2, 4,
 * 5 or 10; 0 = 5) and the layers between checkpoints are recomputed. nlayer <= 64.
 * Arithmetic: FP64 throughout (state, trajectory, reverse), so gradients match FP64 finite
 * differences; its trk_out / chi2_out are that FP64 forward rounded to float (closer to the
 * exact result than p2r_forward's FP32 chain). cfg->flags & P2R_FLAG_ADJ_FP32 runs the same
 * kernel in FP32: several times faster, gradients accurate to ~1e-2 where chi2 enters.
 * workspace: device memory of at least p2r_forward_backward_workspace_size(cfg) bytes,
 * 256-byte aligned (per-warp partial sums of the shared gradients, reduced in a fixed order
 * in double, so results are deterministic). With the checkpoints held per thread, the
 * kernel keeps them in thread-local memory; a workspace of
 * p2r_forward_backward_workspace_size_tape(cfg, ckpt_stride) bytes also holds them, and the
 * recomputed segment states, as a tape in device memory ([slot][27][thread], 27*(nlayer /
 * ckpt_stride + ckpt_stride - 1) values per track), which runs the forward and the reverse
 * as two lighter kernels. Same results either way. */
size_t p2r_forward_backward_workspace_size(const p2r_config* cfg);
size_t p2r_forward_backward_workspace_size_tape(const p2r_config* cfg, int32_t ckpt_stride);
int p2r_forward_backward(const p2r_config* cfg, const void* trk_in, const void* hits, const float* dr,
                         const int32_t* nlay_lane, void* trk_out, float* chi2_out, const void* grad_trk_out,
                         const float* grad_chi2, void* grad_trk_in, void* grad_hits, double* grad_dr,
                         double* grad_bz, double* grad_dr_event, double* grad_bz_event, int32_t ckpt_stride,
                         void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free variant of p2r_forward_backward (no counterpart in the reference): the
 * same arguments without a workspace; the workspace is a fixed 8 MiB device array inside the
 * library, held by every GPU that loads it until the process exits. For callers that cannot
 * allocate device memory when they need gradients: code running while another framework
 * captures a CUDA graph, event loops that forbid allocation after start-up, plugin hosts whose
 * device memory belongs to the host framework's pool. Batches whose workspace
 * (p2r_forward_backward_workspace_size) exceeds 8 MiB are rejected with P2R_ERR_WORKSPACE
 * (about 1.5 M tracks at 20 layers, fewer with more layers or events). The array has its own
 * address in every CUDA context (each device's primary context, and any context a plugin
 * host creates and makes current): the first call in each context looks that address up
 * (cudaGetSymbolAddress, with the context current) and caches it under the context's unique
 * id; make that first call before any stream capture. Every call shares the array:
 * calls that overlap on the GPU race. Nothing in it needs clearing (each call writes
 * everything it reads). No cudaMalloc / cudaFree. */
int p2r_forward_backward_noalloc(const p2r_config* cfg, const void* trk_in, const void* hits, const float* dr,
                                 const int32_t* nlay_lane, void* trk_out, float* chi2_out, const void* grad_trk_out,
                                 const float* grad_chi2, void* grad_trk_in, void* grad_hits, double* grad_dr,
                                 double* grad_bz, double* grad_dr_event, double* grad_bz_event, int32_t ckpt_stride,
                                 void* stream);

/* Fused forward + adjoint of an uneven batch in ONE persistent launch over the work queue
 * (no counterpart in the reference): the batch, its events, work items and per-lane layer
 * counts are described by `q` as for p2r_run_queue; the arrays and the gradients are those of
 * p2r_forward_backward (FP64 throughout, the stride-1 structure: every layer's propagated state
 * is kept and the reverse starts each layer from it). Each warp keeps its slice's tape in its
 * own region of the workspace and reuses it slice after slice, so the workspace is bounded by
 * the resident warps, not by the batch: p2r_queue_adjoint_workspace_size(q) bytes (the slice
 * and event partial sums, plus nlayer*27*32 doubles per resident warp on the current device); a
 * smaller workspace runs fewer CTAs, at least one CTA's tapes is required. grad_dr_event /
 * grad_bz_event: the same per event. Shared gradients are summed in a fixed order (per 32-lane
 * slice, then per event, then in total): deterministic. Work items are checked on the device
 * (p2r_queue_error reads the result from this workspace too; bit 16: a track-order entry outside
 * the batch, which overlapping event ranges can cause). q->flags: 0 or P2R_FLAG_ORDER_BY_LAYERS
 * (the ordering runs inside the launch: a stable counting sort per event); other flags are
 * rejected (P2R_ERR_UNSUPPORTED). nlayer <= 64, bsize a multiple of 32. */
size_t p2r_queue_adjoint_workspace_size(const p2r_queue* q);
int p2r_run_queue_adjoint(const p2r_queue* q, const void* trk_in, const void* hits, const float* dr, void* trk_out,
                          float* chi2_out, const void* grad_trk_out, const float* grad_chi2, void* grad_trk_in,
                          void* grad_hits, double* grad_dr, double* grad_bz, double* grad_dr_event,
                          double* grad_bz_event, void* workspace, size_t workspace_bytes, void* stream);
/* The same launch sequence (workspace clears, the persistent kernel, the fixed-order sums)
 * captured once into a CUDA graph; replay with p2r_graph_launch. */
int p2r_queue_adjoint_graph_create(const p2r_queue* q, const void* trk_in, const void* hits, const float* dr,
                                   void* trk_out, float* chi2_out, const void* grad_trk_out, const float* grad_chi2,
                                   void* grad_trk_in, void* grad_hits, double* grad_dr, double* grad_bz,
                                   double* grad_dr_event, double* grad_bz_event, void* workspace,
                                   size_t workspace_bytes, p2r_graph** out);

/* ---------------------------------------------------------------- autotuning
 * Times p2r_forward on the caller's arrays for every (threads[i], stages[j]) pair
 * (CUDA events on `stream`, one warm-up launch then `reps` launches each) and reports the
 * fastest; synchronises the stream. The reference has no tuner (its sizes are macros). */
typedef struct p2r_tune_result {
  float best_ms;
  int32_t block_threads, stages, n_tried;
  int32_t tried_threads[64], tried_stages[64];
  float tried_ms[64];
} p2r_tune_result;

int p2r_autotune_forward(const p2r_config* cfg, const void* trk_in, const void* hits, void* trk_out,
                         const int32_t* threads, int32_t n_threads, const int32_t* stages, int32_t n_stages,
                         int32_t reps, p2r_tune_result* out, void* stream);

/* ---------------------------------------------------------------- measurement helper
 * FP32 FMA throughput probe (the denominator of the FP32 compute roofline): blocks x
 * threads threads each run 8 independent FMA chains for 4*iters rounds; FLOPs per launch
 * = 64 * iters * blocks * threads. out: blocks*threads floats. threads: 32..256. */
int p2r_fp32_fma_probe(int64_t iters, int32_t blocks, int32_t threads, float* out, void* stream);
/* The same probe with packed f32x2 FMAs (sm_100's two-lane form); same FLOPs per launch. */
int p2r_fp32x2_fma_probe(int64_t iters, int32_t blocks, int32_t threads, float* out, void* stream);
/* The same probe in FP64 (the denominator of the FP64 adjoint's roofline); same FLOPs per
 * launch, out: blocks*threads doubles. */
int p2r_fp64_fma_probe(int64_t iters, int32_t blocks, int32_t threads, double* out, void* stream);

/* The division / square-root build of the hot path (no reference counterpart; the reference
 * takes whatever its compiler flags give). P2R_MATH_REFINED: hardware reciprocal and
 * reciprocal square root refined by one Newton-Raphson step (the default build);
 * P2R_MATH_IEEE: correctly rounded; P2R_MATH_FAST: the approximations alone. */
enum p2r_math { P2R_MATH_REFINED = 0, P2R_MATH_IEEE = 1, P2R_MATH_FAST = 2 };
int32_t p2r_math_variant(void);

/* Evaluates the hot path's own division and square root elementwise on the device:
 * quot[i] = a[i] / b[i], root[i] = sqrt(a[i]), for measuring their error against the
 * correctly rounded results. Device pointers, n >= 0. */
int p2r_math_check(int64_t n, const float* a, const float* b, float* quot, float* root, void* stream);

/* ---------------------------------------------------------------- host-side helpers */

/* Parameters of the synthetic helix generator (p2r_gen_helix).
 * Track population: true helices from the origin with pT = pt*(1 + pop_smear*N(0,1)),
 * phi uniform in [-pi, pi], theta uniform in [theta_min, theta_max], charge +-1 with equal
 * probability; the seed is the true state where the helix crosses
 * r_seed*(1 + pop_smear*N(0,1)). The initial estimate handed to the filter is the seed
 * displaced by est_smear standard deviations of the diagonal seed covariance
 * (cov_pos for x, y, z; cov_ang for 1/pT, phi, theta). Hits: the helix crossing the
 * cylinders r_first..r_last (equally spaced), smeared by hit_sigma per coordinate, with
 * covariance hit_sigma^2 * I. */
typedef struct p2r_gen_params {
  uint64_t seed;
  double bz;                   /* field [T] */
  double r_seed;               /* nominal seed radius [cm] */
  double r_first, r_last;      /* hit cylinders [cm] */
  double pt;                   /* nominal pT [GeV] */
  double pop_smear;            /* relative Gaussian spread of pT and seed radius over the population */
  double theta_min, theta_max; /* polar-angle range [rad] */
  double cov_pos, cov_ang;     /* seed covariance diagonal [cm^2] and [GeV^-2, rad^2] */
  double est_smear;            /* displacement of the initial estimate, in seed-covariance sigmas */
  double hit_sigma;            /* hit smear per coordinate [cm] */
} p2r_gen_params;

/* Defaults: 3.8 T, seeds near r = 15 cm, hits on r = 20..100 cm, pT near 4 GeV, 10 %
 * population spread, theta 0.3..2.8, seed cov diag 1e-4 / 1e-3, estimates displaced by
 * one sigma draw, 10 um hits. */
void p2r_gen_params_default(p2r_gen_params* gp);

/* Fills HOST arrays host_trk (nevts*nb MPTRK blocks) and host_hits (nevts*nb*nlayer MPHIT
 * blocks), geometry in FP64 (see p2r_gen_params). ntrk_event (nullable, nevts entries):
 * tracks per event; lanes past it are padding and carry their undisplaced true seed.
 * Deterministic for a given seed and any nthreads (<= 0: all host threads). */
int p2r_gen_helix(const p2r_gen_params* gp, int32_t bsize, int64_t nevts, int64_t nb, int32_t nlayer,
                  const int32_t* ntrk_event, void* host_trk, void* host_hits, int32_t nthreads);

/* The same generator on the device: DEVICE arrays trk_out / hits_out, ntrk_event a DEVICE
 * pointer (nullable), stream-ordered. Same random streams and arithmetic as p2r_gen_helix;
 * the outputs equal its outputs bit for bit except for rare 1-ulp differences where the
 * device and host transcendental functions round differently. No reference counterpart
 * (the reference generates its inputs on the host, TBB:243-293). */
int p2r_gen_helix_device(const p2r_gen_params* gp, int32_t bsize, int64_t nevts, int64_t nb, int32_t nlayer,
                         const int32_t* ntrk_event, void* trk_out, void* hits_out, void* stream);

/* The reference's input recipe (prepareTracks / prepareHits, TBB:243-293 with randn
 * TBB:127-145) on HOST arrays, from a caller-supplied seed track (par[6], cov[21], q) and
 * n_input_hits hits (pos[3], cov[6] each, in layer order). Draws from glibc rand() in the
 * reference's order; call srand(1) first to reproduce a fresh run of the reference. */
int p2r_gen_fixture(const float* seed_par6, const float* seed_cov21, int32_t seed_q, const float* hits_lx9,
                    int32_t n_input_hits, int32_t bsize, int64_t nevts, int64_t nb, int32_t nlayer, double smear,
                    void* host_trk, void* host_hits);

/* The reference's end-of-run validation summary (TBB:935-1048) over HOST output tracks,
 * against the last layer's unsmeared hit position host_hit_xyz[3]. */
typedef struct p2r_summary_stats {
  double avg_x, avg_y, avg_z, avg_r, avg_pt, avg_phi, avg_theta;
  double avg_dx, avg_dy, avg_dz, avg_dr;
  double std_x, std_y, std_z, std_r, std_dx, std_dy, std_dz, std_dr;
  int64_t nnans, nfail;
} p2r_summary_stats;

int p2r_summary(const void* host_trk, int32_t bsize, int64_t nevts, int64_t nb, const float* host_hit_xyz,
                p2r_summary_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* P2R_B200_H */
