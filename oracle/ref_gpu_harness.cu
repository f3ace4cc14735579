// Reference GPU harness: compiles one of the reference's own CUDA programs UNMODIFIED, from
// where it lies in the reference checkout, and exposes its kernel through a small C ABI so the
// benchmark can time it with CUDA events on the same device-resident inputs as this library's
// kernel.
//
// TEST INFRASTRUCTURE ONLY (oracle). Built by oracle/Makefile into oracle/_ref/; only bench.py
// and tests/ load it, as a timed comparison point and as a checker, never as the product.
//
// Two programs, one library each (they define the same names):
//   P2R_REF_V4  src/propagate-tor-test_cuda_v4.cu: GPUsequence (cuda_v4.cu:821-849), the CHAINED
//               layer loop, one CTA of threadsperblockx (32) threads per Matriplex block, its
//               scratch matrices in shared memory.
//   P2R_REF_UVM src/propagate-tor-test_cuda_uvm.cu: launch_p2r_kernel (cuda_uvm.cu:887-915), the
//               RESTART layer loop (every layer starts from the input track and only the last
//               result is stored, so the compiler may drop the other layers), one thread per
//               track, grid-stride.
// Sizes are the programs' own compile-time macros (ntrks, nevts, nlayer, bsize), set by the
// Makefile to the benchmark workload; the arrays passed in must hold nevts*nb track blocks and
// nevts*nb*nlayer hit blocks in the Matriplex layout, which is the same in both programs and in
// this library.
// <array> is used by the uvm program without its own #include (older standard libraries
// pulled it in through other headers); it is included here first.
#include <array>

#define main p2r_ref_gpu_program_main
#include P2R_REF_CU
#undef main

#include <cuda_runtime.h>

namespace {

cudaError_t launch_once(const void* trk, const void* hit, void* out, cudaStream_t st) {
#if defined(P2R_REF_V4)
  // the program's own launch shape (cuda_v4.cu:890-891, 981), one stream
  GPUsequence<<<dim3(blockspergrid, 1, 1), dim3(threadsperblockx, 1, 1), 0, st>>>(
      (MPTRK*)trk, (MPHIT*)hit, (MPTRK*)out, 0);
#elif defined(P2R_REF_UVM)
  // the program's own launch shape (cuda_uvm.cu:975-979, 991)
  const int phys_length = nevts * nb;
  const int outer_loop_range = phys_length * bsize;
  launch_p2r_kernel<bsize, nlayer><<<dim3((outer_loop_range + threadsperblock - 1) / threadsperblock, 1, 1),
                                     dim3(threadsperblock, 1, 1), 0, st>>>((MPTRK*)out, (MPTRK*)trk, (MPHIT*)hit,
                                                                           outer_loop_range);
#else
#error "define P2R_REF_V4 or P2R_REF_UVM"
#endif
  return cudaGetLastError();
}

}  // namespace

extern "C" {

// The program's compile-time sizes: nevts, nb (= ntrks / bsize), nlayer, bsize.
void refgpu_sizes(long* n_evts, long* n_b, int* n_layer, int* b_size) {
  *n_evts = nevts;
  *n_b = nb;
  *n_layer = nlayer;
  *b_size = bsize;
}

// 1 for the chained program (v4), 0 for the restart program (uvm).
int refgpu_chained(void) {
#if defined(P2R_REF_V4)
  return 1;
#else
  return 0;
#endif
}

// `warmup` untimed launches, then `iters` launches between two CUDA events on `stream`
// (device pointers; out may not alias trk). *ms_total receives the event time of the `iters`
// launches. Returns 0, or the cudaError_t of the first failing call.
int refgpu_run(const void* trk, const void* hit, void* out, int warmup, int iters, void* stream, float* ms_total) {
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < warmup && e == cudaSuccess; ++i) e = launch_once(trk, hit, out, st);
  if (e != cudaSuccess) return (int)e;
  cudaEvent_t a, b;
  if ((e = cudaEventCreate(&a)) != cudaSuccess) return (int)e;
  if ((e = cudaEventCreate(&b)) != cudaSuccess) {
    cudaEventDestroy(a);
    return (int)e;
  }
  e = cudaEventRecord(a, st);
  for (int i = 0; i < iters && e == cudaSuccess; ++i) e = launch_once(trk, hit, out, st);
  if (e == cudaSuccess) e = cudaEventRecord(b, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms_total, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return (int)e;
}

}  // extern "C"
