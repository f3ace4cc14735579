// Internal helpers shared by the library's translation units (not part of the ABI).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <initializer_list>

#include <cuda_runtime_api.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/p2r.h"

// Records `msg` as the calling thread's last error and returns `code`.
int p2r_set_error(int code, const char* msg);
// printf-style variant.
int p2r_set_errorf(int code, const char* fmt, ...);
// Clears the calling thread's last error; returns P2R_OK.
int p2r_clear_error();

// Validates the sizes of a p2r_config; returns P2R_OK or P2R_ERR_INVALID with a message.
int p2r_check_config(const p2r_config* cfg, const char* who);

// P2R_ERR_INVALID unless every non-null pointer in `ptrs` is a multiple of `align` bytes. The
// kernels read and write device arrays as 4-byte (8-byte for double and 64-bit counters) words;
// a misaligned address would fault the kernel, so it is rejected on the host instead.
int p2r_check_aligned(const char* who, unsigned align, std::initializer_list<const void*> ptrs);

// P2R_ERR_INVALID when the byte ranges [a, a + na) and [b, b + nb) share a byte, naming them
// by `what`. A written array that overlaps another array of the same launch would let one
// track's writes land in another track's inputs. With allow_same, a = b with na = nb is
// accepted: in-place use, where every thread reads and writes only its own track's words.
// Null pointers and empty ranges overlap nothing.
int p2r_check_disjoint(const char* who, const char* what, const void* a, size_t na, const void* b, size_t nb,
                       bool allow_same = false);

// One array argument of a launch: its name, first byte, size in bytes, and whether the launch
// writes it.
struct P2rSpan {
  const char* name;
  const void* ptr;
  size_t bytes;
  bool written;
};

// P2R_ERR_INVALID when a written array shares a byte with any other array of the same launch
// (written or read), naming the pair. Null pointers and empty ranges overlap nothing.
int p2r_check_spans(const char* who, std::initializer_list<P2rSpan> spans);

// Names an entry point's span on a profiler's host timeline (an NVTX range: header-only, a
// no-op unless a tool such as Nsight Systems or Nsight Compute is attached).
struct P2rRange {
  explicit P2rRange(const char* name) { nvtxRangePushA(name); }
  ~P2rRange() { nvtxRangePop(); }
  P2rRange(const P2rRange&) = delete;
  P2rRange& operator=(const P2rRange&) = delete;
};

// Validates a p2r_queue description's sizes and options on the host (not its device arrays,
// which the kernels check); returns P2R_OK or an error status with a message.
int p2r_check_queue(const p2r_queue* q, const char* who);

// A captured launch sequence (p2r_queue_graph_create, p2r_queue_adjoint_graph_create).
struct p2r_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

// kfact exactly as the reference rounds it (TBB:654); bz == 0 means 3.8112 T.
float p2r_kfact_of(double bz);
