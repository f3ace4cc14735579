// Device-side checks of the persistent queue's work items, shared by the forward queue kernel
// (p2r_queue.cu) and the forward + adjoint queue kernel (p2r_adjoint.cu). The items and event
// offsets are device data the host did not re-read: a kernel checks each item before using it
// as an index, skips a bad one and ORs the reason into an error word that p2r_queue_error
// reads from the workspace.
#pragma once

#include <stdint.h>

#include "../../include/p2r.h"

namespace p2r {

constexpr unsigned kQerrEvent = 1u;       // an item's event outside [0, nevts)
constexpr unsigned kQerrBlocks = 2u;      // an item's blocks outside [0, nblocks) or nblk < 0
constexpr unsigned kQerrEventRange = 4u;  // an item's blocks outside its event's block range
constexpr unsigned kQerrOffsets = 8u;     // event offsets decreasing, outside [0, nblocks], or too large
constexpr unsigned kQerrOrder = 16u;      // a track order entry outside the batch (offsets that overlap)

// Byte offsets in every queue workspace: the item counter and the error word.
constexpr size_t kQueueCounterOff = 0;
constexpr size_t kQueueErrorOff = 128;

// 0 if item qi may be used (its blocks lie in [0, nblocks) and in its event's range), else the
// error bit. Reads ev_off only at indices the event check has put in range.
__device__ __forceinline__ unsigned queue_item_error(const p2r_queue_item& qi, long long nevts, long long nblocks,
                                                     const int64_t* ev_off) {
  if (qi.event < 0 || qi.event >= nevts) return kQerrEvent;
  if (qi.nblk < 0 || qi.block0 < 0 || qi.block0 > nblocks - qi.nblk) return kQerrBlocks;
  if (qi.block0 < ev_off[qi.event] || qi.block0 + qi.nblk > ev_off[qi.event + 1]) return kQerrEventRange;
  return 0u;
}

}  // namespace p2r
