// Masked row traversal shared by the kernels that must reproduce the
// reference's per-lane association order over live entries
// (live_matrix.cuh:13-81 in the reference visits the same sequence).
#pragma once

#include "common.cuh"

namespace gpp {

// Visit the live entries of [first, last) so that the thread with index
// `lane` (0..W-1) sees live ranks lane, lane+W, ... in order.  `slots` is W
// ints of shared memory private to the warp (W=32) or block (W=256).
template <int W, class Visit>
__device__ __forceinline__ void live_visit(offset_t first, offset_t last, const int32_t* __restrict__ idx,
                                           const uint8_t* __restrict__ keep, int* slots,
                                           int* warp_counts, Visit visit) {
  const int lane = W == 32 ? (threadIdx.x & 31) : threadIdx.x;
  if (!keep) {
    for (offset_t p = first + lane; p < last; p += W) visit(p);
    return;
  }
  int carry = 0;
  for (offset_t chunk = first; chunk < last; chunk += W) {
    const offset_t p = chunk + lane;
    const bool live = p < last && keep[__ldcs(idx + p)];
    const unsigned mask = __ballot_sync(0xffffffffu, live);
    int rank = __popc(mask & ((1u << (threadIdx.x & 31)) - 1u));
    int c = __popc(mask);
    if constexpr (W == 256) {
      const int warp = threadIdx.x >> 5;
      if ((threadIdx.x & 31) == 0) warp_counts[warp] = c;
      __syncthreads();
      int before = 0, total = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) {
        const int k = warp_counts[w];
        before += w < warp ? k : 0;
        total += k;
      }
      rank += before;
      c = total;
    }
    if (live) slots[(carry + rank) & (W - 1)] = int(p - first);
    if constexpr (W == 32) __syncwarp(); else __syncthreads();
    if (((lane - carry) & (W - 1)) < c) visit(first + slots[lane]);
    if constexpr (W == 32) __syncwarp(); else __syncthreads();
    carry = (carry + c) & (W - 1);
  }
}

// The same traversal with liveness given per stored position: `all_live`
// when every entry of the range is live, else `live_at(p)`.
template <int W, class LiveAt, class Visit>
__device__ __forceinline__ void live_visit_by(offset_t first, offset_t last, bool all_live, LiveAt live_at,
                                              int* slots, int* warp_counts, Visit visit) {
  const int lane = W == 32 ? (threadIdx.x & 31) : threadIdx.x;
  if (all_live) {
    for (offset_t p = first + lane; p < last; p += W) visit(p);
    return;
  }
  int carry = 0;
  for (offset_t chunk = first; chunk < last; chunk += W) {
    const offset_t p = chunk + lane;
    const bool live = p < last && live_at(p);
    const unsigned mask = __ballot_sync(0xffffffffu, live);
    int rank = __popc(mask & ((1u << (threadIdx.x & 31)) - 1u));
    int c = __popc(mask);
    if constexpr (W == 256) {
      const int warp = threadIdx.x >> 5;
      if ((threadIdx.x & 31) == 0) warp_counts[warp] = c;
      __syncthreads();
      int before = 0, total = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) {
        const int k = warp_counts[w];
        before += w < warp ? k : 0;
        total += k;
      }
      rank += before;
      c = total;
    }
    if (live) slots[(carry + rank) & (W - 1)] = int(p - first);
    if constexpr (W == 32) __syncwarp(); else __syncthreads();
    if (((lane - carry) & (W - 1)) < c) visit(first + slots[lane]);
    if constexpr (W == 32) __syncwarp(); else __syncthreads();
    carry = (carry + c) & (W - 1);
  }
}

}  // namespace gpp
