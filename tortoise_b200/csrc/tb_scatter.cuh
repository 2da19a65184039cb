// tb_scatter.cuh -- warp-aggregated scatter-add of per-tuple results.
//
// Tuples are stored in the reference's enumeration order (sections of leg 0
// outermost), so consecutive lanes of a warp usually carry the same element
// of leg 0 (and often of leg 1).  A segmented warp scan over runs of equal
// keys sums those lanes first and one lane per run issues the FP64 atomic,
// which cuts the L2 atomic traffic that otherwise bounds batched launches.
// Correct for any key order: only lanes that are contiguous *and* equal are
// merged; everything else falls back to one atomic per lane.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tb {

// All 32 lanes must call this together.  key < 0 marks a lane with nothing
// to add.  dst is the lane's destination (3 consecutive doubles).
__device__ __forceinline__ void warp_scatter3(int64_t key, double* dst, double v0, double v1, double v2) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t kprev = __shfl_up_sync(full, key, 1);
    const bool head = (lane == 0) || (kprev != key);
    const unsigned heads = __ballot_sync(full, head);
    const unsigned le = (lane == 31) ? full : ((1u << (lane + 1)) - 1u);
    const int seg = __popc(heads & le);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double t0 = __shfl_up_sync(full, v0, d);
        const double t1 = __shfl_up_sync(full, v1, d);
        const double t2 = __shfl_up_sync(full, v2, d);
        const int sg = __shfl_up_sync(full, seg, d);
        if (lane >= d && sg == seg) { v0 += t0; v1 += t1; v2 += t2; }
    }
    const int snext = __shfl_down_sync(full, seg, 1);
    const bool tail = (lane == 31) || (snext != seg);
    if (tail && key >= 0) {
        atomicAdd(dst + 0, v0);
        atomicAdd(dst + 1, v1);
        atomicAdd(dst + 2, v2);
    }
}

}  // namespace tb
