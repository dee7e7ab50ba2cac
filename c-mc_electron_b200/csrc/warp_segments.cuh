// warp_segments.cuh -- sums over runs of equal keys within a warp.
//
// The particle store is counting-sorted by cell, so neighbouring lanes of a
// warp mostly hold particles of the same cell.  Before an int64 fixed-point
// tally goes to global memory, the lanes of each run of equal keys add
// their (already converted) integers with shuffles and only the run's last
// lane issues the atomic.  Integer addition is associative, so every sum is
// bit-identical to one atomic per lane; only the number of atomics drops.
#pragma once

#include <cuda_runtime.h>

namespace mcb200 {

struct WarpRuns {
  unsigned lane, head;  // this lane, the first lane of its run
  unsigned span;        // longest run in the warp
  bool tail;            // last lane of its run: issues the run's atomics

  // All 32 lanes must call this (and sum) together.
  __device__ __forceinline__ explicit WarpRuns(unsigned key) {
    lane = threadIdx.x & 31u;
    const unsigned prev = __shfl_up_sync(0xffffffffu, key, 1);
    const unsigned next = __shfl_down_sync(0xffffffffu, key, 1);
    const bool is_head = lane == 0 || prev != key;
    tail = lane == 31 || next != key;
    const unsigned heads = __ballot_sync(0xffffffffu, is_head);
    head = 31u - __clz(heads & (0xffffffffu >> (31u - lane)));
    span = __reduce_max_sync(0xffffffffu, lane - head + 1u);
  }
  // Inclusive sum over the run up to this lane; the tail lane holds the run's total.
  __device__ __forceinline__ long long sum(long long v) const {
    for (unsigned o = 1; o < span; o <<= 1) {
      const long long u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= head + o) v += u;
    }
    return v;
  }
};

}  // namespace mcb200
