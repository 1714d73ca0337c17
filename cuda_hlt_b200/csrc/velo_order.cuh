// Launched between fill_candidates and search_by_triplet: the queue order of the warp search.
#pragma once
#include "velo_kernels.cuh"

namespace velo {

// Longest-processing-time-first order of the warp search's events. The search hands events
// out through an atomic queue, a few per warp in a batch, and its time per event spreads
// about tenfold with the occupancy, so large events that come last set the kernel's length.
// Taken largest first (counting sort on the cluster count in buckets of 16, one CTA), the
// small events fill the tail. The order within a bucket is free: every event's result is
// independent of when it runs.
constexpr uint32_t kOrderThreads = 1024;
constexpr uint32_t kOrderBuckets = kOrderThreads;
constexpr uint32_t kOrderShift = 4;

__global__ void __launch_bounds__(kOrderThreads) order_events_kernel(ChainPointers P)
{
  __shared__ uint32_t s_off[kOrderBuckets];
  __shared__ uint32_t s_warp[kOrderThreads / 32];
  const uint32_t n = P.queue[4];
  const uint32_t t = threadIdx.x, lane = t & 31u;
  auto bucket = [&](uint32_t e) {
    return kOrderBuckets - 1u - min(P.event_hits[e] >> kOrderShift, kOrderBuckets - 1u);
  };
  s_off[t] = 0;
  __syncthreads();
  for (uint32_t i = t; i < n; i += kOrderThreads) atomicAdd(&s_off[bucket(P.warp_events[i])], 1u);
  __syncthreads();
  // exclusive scan of the bucket counts
  const uint32_t v = s_off[t];
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= static_cast<uint32_t>(o)) incl += y;
  }
  if (lane == 31) s_warp[t >> 5] = incl;
  __syncthreads();
  if (t < 32) {
    const uint32_t w = s_warp[t];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= static_cast<uint32_t>(o)) wi += y;
    }
    s_warp[t] = wi - w;
  }
  __syncthreads();
  s_off[t] = s_warp[t >> 5] + incl - v;
  __syncthreads();
  for (uint32_t i = t; i < n; i += kOrderThreads) {
    const uint32_t e = P.warp_events[i];
    P.event_order[atomicAdd(&s_off[bucket(e)], 1u)] = e;
  }
}

}  // namespace velo
