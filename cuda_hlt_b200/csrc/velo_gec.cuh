// Global event cut: the first algorithm of the VELO sequence (configuration/sequences/Velo.h:5-18,
// global_event_cut_t), launched before decode when the caller passes UT and SciFi raw events.
#pragma once
#include "velo_kernels.cuh"

namespace velo {

// Follows global_event_cut (cuda/global_event_cut/src/GlobalEventCut.cu:3-55, with
// maxSciFiUTClusters = 9750 from GlobalEventCut.cuh:9):
//   SciFi estimate = (sum over FTCluster banks of (bank bytes - 4)) / 2 - 2, in 32-bit
//                    unsigned arithmetic (an event with no bank bytes wraps and fails);
//   UT hits        = sum over UT banks of the low 16 bits of the bank's second word;
//   pass           = SciFi < max  and  UT + SciFi < max.
// Raw event layout of both detectors (SciFiRaw.cuh, UTRaw.cuh): u32 number of banks, u32
// bank byte offsets [banks + 1], then the banks. The reference reads the bank tables without
// bounds; here an event whose table or bank headers fall outside its byte range fails the cut
// with kGecMalformed. The UT sum is kept in 64 bits: the reference's 32-bit counter could
// only wrap beyond 65,536 banks.
//
// The reference appends passing events to its list with an atomic counter, so its list order
// is unspecified; here the list is in ascending event order (a stable compaction), one of the
// orders the reference can produce.
constexpr uint32_t kGecMaxClusters = 9750;
constexpr uint8_t kGecPass = 1;
constexpr uint8_t kGecMalformed = 2;
constexpr uint32_t kGecThreads = 256;
constexpr uint32_t kGecListThreads = 1024;

struct GecPointers {
  const RunParams* run;  // inputs: UT and SciFi raw events, their offsets, the threshold
  uint32_t* counts;      // [2N] {SciFi estimate, UT hits} per event (0xFFFFFFFF when malformed)
  uint8_t* flags;        // [N] kGecPass | kGecMalformed
  uint32_t* event_list;  // [N] passing events, ascending
  uint32_t* n_selected;  // [1]
};

// Bank table of one raw event: false when the event is misaligned or its table does not fit.
__device__ __forceinline__ bool gec_table(const uint8_t* raw, const uint64_t* offsets, uint32_t e,
                                          const uint32_t*& ev, uint32_t& n_banks, uint64_t& bytes)
{
  const uint64_t off = offsets[e];
  bytes = offsets[e + 1] - off;
  ev = reinterpret_cast<const uint32_t*>(raw + off);
  if ((reinterpret_cast<uintptr_t>(ev) & 3) || offsets[e + 1] < off || bytes < 8) return false;
  n_banks = __ldg(ev);
  return (static_cast<uint64_t>(n_banks) + 2) * 4 <= bytes;
}

// One warp per event, grid-stride: per-event counts and the pass flag.
__global__ void __launch_bounds__(kGecThreads) gec_count_kernel(GecPointers G)
{
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warps = gridDim.x * (kGecThreads / 32);
  const RunParams& R = *G.run;
  for (uint32_t e = blockIdx.x * (kGecThreads / 32) + (threadIdx.x >> 5); e < R.n_events; e += warps) {
    // SciFi: only the bank offset table is read
    const uint32_t* sf;
    uint32_t nb = 0;
    uint64_t bytes = 0;
    bool bad = !gec_table(R.scifi_raw, R.scifi_offsets, e, sf, nb, bytes);
    uint32_t sum = 0;
    if (!bad)
      for (uint32_t i = lane; i < nb; i += 32)
        sum += __ldg(sf + 2 + i) - __ldg(sf + 1 + i) - 4u;  // 32-bit wrap, as the reference's uint atomicAdd
    sum = __reduce_add_sync(0xFFFFFFFFu, sum);
    const uint32_t n_scifi = sum / 2u - 2u;
    // UT: the hit count in each bank's second word
    const uint32_t* ut;
    uint32_t nu = 0;
    bool ut_bad = !gec_table(R.ut_raw, R.ut_offsets, e, ut, nu, bytes);
    uint64_t hits = 0;
    if (!ut_bad) {
      const uint64_t payload = bytes - (static_cast<uint64_t>(nu) + 2) * 4;
      const uint32_t* data = ut + nu + 2;
      bool lane_bad = false;
      for (uint32_t i = lane; i < nu; i += 32) {
        const uint32_t o = __ldg(ut + 1 + i);
        if ((o & 3) || static_cast<uint64_t>(o) + 8 > payload) {
          lane_bad = true;
        } else {
          hits += __ldg(data + o / 4 + 1) & 0xFFFFu;
        }
      }
      ut_bad = __any_sync(0xFFFFFFFFu, lane_bad);
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) hits += __shfl_xor_sync(0xFFFFFFFFu, hits, s);
    }
    if (lane == 0) {
      const uint32_t n_ut = ut_bad ? 0xFFFFFFFFu : static_cast<uint32_t>(hits < 0xFFFFFFFEull ? hits : 0xFFFFFFFEull);
      const bool pass = !bad && !ut_bad && n_scifi < R.gec_max &&
                        hits + static_cast<uint64_t>(n_scifi) < R.gec_max;
      G.counts[2 * e] = bad ? 0xFFFFFFFFu : n_scifi;
      G.counts[2 * e + 1] = n_ut;
      G.flags[e] = (pass ? kGecPass : 0) | (bad || ut_bad ? kGecMalformed : 0);
    }
  }
}

// One CTA: stable compaction of the passing events (contiguous range per thread, block scan).
__global__ void __launch_bounds__(kGecListThreads) gec_list_kernel(GecPointers G)
{
  __shared__ uint32_t s_warp[kGecListThreads / 32];
  const uint32_t t = threadIdx.x, lane = t & 31u;
  const uint32_t n_events = G.run->n_events;
  const uint32_t per = (n_events + kGecListThreads - 1) / kGecListThreads;
  const uint32_t begin = min(t * per, n_events), end = min(begin + per, n_events);
  uint32_t mine = 0;
  for (uint32_t e = begin; e < end; ++e) mine += G.flags[e] & kGecPass;
  uint32_t incl = mine;
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
    if (t == 31) *G.n_selected = wi;
  }
  __syncthreads();
  uint32_t pos = s_warp[t >> 5] + incl - mine;
  for (uint32_t e = begin; e < end; ++e)
    if (G.flags[e] & kGecPass) G.event_list[pos++] = e;
}

}  // namespace velo
