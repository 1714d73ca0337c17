// Device code of the B200 VELO chain.
//
// Five kernels per batch, no host round trip between them:
//   decode_cluster_sort   one block per event (persistent, events pulled from a queue);
//                         each warp owns whole modules: SuperPixel decode, masked
//                         clustering, phi, per-module sort, compact SoA write.
//   fill_candidates       one block per event (persistent, queue): phi windows of every
//                         h1; in the pruned mode also the learned seed/extension scores
//                         (tensor cores).
//   search_by_triplet     one warp per event (persistent, queue): seeding over the
//                         precomputed windows, forwarding, weak-track recovery; hit_used
//                         is a shared-memory bitmask.
//   event_scan            one block: exclusive scans of tracks and track hits per event.
//   consolidate_fit       one warp per event: hit gather into the consolidated SoA, the
//                         beamline least-squares state and the simplified Kalman state.
//
// Floating-point expressions that decide results (cluster positions, phi, triplet scatter,
// forwarding fit, fits) keep the reference's operation order so that, compiled with the
// same --use_fast_math flags, they round identically; the reference line for each is cited.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "velo_format.hpp"

namespace velo {

// ---------------------------------------------------------------------------
// Capacities of this implementation
// ---------------------------------------------------------------------------
constexpr uint32_t kEventHitCap = 16384;         // hits per event in the search (used bitmask)
constexpr uint32_t kWeakCap = 4096;              // weak tracklets kept per event
constexpr uint32_t kTrackletRing = kTtfModulo;   // tracklet ring (reference ring size)
constexpr uint32_t kStatusEmptyModuleRead = 1u << 10;  // forwarding into an empty module
constexpr uint32_t kStatusSeedTie = 1u << 11;           // exact scatter tie in seeding

__constant__ float c_module_z[kModules] = {VELO_MODULE_Z_VALUES};

struct DeviceConstants {
  const float* geometry;      // 19456-byte blob
  const uint8_t* sp_patterns; // [256]
  const float* sp_fx;         // [512]
  const float* sp_fy;         // [512]
  const uint8_t* sp_sizes;    // [256] pixels of the first (low nibble) and second cluster
};

// Parameters of the learned seed/extension scorer as the kernels read them.
struct MlpDevice {
  const __nv_bfloat16* w;  // W1 [64][16], W2 [64][80], W3 [16][80], row-major, bias in the ones column
  const float* norm;       // feature mean[16], 1/std[16]
  float seed_logit;        // h1 kept as a seed when logit 0 >= seed_logit
  float ext_logit;         // hit kept as an extension candidate when logit 1 >= ext_logit
  uint32_t use_ext;        // extension pruning on
  uint32_t max_hits;       // events with more clusters fall back to the plain search
  uint32_t min_pairs;      // seeds with fewer (h0, h2) pairs are kept unscored
  uint32_t min_hits;       // events with fewer clusters are not scored (every seed kept)
};

// Clusters after the phi sort: position and phi of a cluster in one 16-byte record (one
// 128-bit load in the search), LHCb id alongside.
struct HitsAoS {
  float4* xyzp;  // x, y, z, phi
  uint32_t* id;
};

// Per-event scratch of the search (global memory).
struct SearchScratch {
  uint16_t* track_n;       // [N * kMaxTracks]
  uint16_t* track_hits;    // [N * kMaxTracks * kMaxTrackSize]
  uint16_t* tracklets;     // [N * kTrackletRing * 3]
  uint32_t* ttf;           // [N * kTtfModulo]
  uint16_t* weak;          // [N * kWeakCap * 3]
};

// Inputs of one run, read by the kernels from device memory: set_run_kernel writes them
// before each run, so that a CUDA graph captured for a batch-size bucket serves every batch
// of that bucket, wherever its buffers are.
struct RunParams {
  const uint8_t* raw;
  const uint64_t* raw_offsets;    // [n_events + 1] byte offsets, or null: raw_offsets32
  const uint32_t* raw_offsets32;  // [n_events + 1] u32 byte offsets (the reference's own format)
  uint32_t n_events;
  const uint32_t* event_list;     // [n_events] raw event decoded at each position, or null
                                  // (identity); entries at or beyond n_raw mark the position bad
  uint32_t n_raw;                 // raw events in the batch (with event_list)
  uint32_t gec_max;               // global event cut threshold (velo_run_gec)
  const uint8_t* ut_raw;          // global event cut inputs (null without the cut)
  const uint64_t* ut_offsets;
  const uint8_t* scifi_raw;
  const uint64_t* scifi_offsets;
};

__device__ __forceinline__ uint64_t raw_offset(const RunParams& R, uint32_t e)
{
  return R.raw_offsets ? R.raw_offsets[e] : static_cast<uint64_t>(R.raw_offsets32[e]);
}

struct ChainPointers {
  // input: the run's parameters in device memory; n_grid is the number of events the launch
  // grids are sized for (the bucket of a graph, at least run->n_events): kernels take the
  // run's own count from run->n_events
  const RunParams* run;
  uint32_t n_grid;
  // global event cut (null without it): position e < *n_selected decodes raw event
  // event_list[e]; later positions are left empty
  const uint32_t* event_list;
  const uint32_t* n_selected;
  DeviceConstants k;
  // clusters
  HitsAoS hits;
  HitsAoS stage;           // unsorted clusters, per module (capacity 2 per SP word)
  uint32_t* module_start;  // [N*52] absolute
  uint32_t* module_num;    // [N*52]
  uint32_t* event_hit_base;// [N] absolute index of the event's first hit
  uint32_t* event_hits;    // [N]
  uint32_t* status;        // [N]
  uint8_t* hit_size;       // [hit capacity] pixels of each cluster, at most 3
  // candidates
  uint2* windows;          // [hit capacity] {h0 first | last << 16, h2 first | last << 16}
  uint8_t* keep;           // [hit capacity] learned keep bits; nullptr in the plain mode
  uint8_t* cand_feat;      // pruned mode: bf16 feature rows of the seeding candidates, 128-row
                           // tiles of 4 KB in the tensor core's K-major layout
  uint32_t* cand_slot;     // pruned mode: hit slot of each candidate row
  uint2* cand_rec;         // pruned mode: {event hit base, h1 | module << 16} of each row
  // search
  SearchScratch scratch;
  uint32_t* event_tracks;      // [N] tracks per event
  uint32_t* event_track_hits;  // [N] hits on tracks per event
  // consolidated outputs
  uint32_t* atomics;           // [2N+1]
  uint32_t* track_hit_number;  // [max_tracks+1]
  uint32_t* event_hit_offset;  // [N+1] exclusive scan of event_track_hits
  char* track_hits_out;
  char* states;
  char* kalman_states;
  uint32_t max_tracks_total;
  uint32_t max_track_hits_total;
  uint64_t hit_capacity;       // entries of the hit SoA arrays
  // work queues: [0] decode, [1] warp search, [2] block search, [3] fill_candidates,
  // [4] / [5] sizes of the warp / block event lists, [6] error bits, [7] candidate rows
  uint32_t* queue;             // [8]
  uint32_t* warp_events;       // [N] events routed to the warp-per-event search
  uint32_t* event_order;       // [N] warp_events, largest first: the warp search's queue order
  uint32_t* block_events;      // [N] events routed to the block-per-event search
  uint32_t block_threshold;    // events with more clusters than this go to the block search
  // learned pruning (read when keep != nullptr)
  MlpDevice mlp;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// ---------------------------------------------------------------------------
// Masks of the 3-column pixel flood (MaskedVeloClustering.cu:4-46; masks
// ClusteringDefinitions.cuh:14-19). Bit layout: per SP column 16 rows in the low half,
// the second pixel column of the SP in the high half.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t flood_mask(uint32_t p)
{
  return ((p & kMaskTop) << 1) | ((p & kMaskBottom) >> 1) | ((p & kMaskBottomRight) << 15) |
         ((p & kMaskTopLeft) >> 15) | (p >> 16) | (p >> 17) | (p << 16) | (p << 17);
}
__device__ __forceinline__ uint32_t flood_left_to_right(uint32_t p)
{
  return ((p & kMaskLtrTopRight) >> 15) | (p >> 16) | (p >> 17);
}
__device__ __forceinline__ uint32_t flood_right_to_left(uint32_t p)
{
  return ((p & kMaskRtlBottomLeft) << 15) | (p << 16) | (p << 17);
}
__device__ __forceinline__ uint32_t found_cluster_mask(uint32_t p)
{
  return ((p & kMaskTop) << 1) | ((p & kMaskBottomRight) << 15) | (p << 16) | (p << 17);
}
__device__ __forceinline__ uint32_t precedence_candidates(uint32_t p, uint32_t rp)
{
  return ((p & kMaskBottom) >> 1) & (((p & kMaskTopLeft) >> 15) | (rp << 17)) & ((p >> 16) | (rp << 16)) &
         ((p >> 17) | ((rp & kMaskRtlBottomLeft) << 15));
}

__device__ __forceinline__ uint32_t candidate_k(uint32_t code_nibble)
{
  // one-hot nibble -> position (Constants.cu:36 table {0,0,1,4,4,5,5,5,5})
  return code_nibble == 2u ? 1u : (code_nibble >= 5u ? 5u : (code_nibble >= 3u ? 4u : 0u));
}

// Global position of a cluster centroid (MaskedVeloClustering.cu:124-133, :431-449).
struct ClusterPoint {
  float x, y, z;
  uint32_t id;
};

__device__ __forceinline__ ClusterPoint place_cluster(const GeometryView& g, uint32_t sensor, uint32_t cx, uint32_t cy,
                                                      float fx, float fy, uint32_t chip)
{
  const float* ltg = g.ltg + 16 * sensor;
  const float local_x = g.local_x[cx] + fx * g.x_pitch[cx];
  const float local_y = (cy + 0.5 + fy) * kPixelSize;
  ClusterPoint p;
  p.x = ltg[0] * local_x + ltg[1] * local_y + ltg[9];
  p.y = ltg[3] * local_x + ltg[4] * local_y + ltg[10];
  p.z = ltg[6] * local_x + ltg[7] * local_y + ltg[11];
  p.id = lhcb_id(channel_id(sensor, chip, cx % kChipColumns, cy));
  return p;
}

// phi conventions (cuda/velo/common/src/VeloTools.cu:3-10): odd modules in (-pi, pi],
// even modules shifted to [0, 2pi).
__device__ __forceinline__ float phi_odd_side(float x, float y) { return atan2f(y, x); }
__device__ __forceinline__ float phi_even_side(float x, float y)
{
  const float phi = atan2f(y, x);
  const bool below = phi < 0.f;
  return phi + below * 2 * 3.141592654f;
}

__device__ __forceinline__ uint32_t orderable(float f)
{
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// phi-window searches of cuda/velo/common/include/VeloTools.cuh:6-42 (the "found" flag
// accumulates over every probed element, as there).
__device__ __forceinline__ int window_first(const float* a, uint32_t size, float value, float margin)
{
  bool found = false;
  int l = 0, r = static_cast<int>(size) - 1;
  while (l < r) {
    const int m = (l + r) / 2;
    const float e = a[m];
    found |= fabsf(value - e) < margin;
    if (value - margin > e) l = m + 1; else r = m;
  }
  found |= fabsf(value - a[l]) < margin;
  return found ? l : -1;
}
__device__ __forceinline__ int window_second(const float* a, uint32_t size, float value, float margin)
{
  int l = 0, r = static_cast<int>(size) - 1;
  while (l < r) {
    const int m = (l + r) / 2;
    if (value + margin > a[m]) l = m + 1; else r = m;
  }
  return fabsf(value - a[l]) < margin ? l + 1 : l;
}
// The same two searches over the phi lane (.w) of the float4 cluster records.
__device__ __forceinline__ int window_first4(const float4* a, uint32_t size, float value, float margin)
{
  bool found = false;
  int l = 0, r = static_cast<int>(size) - 1;
  while (l < r) {
    const int m = (l + r) / 2;
    const float e = a[m].w;
    found |= fabsf(value - e) < margin;
    if (value - margin > e) l = m + 1; else r = m;
  }
  found |= fabsf(value - a[l].w) < margin;
  return found ? l : -1;
}
__device__ __forceinline__ int window_second4(const float4* a, uint32_t size, float value, float margin)
{
  int l = 0, r = static_cast<int>(size) - 1;
  while (l < r) {
    const int m = (l + r) / 2;
    if (value + margin > a[m].w) l = m + 1; else r = m;
  }
  return fabsf(value - a[l].w) < margin ? l + 1 : l;
}
__device__ __forceinline__ void phi_window4(const float4* H, uint32_t start, uint32_t num, float value, float margin,
                                            int& first, int& last)
{
  first = window_first4(H + start, num, value, margin);
  last = -1;
  if (first != -1) {
    const int s = window_second4(H + start + first, num - first, value, margin);
    first += start;
    last = s == 0 ? first + 1 : first + s;
  }
}

// [first, last) of hits in a phi-sorted module within margin of value; first = -1 if none.
__device__ __forceinline__ void phi_window(const float* phis, uint32_t start, uint32_t num, float value, float margin,
                                           int& first, int& last)
{
  first = window_first(phis + start, num, value, margin);
  last = -1;
  if (first != -1) {
    const int s = window_second(phis + start + first, num - first, value, margin);
    first += start;
    last = s == 0 ? first + 1 : first + s;
  }
}

}  // namespace velo
