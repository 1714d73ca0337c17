// B200 VELO chain: kernels and the C-ABI context (include/velo_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <array>
#include <list>
#include <map>
#include <tuple>
#include <vector>

#include "../../include/velo_b200.h"
#include "velo_kernels.cuh"

#include "velo_ctx.hpp"
#include "velo_decode.cuh"
#include "velo_fill.cuh"
#include "velo_order.cuh"
#include "velo_search.cuh"
#include "velo_search_block.cuh"
#include "velo_consolidate.cuh"
#include "velo_pv.cuh"
#include "velo_gec.cuh"

// ============================================================================
// C-ABI context
// ============================================================================
using namespace velo;

struct VeloCtx {
  VeloConfig cfg{};
  int device = 0;
  int sm_count = 0;
  cudaStream_t own_stream = nullptr;
  // constants
  uint8_t* d_geometry = nullptr;
  uint8_t* d_sp_patterns = nullptr;
  float* d_sp_fx = nullptr;
  float* d_sp_fy = nullptr;
  uint8_t* d_sp_sizes = nullptr;
  // learned scorer
  __nv_bfloat16* d_mlp_w = nullptr;
  float* d_mlp_norm = nullptr;
  MlpDevice mlp{};
  bool mlp_loaded = false;
  // labels of a plain run kept by velo_capture_labels (VELO_MODE_LABELS)
  uint8_t* d_labels = nullptr;
  bool labels_ready = false;
  uint32_t labels_ext = 0;
  uint32_t labels_max_hits = 0;
  uint32_t mode = VELO_MODE_PLAIN;
  // input staging (for velo_run_host / velo_run_host_u32)
  uint8_t* d_raw = nullptr;
  uint64_t* d_raw_offsets = nullptr;
  uint32_t* d_raw_offsets32 = nullptr;
  // the parameters of the current run, read by the kernels (set_run_kernel)
  RunParams* d_run = nullptr;
  // work buffers
  float4* d_hxyzp = nullptr;
  uint32_t* d_hid = nullptr;
  float4* d_stage_xyzp = nullptr;
  uint32_t* d_stage_id = nullptr;
  uint8_t* d_hit_size = nullptr;
  uint2* d_windows = nullptr;
  uint8_t* d_keep = nullptr;
  uint8_t* d_cand_feat = nullptr;
  uint32_t* d_cand_slot = nullptr;
  uint2* d_cand_rec = nullptr;
  uint64_t hit_capacity = 0;
  uint32_t *d_module_start = nullptr, *d_module_num = nullptr, *d_event_hit_base = nullptr, *d_event_hits = nullptr,
           *d_status = nullptr;
  uint16_t *d_track_n = nullptr, *d_track_hits = nullptr, *d_tracklets = nullptr, *d_weak = nullptr;
  uint32_t* d_ttf = nullptr;
  uint32_t *d_event_tracks = nullptr, *d_event_track_hits = nullptr;
  uint32_t *d_atomics = nullptr, *d_track_hit_number = nullptr, *d_event_hit_offset = nullptr;
  char *d_track_hits_out = nullptr, *d_states = nullptr, *d_kalman = nullptr;
  uint32_t* d_queue = nullptr;
  uint32_t *d_warp_events = nullptr, *d_block_events = nullptr, *d_event_order = nullptr;
  uint32_t block_threshold = 0;  // clusters above which an event takes the block search
  // beamline PV stage (velo_set_pv)
  bool pv = false;
  PvTrack* d_pv_tracks = nullptr;
  PvVertex* d_pv_vertices = nullptr;
  uint32_t *d_pv_count = nullptr, *d_pv_npeaks = nullptr;
  float* d_pv_zpeaks = nullptr;
  // global event cut (velo_run_gec): per-event counts and flags, the selected list, and the
  // UT / SciFi staging of velo_run_gec_host (grown on demand)
  uint32_t *d_gec_counts = nullptr, *d_event_list = nullptr, *d_n_selected = nullptr;
  uint8_t* d_gec_flags = nullptr;
  uint8_t *d_gec_ut = nullptr, *d_gec_scifi = nullptr;
  uint64_t *d_gec_ut_offsets = nullptr, *d_gec_scifi_offsets = nullptr;
  size_t gec_ut_cap = 0, gec_scifi_cap = 0;
  uint32_t gec_blocks = 0;
  uint32_t* h_totals = nullptr;  // pinned [4]: tracks, track hits, error bits of the last run
  // pinned staging of host offsets (three slots of max_events + 1: raw, UT, SciFi) and the
  // event that marks when the last copies out of it completed
  uint64_t* h_offsets = nullptr;
  cudaEvent_t ev_offsets = nullptr;
  bool offsets_pending = false;
  cudaStream_t last_stream = nullptr;
  uint32_t last_n = 0;
  uint32_t launches = 0;
  bool timing = false;
  // Stage timing: one set of kStageEvents events per launch sequence, taken in turn from a
  // pool of kEventSets sets by plain launches and graph launches alike (a graph's event-record
  // nodes are pointed at the set before it is launched).
  // Events 0..6 bound the six chain stages in order; 7 and 8 bound the global event cut
  // (recorded back to back when it does not run).
  static constexpr int kStageEvents = 9;
  std::vector<std::array<cudaEvent_t, kStageEvents>> ev_sets;
  std::vector<uint8_t> ev_used;
  uint32_t ev_next = 0;
  int ev_current = -1;
  int decode_warps = 8;
  int search_wpb = 4;
  uint32_t decode_blocks = 0, search_blocks = 0, search_block_blocks = 0, fill_blocks = 0,
           feature_blocks = 0, score_blocks = 0;
  // CUDA graphs per (batch-size bucket, stream, global event cut on or off): the kernels read
  // the run's inputs from d_run, so a graph serves every batch of its bucket; at most
  // kMaxGraphs are kept, the least recently launched evicted first
  static constexpr size_t kMaxGraphs = 16;
  struct GraphKey {
    uint32_t bucket;
    cudaStream_t stream;
    bool gec;
    bool operator<(const GraphKey& o) const { return std::tie(bucket, stream, gec) < std::tie(o.bucket, o.stream, o.gec); }
  };
  struct GraphEntry {
    cudaGraphExec_t exec;
    cudaGraph_t graph;  // kept: its event-record nodes are rebound before each timed launch
    std::array<cudaGraphNode_t, kStageEvents> ev_nodes;  // event-record node of each stage event
    bool timed;         // captured with the stage events
    uint32_t launches;  // kernels in the graph
    std::list<GraphKey>::iterator lru;
  };
  std::list<GraphKey> lru;  // most recently launched first
  std::map<GraphKey, GraphEntry> graphs;
};

#define VCK(x)                                                                                  \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) {                                                                    \
      std::fprintf(stderr, "velo_b200: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return VELO_ERR_CUDA;                                                                     \
    }                                                                                           \
  } while (0)

extern "C" void velo_build_sp_luts(uint8_t* patterns, uint8_t* sizes, float* fx, float* fy);

namespace {


template<class T>
cudaError_t dalloc(T*& p, size_t count)
{
  return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T));
}

void free_all(VeloCtx* c)
{
  void* ptrs[] = {c->d_labels, c->d_geometry, c->d_sp_patterns, c->d_sp_fx, c->d_sp_fy, c->d_sp_sizes, c->d_mlp_w, c->d_mlp_norm,
                  c->d_hit_size, c->d_windows, c->d_keep, c->d_cand_slot, c->d_cand_rec, c->d_raw, c->d_raw_offsets, c->d_hxyzp,
                  c->d_hid, c->d_stage_xyzp, c->d_stage_id, c->d_module_start, c->d_module_num, c->d_event_hit_base,
                  c->d_event_hits, c->d_status, c->d_track_n, c->d_track_hits, c->d_tracklets, c->d_weak, c->d_ttf,
                  c->d_event_tracks, c->d_event_track_hits, c->d_atomics, c->d_track_hit_number,
                  c->d_event_hit_offset, c->d_track_hits_out, c->d_states, c->d_kalman, c->d_queue,
                  c->d_warp_events, c->d_block_events, c->d_event_order, c->d_pv_tracks, c->d_pv_vertices,
                  c->d_pv_count, c->d_pv_npeaks, c->d_pv_zpeaks, c->d_gec_counts, c->d_event_list,
                  c->d_n_selected, c->d_gec_flags, c->d_gec_ut, c->d_gec_scifi, c->d_gec_ut_offsets,
                  c->d_gec_scifi_offsets};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->h_totals) cudaFreeHost(c->h_totals);
  if (c->h_offsets) cudaFreeHost(c->h_offsets);
  if (c->ev_offsets) cudaEventDestroy(c->ev_offsets);
  for (auto& kv : c->graphs) {
    cudaGraphExecDestroy(kv.second.exec);
    cudaGraphDestroy(kv.second.graph);
  }
  if (c->d_run) cudaFree(c->d_run);
  if (c->d_raw_offsets32) cudaFree(c->d_raw_offsets32);
  for (auto& set : c->ev_sets)
    for (auto& e : set)
      if (e) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
}

constexpr uint32_t kEventSets = 64;  // launch sequences whose stage times are kept

int add_event_set(VeloCtx* c)
{
  std::array<cudaEvent_t, VeloCtx::kStageEvents> set{};
  for (auto& e : set)
    if (cudaEventCreate(&e) != cudaSuccess) return VELO_ERR_CUDA;
  c->ev_sets.push_back(set);
  c->ev_used.push_back(0);
  return static_cast<int>(c->ev_sets.size() - 1);
}

// Kernel parameters of a run whose grids are sized for n_grid events (the run's own inputs
// and count are in c->d_run).
ChainPointers pointers(VeloCtx* c, uint32_t n_grid)
{
  ChainPointers P{};
  P.run = c->d_run;
  P.n_grid = n_grid;
  P.k = DeviceConstants{reinterpret_cast<const float*>(c->d_geometry), c->d_sp_patterns, c->d_sp_fx, c->d_sp_fy,
                        c->d_sp_sizes};
  P.hits = HitsAoS{c->d_hxyzp, c->d_hid};
  P.stage = HitsAoS{c->d_stage_xyzp, c->d_stage_id};
  P.module_start = c->d_module_start;
  P.module_num = c->d_module_num;
  P.event_hit_base = c->d_event_hit_base;
  P.event_hits = c->d_event_hits;
  P.status = c->d_status;
  P.hit_size = c->d_hit_size;
  P.windows = c->d_windows;
  P.keep = c->mode == VELO_MODE_PRUNED ? c->d_keep : (c->mode == VELO_MODE_LABELS ? c->d_labels : nullptr);
  P.cand_feat = c->d_cand_feat;
  P.cand_slot = c->d_cand_slot;
  P.cand_rec = c->d_cand_rec;
  P.scratch = SearchScratch{c->d_track_n, c->d_track_hits, c->d_tracklets, c->d_ttf, c->d_weak};
  P.event_tracks = c->d_event_tracks;
  P.event_track_hits = c->d_event_track_hits;
  P.atomics = c->d_atomics;
  P.track_hit_number = c->d_track_hit_number;
  P.event_hit_offset = c->d_event_hit_offset;
  P.track_hits_out = c->d_track_hits_out;
  P.states = c->d_states;
  P.kalman_states = c->d_kalman;
  P.max_tracks_total = c->cfg.max_tracks;
  P.max_track_hits_total = c->cfg.max_track_hits;
  P.hit_capacity = c->hit_capacity;
  P.queue = c->d_queue;
  P.warp_events = c->d_warp_events;
  P.event_order = c->d_event_order;
  P.block_events = c->d_block_events;
  P.block_threshold = c->block_threshold;
  P.mlp = c->mlp;
  if (c->mode == VELO_MODE_LABELS) {
    P.mlp = MlpDevice{};
    P.mlp.use_ext = c->labels_ext;
    P.mlp.max_hits = c->labels_max_hits;
  }
  return P;
}

// Labels of the hits of one run's events from the tracks of its plain search, one block per
// event: bit 0 on a final track, bit 1 the fourth or a later hit of one (the labels the
// scorer is trained on). Events above `max_hits` clusters get every bit set (nothing pruned).
__global__ void __launch_bounds__(256) capture_labels_kernel(ChainPointers P, uint8_t* labels, uint32_t max_hits)
{
  const uint32_t n_events = P.run->n_events;
  for (uint32_t e = blockIdx.x; e < n_events; e += gridDim.x) {
    const uint32_t nhits = P.event_hits[e], base = P.event_hit_base[e], status = P.status[e];
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (!runnable) continue;
    uint8_t* L = labels + base;
    const bool all = nhits > max_hits;
    for (uint32_t h = threadIdx.x; h < nhits; h += blockDim.x) L[h] = all ? 3u : 0u;
    __syncthreads();
    if (!all) {
      const uint32_t nt = min(P.event_tracks[e], kMaxTracks);  // a hit is on one track at most
      const uint16_t* tn = P.scratch.track_n + static_cast<size_t>(e) * kMaxTracks;
      const uint16_t* th = P.scratch.track_hits + static_cast<size_t>(e) * kMaxTracks * kMaxTrackSize;
      for (uint32_t t = threadIdx.x; t < nt; t += blockDim.x) {
        const uint32_t n = tn[t];
        for (uint32_t k = 0; k < n; ++k) L[th[t * kMaxTrackSize + k]] = k >= 3 ? 3u : 1u;
      }
    }
    __syncthreads();
  }
}

// VELO_MODE_LABELS: seeds without the "on a final track" label lose their h0 window, as the
// scorer's pruned seeds do; the search reads the labels as extension-keep bits.
__global__ void __launch_bounds__(kFillThreads) label_seeds_kernel(ChainPointers P)
{
  const uint32_t n_events = P.run->n_events;
  for (uint32_t e = blockIdx.x; e < n_events; e += gridDim.x) {
    const uint32_t nhits = P.event_hits[e], base = P.event_hit_base[e], status = P.status[e];
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (!runnable) continue;
    if (nhits > P.mlp.max_hits) {
      if (threadIdx.x == 0) P.status[e] = status | kStatusMlpFallback;
      continue;
    }
    const uint32_t lo = P.module_start[e * kModules + 2] - base, hi = P.module_start[e * kModules + 50] - base;
    for (uint32_t h = lo + threadIdx.x; h < hi; h += blockDim.x)
      if (!(P.keep[base + h] & 1u)) P.windows[base + h].x = 0xFFFFFFFFu;
  }
}

// Writes the parameters of the next run where the kernels read them and clears the work
// queues. Launched on the run's stream before the chain (or its graph), outside any capture.
__global__ void set_run_kernel(RunParams* dst, RunParams v, uint32_t* queue)
{
  if (threadIdx.x == 0) *dst = v;
  if (threadIdx.x < 8) queue[threadIdx.x] = 0u;
}

// Inside a stream capture an event record must be marked external to become a node that
// records when the graph runs (a plain record only orders the capture).
cudaError_t record(cudaEvent_t e, cudaStream_t s, bool capturing)
{
  return capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s);
}

int launch_chain(VeloCtx* c, const ChainPointers& P, const GecPointers* G, cudaStream_t s, bool capturing = false)
{
  const uint32_t n = P.n_grid;
  c->launches = 0;
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][7], s, capturing));
  if (G) {  // global event cut: the event list decode reads
    const uint32_t blocks = std::min<uint32_t>((n + kGecThreads / 32 - 1) / (kGecThreads / 32), c->gec_blocks);
    gec_count_kernel<<<blocks, kGecThreads, 0, s>>>(*G);
    VCK(cudaGetLastError());
    gec_list_kernel<<<1, kGecListThreads, 0, s>>>(*G);
    VCK(cudaGetLastError());
    c->launches += 2;
  }
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][8], s, capturing));
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][0], s, capturing));
  const bool pruned = c->mode == VELO_MODE_PRUNED;
  {
    const uint32_t blocks = std::min<uint32_t>(n, c->decode_blocks);
    // the decode kernel also computes the phi windows (fill_candidates) and, in the pruned
    // mode, the scorer's candidate list
    if (c->decode_warps == 8) {
      if (pruned) decode_cluster_sort_kernel<8, true><<<blocks, 256, 0, s>>>(P);
      else decode_cluster_sort_kernel<8, false><<<blocks, 256, 0, s>>>(P);
    } else {
      if (pruned) decode_cluster_sort_kernel<4, true><<<blocks, 128, 0, s>>>(P);
      else decode_cluster_sort_kernel<4, false><<<blocks, 128, 0, s>>>(P);
    }
    VCK(cudaGetLastError());
    ++c->launches;
  }
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][1], s, capturing));
  if (c->mode == VELO_MODE_LABELS) {
    label_seeds_kernel<<<std::min<uint32_t>(n, c->fill_blocks), kFillThreads, 0, s>>>(P);
    ++c->launches;
  } else if (pruned) {
    candidate_features_kernel<<<c->feature_blocks, kFillThreads, 0, s>>>(P);
    VCK(cudaGetLastError());
    score_candidates_kernel<<<c->score_blocks, kScoreThreads, kScoreSmem, s>>>(P);
    c->launches += 2;
  }
  VCK(cudaGetLastError());
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][2], s, capturing));
  {
    // both mappings: each kernel drains its own event list (routed by the decode kernel)
    if (c->block_threshold > 0) {
      order_events_kernel<<<1, kOrderThreads, 0, s>>>(P);
      VCK(cudaGetLastError());
      const uint32_t blocks = std::min<uint32_t>((n + 3) / 4, c->search_blocks);
      search_kernel<4><<<blocks, 128, 0, s>>>(P);
      VCK(cudaGetLastError());
      c->launches += 2;
    }
    if (c->block_threshold < kEventHitCap) {
      const uint32_t blocks = std::min<uint32_t>(n, c->search_block_blocks);
      search_block_kernel<<<blocks, kBlockThreads, kStageCap * sizeof(float4), s>>>(P);
      VCK(cudaGetLastError());
      ++c->launches;
    }
  }
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][3], s, capturing));
  event_scan_kernel<<<1, 1024, 0, s>>>(P);
  VCK(cudaGetLastError());
  ++c->launches;
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][4], s, capturing));
  consolidate_fit_kernel<4><<<(n + 3) / 4, 128, 0, s>>>(P);
  VCK(cudaGetLastError());
  ++c->launches;
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][5], s, capturing));
  if (c->pv) {
    const PvPointers V{c->d_kalman, c->d_pv_tracks, c->d_pv_vertices, c->d_pv_count, c->d_pv_zpeaks, c->d_pv_npeaks};
    pv_beamline_kernel<<<n, kPvThreads, 0, s>>>(P, V);
    VCK(cudaGetLastError());
    ++c->launches;
  }
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][6], s, capturing));
  return 0;
}

// Persistent decode grid: as many blocks of the chosen size as are resident together.
void size_decode_grid(VeloCtx* c)
{
  int occ = 0;
  if (c->decode_warps == 8)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, decode_cluster_sort_kernel<8, true>, 256, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, decode_cluster_sort_kernel<4, true>, 128, 0);
  c->decode_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
}

void size_search_grid(VeloCtx* c)
{
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, search_kernel<4>, 128, 0);
  c->search_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
}

// A bounded wait that runs out: an mbarrier that nothing arrives on, waited for with
// mbar_wait_parity (the wait of the scorer's copies and tensor-core steps) for `polls` polls;
// the kernel then sets the error bit the scorer sets on a timeout and returns. Nothing is in
// flight when it gives up, so it exits cleanly.
__global__ void wait_timeout_kernel(uint32_t* error, uint32_t polls)
{
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) mbar_init1(&bar);
  __syncthreads();
  const bool done = mbar_wait_parity(&bar, 0, polls);
  if (!done && threadIdx.x == 0) atomicOr(error, kErrorMlpTimeout);
}

void drop_graphs(VeloCtx* c)
{
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (auto& kv : c->graphs) {
    cudaGraphExecDestroy(kv.second.exec);
    cudaGraphDestroy(kv.second.graph);
  }
  c->graphs.clear();
  c->lru.clear();
}

// The pruned mode's buffers (keep bits, candidate records, feature rows, hit slots: 45 bytes
// per hit slot), allocated when the mode is first selected.
int ensure_pruned_buffers(VeloCtx* c)
{
  if (c->d_keep) return 0;
  bool ok = true;
  ok &= dalloc(c->d_keep, c->hit_capacity) == cudaSuccess;
  // the feature rows share the decode kernel's staging area: decode has finished with it
  // when candidate_features writes them, and the next run's decode starts after the scorer
  c->d_cand_feat = reinterpret_cast<uint8_t*>(c->d_stage_xyzp);
  ok &= dalloc(c->d_cand_slot, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_cand_rec, c->hit_capacity) == cudaSuccess;
  if (!ok) {
    for (void* p : {static_cast<void*>(c->d_keep), static_cast<void*>(c->d_cand_slot),
                    static_cast<void*>(c->d_cand_rec)})
      if (p) cudaFree(p);
    c->d_keep = nullptr;
    c->d_cand_feat = nullptr;
    c->d_cand_slot = nullptr;
    c->d_cand_rec = nullptr;
    return VELO_ERR_CUDA;
  }
  return 0;
}

// Batch-size bucket of a graph: 1,024 events times a power of 4, at most the context's size.
uint32_t bucket_of(const VeloCtx* c, uint32_t n)
{
  uint64_t b = 1024;
  while (b < n) b *= 4;
  return static_cast<uint32_t>(std::min<uint64_t>(b, c->cfg.max_events));
}

}  // namespace

extern "C" {

const char* velo_version(void) { return "velo_b200 0.1 (sm_100a)"; }

int velo_create(const VeloConfig* cfg, const void* geometry, size_t geometry_bytes, VeloCtx** out)
{
  if (!cfg || !geometry || !out || cfg->max_events == 0) return VELO_ERR_INVALID;
  if (geometry_bytes != kGeometryBytes) return VELO_ERR_BAD_GEOMETRY;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return VELO_ERR_NO_DEVICE;
  if (cfg->device < 0 || cfg->device >= ndev) return VELO_ERR_INVALID;
  auto* c = new VeloCtx();
  c->cfg = *cfg;
  if (c->cfg.max_tracks == 0) c->cfg.max_tracks = 400u * cfg->max_events;
  if (c->cfg.max_track_hits == 0) c->cfg.max_track_hits = 16u * c->cfg.max_tracks;
  c->device = cfg->device;
  auto fail = [&](int code) {
    free_all(c);
    delete c;
    return code;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(VELO_ERR_CUDA);
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
  const uint32_t N = cfg->max_events;
  c->hit_capacity = cfg->max_raw_bytes / 4 + 64;
  const size_t T = c->cfg.max_tracks, TH = c->cfg.max_track_hits;
  bool ok = true;
  ok &= dalloc(c->d_geometry, kGeometryBytes) == cudaSuccess;
  ok &= dalloc(c->d_sp_patterns, 256) == cudaSuccess;
  ok &= dalloc(c->d_sp_fx, 512) == cudaSuccess;
  ok &= dalloc(c->d_sp_fy, 512) == cudaSuccess;
  ok &= dalloc(c->d_sp_sizes, 256) == cudaSuccess;
  ok &= dalloc(c->d_mlp_w, kMlpParams) == cudaSuccess;
  ok &= dalloc(c->d_mlp_norm, 32) == cudaSuccess;
  ok &= dalloc(c->d_raw, cfg->max_raw_bytes + 16) == cudaSuccess;
  ok &= dalloc(c->d_raw_offsets, N + 1) == cudaSuccess;
  ok &= dalloc(c->d_raw_offsets32, N + 1) == cudaSuccess;
  ok &= dalloc(c->d_run, 1) == cudaSuccess;
  ok &= dalloc(c->d_hxyzp, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_hid, c->hit_capacity) == cudaSuccess;
  // 2 records per hit slot; at least the pruned mode's feature rows, which share it
  // ((hit slots + one tile) x 32 bytes)
  ok &= dalloc(c->d_stage_xyzp, 2 * (c->hit_capacity + kMlpTile)) == cudaSuccess;
  ok &= dalloc(c->d_stage_id, 2 * c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_hit_size, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_windows, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_module_start, static_cast<size_t>(N) * kModules) == cudaSuccess;
  ok &= dalloc(c->d_module_num, static_cast<size_t>(N) * kModules) == cudaSuccess;
  ok &= dalloc(c->d_event_hit_base, N) == cudaSuccess;
  ok &= dalloc(c->d_event_hits, N) == cudaSuccess;
  ok &= dalloc(c->d_status, N) == cudaSuccess;
  ok &= dalloc(c->d_track_n, static_cast<size_t>(N) * kMaxTracks) == cudaSuccess;
  ok &= dalloc(c->d_track_hits, static_cast<size_t>(N) * kMaxTracks * kMaxTrackSize) == cudaSuccess;
  ok &= dalloc(c->d_tracklets, static_cast<size_t>(N) * kTrackletRing * 3) == cudaSuccess;
  ok &= dalloc(c->d_ttf, static_cast<size_t>(N) * kTtfModulo) == cudaSuccess;
  ok &= dalloc(c->d_weak, static_cast<size_t>(N) * kWeakCap * 3) == cudaSuccess;
  ok &= dalloc(c->d_event_tracks, N) == cudaSuccess;
  ok &= dalloc(c->d_event_track_hits, N) == cudaSuccess;
  ok &= dalloc(c->d_atomics, 2 * static_cast<size_t>(N) + 1) == cudaSuccess;
  ok &= dalloc(c->d_track_hit_number, T + 1) == cudaSuccess;
  ok &= dalloc(c->d_event_hit_offset, static_cast<size_t>(N) + 1) == cudaSuccess;
  ok &= dalloc(c->d_track_hits_out, 16 * TH) == cudaSuccess;
  ok &= dalloc(c->d_states, 52 * T) == cudaSuccess;
  ok &= dalloc(c->d_kalman, 52 * T) == cudaSuccess;
  ok &= dalloc(c->d_pv_tracks, T) == cudaSuccess;
  ok &= dalloc(c->d_pv_vertices, static_cast<size_t>(N) * kPvMaxVertices) == cudaSuccess;
  ok &= dalloc(c->d_pv_zpeaks, static_cast<size_t>(N) * kPvMaxVertices) == cudaSuccess;
  ok &= dalloc(c->d_pv_count, N) == cudaSuccess;
  ok &= dalloc(c->d_pv_npeaks, N) == cudaSuccess;
  ok &= dalloc(c->d_gec_counts, 2 * static_cast<size_t>(N)) == cudaSuccess;
  ok &= dalloc(c->d_gec_flags, N) == cudaSuccess;
  ok &= dalloc(c->d_event_list, N) == cudaSuccess;
  ok &= dalloc(c->d_n_selected, 1) == cudaSuccess;
  ok &= dalloc(c->d_gec_ut_offsets, static_cast<size_t>(N) + 1) == cudaSuccess;
  ok &= dalloc(c->d_gec_scifi_offsets, static_cast<size_t>(N) + 1) == cudaSuccess;
  ok &= dalloc(c->d_queue, 8) == cudaSuccess;
  ok &= dalloc(c->d_warp_events, N) == cudaSuccess;
  ok &= dalloc(c->d_block_events, N) == cudaSuccess;
  ok &= dalloc(c->d_event_order, N) == cudaSuccess;
  ok &= cudaMallocHost(reinterpret_cast<void**>(&c->h_totals), 4 * sizeof(uint32_t) + 8) == cudaSuccess;
  ok &= cudaMallocHost(reinterpret_cast<void**>(&c->h_offsets), 3 * (static_cast<size_t>(N) + 1) * sizeof(uint64_t)) ==
        cudaSuccess;
  ok &= cudaEventCreateWithFlags(&c->ev_offsets, cudaEventDisableTiming) == cudaSuccess;
  if (ok) std::memset(c->h_totals, 0, 4 * sizeof(uint32_t) + 8);
  if (!ok) return fail(VELO_ERR_CUDA);
  uint8_t pat[256], sizes[256];
  float fx[512], fy[512];
  velo_build_sp_luts(pat, sizes, fx, fy);
  if (cudaMemcpy(c->d_geometry, geometry, kGeometryBytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_sp_patterns, pat, 256, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_sp_fx, fx, sizeof fx, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_sp_fy, fy, sizeof fy, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_sp_sizes, sizes, 256, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(VELO_ERR_CUDA);
  int occ = 0;
  size_decode_grid(c);
  size_search_grid(c);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, gec_count_kernel, kGecThreads, 0);
  c->gec_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
  cudaFuncSetAttribute(search_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(kStageCap * sizeof(float4)));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, search_block_kernel, kBlockThreads, kStageCap * sizeof(float4));
  c->search_block_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, label_seeds_kernel, kFillThreads, 0);
  c->fill_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, candidate_features_kernel, kFillThreads, 0);
  c->feature_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
  // the scorer: as many CTAs per SM as shared memory holds (1 KB of it is reserved per
  // block), at most 4 (each holds 128 of the SM's 512 tensor-memory columns)
  cudaFuncSetAttribute(score_candidates_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(kScoreSmem));
  int smem_sm = 0;
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device);
  const int score_per_sm =
    std::max(1, std::min(static_cast<int>(512 / kScoreTmemCols), smem_sm / static_cast<int>(kScoreSmem + 1024)));
  c->score_blocks = static_cast<uint32_t>(score_per_sm * c->sm_count);
  c->mode = cfg->mode == VELO_MODE_PRUNED ? VELO_MODE_PRUNED : VELO_MODE_PLAIN;
  if (c->mode == VELO_MODE_PRUNED && ensure_pruned_buffers(c) != 0) return fail(VELO_ERR_CUDA);
  // mapping: VELO_MAP_WARP keeps every event on warps, VELO_MAP_BLOCK on blocks; the
  // default splits at a cluster count (velo_set_block_threshold / the autotuner move it)
  c->block_threshold = cfg->mapping == VELO_MAP_WARP ? kEventHitCap : (cfg->mapping == VELO_MAP_BLOCK ? 0u : 1536u);
  if (cudaGetLastError() != cudaSuccess) return fail(VELO_ERR_CUDA);
  *out = c;
  return 0;
}

static int fill_outputs(VeloCtx* c, uint32_t n, VeloOutputs* out)
{
  if (!out) return 0;
  std::memset(out, 0, sizeof(*out));
  out->n_events = n;
  out->atomics = c->d_atomics;
  out->track_hit_number = c->d_track_hit_number;
  out->track_hits = c->d_track_hits_out;
  out->states = c->d_states;
  out->kalman_states = c->d_kalman;
  out->status = c->d_status;
  out->module_hit_start = c->d_module_start;
  out->module_hit_num = c->d_module_num;
  out->hit_xyzp = reinterpret_cast<float*>(c->d_hxyzp);
  out->hit_id = c->d_hid;
  out->hit_capacity = c->hit_capacity;
  out->hit_size = c->d_hit_size;
  out->hit_windows = reinterpret_cast<uint32_t*>(c->d_windows);
  out->hit_keep = c->mode == VELO_MODE_PRUNED ? c->d_keep : (c->mode == VELO_MODE_LABELS ? c->d_labels : nullptr);
  if (c->pv) {
    out->pv_vertices = c->d_pv_vertices;
    out->pv_count = c->d_pv_count;
    out->pv_zpeaks = c->d_pv_zpeaks;
    out->pv_npeaks = c->d_pv_npeaks;
  }
  return 0;
}

// velo_run with or without the global event cut in front (gec: device inputs, or null), raw
// offsets as u64 (raw_offsets) or u32 (raw_offsets32).
static int launch_run(VeloCtx* c, const void* raw, const uint64_t* raw_offsets, const uint32_t* raw_offsets32,
                      const VeloGecInput* gec, uint32_t n_events, void* stream, VeloOutputs* out,
                      const uint32_t* event_list, uint32_t n_raw)
{
  if (!c || (!raw && n_events) || (!raw_offsets && !raw_offsets32 && n_events)) return VELO_ERR_INVALID;
  if (gec && n_events && (!gec->ut_raw || !gec->ut_offsets || !gec->scifi_raw || !gec->scifi_offsets))
    return VELO_ERR_INVALID;
  if (n_events > c->cfg.max_events) return VELO_ERR_CAPACITY;
  if (c->mode == VELO_MODE_PRUNED && !c->mlp_loaded) return VELO_ERR_STATE;
  if (c->mode == VELO_MODE_LABELS && !c->labels_ready) return VELO_ERR_STATE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  c->last_stream = s;
  c->last_n = n_events;
  fill_outputs(c, n_events, out);
  if (gec && out) {
    out->event_list = c->d_event_list;
    out->n_selected = c->d_n_selected;
    out->gec_counts = c->d_gec_counts;
    out->gec_flags = c->d_gec_flags;
  }
  if (n_events == 0) {
    VCK(cudaMemsetAsync(c->d_atomics, 0, sizeof(uint32_t), s));
    VCK(cudaMemsetAsync(c->d_track_hit_number, 0, sizeof(uint32_t), s));
    VCK(cudaMemsetAsync(c->d_event_hit_offset, 0, sizeof(uint32_t), s));
    if (gec) VCK(cudaMemsetAsync(c->d_n_selected, 0, sizeof(uint32_t), s));
    return 0;
  }
  // the run's inputs, where the kernels read them
  RunParams v{};
  v.raw = static_cast<const uint8_t*>(raw);
  v.raw_offsets = raw_offsets;
  v.raw_offsets32 = raw_offsets ? nullptr : raw_offsets32;
  v.n_events = n_events;
  v.event_list = event_list;
  v.n_raw = n_raw;
  if (gec) {
    v.gec_max = gec->max_clusters;
    v.ut_raw = static_cast<const uint8_t*>(gec->ut_raw);
    v.ut_offsets = gec->ut_offsets;
    v.scifi_raw = static_cast<const uint8_t*>(gec->scifi_raw);
    v.scifi_offsets = gec->scifi_offsets;
  }
  set_run_kernel<<<1, 32, 0, s>>>(c->d_run, v, c->d_queue);
  VCK(cudaGetLastError());
  const uint32_t n_grid = c->cfg.use_graphs ? bucket_of(c, n_events) : n_events;
  ChainPointers P = pointers(c, n_grid);
  GecPointers G{};
  if (gec) {
    G = GecPointers{c->d_run, c->d_gec_counts, c->d_gec_flags, c->d_event_list, c->d_n_selected};
    P.event_list = c->d_event_list;
    P.n_selected = c->d_n_selected;
  }
  const GecPointers* Gp = gec ? &G : nullptr;
  if (c->cfg.use_graphs) {
    const VeloCtx::GraphKey key{n_grid, s, gec != nullptr};
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
      if (c->graphs.size() >= VeloCtx::kMaxGraphs) {  // evict the least recently launched
        auto old = c->graphs.find(c->lru.back());
        VCK(cudaStreamSynchronize(old->first.stream));
        cudaGraphExecDestroy(old->second.exec);
        cudaGraphDestroy(old->second.graph);
        c->lru.pop_back();
        c->graphs.erase(old);
      }
      cudaStream_t cap = s;
      bool tmp = false;
      if (cap == nullptr) {  // the legacy default stream cannot be captured
        VCK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        tmp = true;
      }
      // with timing on, the capture records set 0's events: they only mark the nodes
      c->ev_current = c->timing ? 0 : -1;
      cudaGraph_t g;
      VCK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
      const int rc = launch_chain(c, P, Gp, cap, true);
      cudaError_t ce = cudaStreamEndCapture(cap, &g);
      if (tmp) cudaStreamDestroy(cap);
      if (rc != 0) return rc;
      VCK(ce);
      VeloCtx::GraphEntry entry{};
      entry.graph = g;
      entry.timed = c->timing;
      entry.launches = c->launches;
      if (entry.timed) {
        size_t nn = 0;
        VCK(cudaGraphGetNodes(g, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        VCK(cudaGraphGetNodes(g, nodes.data(), &nn));
        for (cudaGraphNode_t node : nodes) {
          cudaGraphNodeType type;
          VCK(cudaGraphNodeGetType(node, &type));
          if (type != cudaGraphNodeTypeEventRecord) continue;
          cudaEvent_t ev;
          VCK(cudaGraphEventRecordNodeGetEvent(node, &ev));
          for (int i = 0; i < VeloCtx::kStageEvents; ++i)
            if (c->ev_sets[0][i] == ev) entry.ev_nodes[i] = node;
        }
      }
      VCK(cudaGraphInstantiate(&entry.exec, g, 0));
      c->lru.push_front(key);
      entry.lru = c->lru.begin();
      it = c->graphs.emplace(key, entry).first;
    } else {
      c->lru.splice(c->lru.begin(), c->lru, it->second.lru);
    }
    if (c->timing && it->second.timed) {
      // this launch records into the next set of the pool
      const int k = static_cast<int>(c->ev_next++ % kEventSets);
      for (int i = 0; i < VeloCtx::kStageEvents; ++i)
        if (it->second.ev_nodes[i]) VCK(cudaGraphExecEventRecordNodeSetEvent(it->second.exec, it->second.ev_nodes[i],
                                                                          c->ev_sets[k][i]));
      c->ev_used[k] = 1;
    }
    VCK(cudaGraphLaunch(it->second.exec, s));
    c->launches = it->second.launches + 1;  // the graph's kernels and set_run_kernel
    return 0;
  }
  c->ev_current = -1;
  if (c->timing) {
    c->ev_current = static_cast<int>(c->ev_next++ % kEventSets);
    c->ev_used[c->ev_current] = 1;
  }
  const int rc = launch_chain(c, P, Gp, s);
  ++c->launches;  // set_run_kernel
  return rc;
}

// Reads the run's totals (tracks, track hits, error bits) into the pinned h_totals on the
// run's stream, queued right behind the run so that velo_sync only waits: a read queued at
// sync time would wait behind whatever the caller queued on the stream's copy engine since.
static int queue_totals(VeloCtx* c, cudaStream_t s, uint32_t n)
{
  VCK(cudaMemcpyAsync(c->h_totals, c->d_atomics + 2 * n, 4, cudaMemcpyDeviceToHost, s));
  VCK(cudaMemcpyAsync(c->h_totals + 1, c->d_event_hit_offset + n, 4, cudaMemcpyDeviceToHost, s));
  VCK(cudaMemcpyAsync(c->h_totals + 2, c->d_queue + 6, 4, cudaMemcpyDeviceToHost, s));
  return 0;
}

static int run_chain(VeloCtx* c, const void* raw, const uint64_t* raw_offsets, const uint32_t* raw_offsets32,
                     const VeloGecInput* gec, uint32_t n_events, void* stream, VeloOutputs* out,
                     const uint32_t* event_list = nullptr, uint32_t n_raw = 0)
{
  const int rc = launch_run(c, raw, raw_offsets, raw_offsets32, gec, n_events, stream, out, event_list, n_raw);
  if (rc) return rc;
  return queue_totals(c, static_cast<cudaStream_t>(stream), n_events);
}

int velo_run(VeloCtx* c, const void* raw, const uint64_t* raw_offsets, uint32_t n_events, void* stream,
             VeloOutputs* out)
{
  if (!raw_offsets && n_events) return VELO_ERR_INVALID;
  return run_chain(c, raw, raw_offsets, nullptr, nullptr, n_events, stream, out);
}

int velo_run_u32(VeloCtx* c, const void* raw, const uint32_t* raw_offsets, uint32_t n_events, void* stream,
                 VeloOutputs* out)
{
  if (!raw_offsets && n_events) return VELO_ERR_INVALID;
  return run_chain(c, raw, nullptr, raw_offsets, nullptr, n_events, stream, out);
}

int velo_run_selected_u32(VeloCtx* c, const void* raw, const uint32_t* raw_offsets, uint32_t n_raw,
                          const uint32_t* event_list, uint32_t n_events, void* stream, VeloOutputs* out)
{
  if ((!raw_offsets || !event_list) && n_events) return VELO_ERR_INVALID;
  return run_chain(c, raw, nullptr, raw_offsets, nullptr, n_events, stream, out, event_list, n_raw);
}

int velo_run_gec(VeloCtx* c, const void* raw, const uint64_t* raw_offsets, const VeloGecInput* gec,
                 uint32_t n_events, void* stream, VeloOutputs* out)
{
  if (!gec || (!raw_offsets && n_events)) return VELO_ERR_INVALID;
  return run_chain(c, raw, raw_offsets, nullptr, gec, n_events, stream, out);
}

// Host offsets go through the context's pinned staging (rebased on the way), so that their
// copy is asynchronous whatever memory the caller's offsets live in: a copy from pageable
// memory may wait for the stream's earlier work. begin_upload waits until the previous run's
// copies out of the staging have completed (long before, in a pipeline); end_upload marks them.
static int begin_upload(VeloCtx* c)
{
  if (c->offsets_pending) VCK(cudaEventSynchronize(c->ev_offsets));
  c->offsets_pending = false;
  return 0;
}

static int end_upload(VeloCtx* c, cudaStream_t s)
{
  VCK(cudaEventRecord(c->ev_offsets, s));
  c->offsets_pending = true;
  return 0;
}

// Copies a host batch (bytes from offsets[0] to offsets[n], offsets[n + 1]) to device buffers,
// with the offsets rebased to the batch's first byte through staging slot `slot`.
static int upload_batch(VeloCtx* c, const void* raw_host, const uint64_t* offsets_host, uint32_t n, uint8_t* d_raw,
                        uint64_t* d_offsets, cudaStream_t s, int slot)
{
  const uint64_t first = offsets_host[0];
  const uint64_t bytes = offsets_host[n] - first;
  VCK(cudaMemcpyAsync(d_raw, static_cast<const uint8_t*>(raw_host) + first, bytes, cudaMemcpyHostToDevice, s));
  uint64_t* staged = c->h_offsets + static_cast<size_t>(slot) * (c->cfg.max_events + 1);
  for (uint32_t i = 0; i <= n; ++i) staged[i] = offsets_host[i] - first;
  VCK(cudaMemcpyAsync(d_offsets, staged, 8ull * (n + 1), cudaMemcpyHostToDevice, s));
  return 0;
}

// Grows a staging buffer to hold `bytes` (the graphs that recorded the old address go).
static int ensure_staging(VeloCtx* c, uint8_t*& p, size_t& cap, uint64_t bytes)
{
  if (bytes <= cap && p) return 0;
  drop_graphs(c);
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  const size_t want = std::max<size_t>(bytes + bytes / 4, 1 << 20);
  VCK(cudaMalloc(reinterpret_cast<void**>(&p), want));
  cap = want;
  return 0;
}

int velo_run_gec_host(VeloCtx* c, const void* raw_host, const uint64_t* raw_offsets_host,
                      const VeloGecInput* gec_host, uint32_t n_events, void* stream, VeloOutputs* out)
{
  if (!c || !raw_host || !raw_offsets_host || !gec_host || !gec_host->ut_raw || !gec_host->ut_offsets ||
      !gec_host->scifi_raw || !gec_host->scifi_offsets)
    return VELO_ERR_INVALID;
  if (n_events > c->cfg.max_events) return VELO_ERR_CAPACITY;
  if (raw_offsets_host[n_events] - raw_offsets_host[0] > c->cfg.max_raw_bytes) return VELO_ERR_CAPACITY;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  const uint64_t ut_bytes = gec_host->ut_offsets[n_events] - gec_host->ut_offsets[0];
  const uint64_t scifi_bytes = gec_host->scifi_offsets[n_events] - gec_host->scifi_offsets[0];
  int rc = ensure_staging(c, c->d_gec_ut, c->gec_ut_cap, ut_bytes);
  if (rc == 0) rc = ensure_staging(c, c->d_gec_scifi, c->gec_scifi_cap, scifi_bytes);
  if (rc == 0) rc = begin_upload(c);
  if (rc == 0) rc = upload_batch(c, raw_host, raw_offsets_host, n_events, c->d_raw, c->d_raw_offsets, s, 0);
  if (rc == 0)
    rc = upload_batch(c, gec_host->ut_raw, gec_host->ut_offsets, n_events, c->d_gec_ut, c->d_gec_ut_offsets, s, 1);
  if (rc == 0)
    rc = upload_batch(c, gec_host->scifi_raw, gec_host->scifi_offsets, n_events, c->d_gec_scifi,
                      c->d_gec_scifi_offsets, s, 2);
  if (rc == 0) rc = end_upload(c, s);
  if (rc) return rc;
  const VeloGecInput dev{c->d_gec_ut, c->d_gec_ut_offsets, c->d_gec_scifi, c->d_gec_scifi_offsets,
                         gec_host->max_clusters};
  return run_chain(c, c->d_raw, c->d_raw_offsets, nullptr, &dev, n_events, stream, out);
}

// Copies a host batch with u32 offsets (bytes from offsets[0] to offsets[n]) to the
// context's device buffers, the offsets rebased through the pinned staging.
static int upload_batch_u32(VeloCtx* c, const void* raw_host, const uint32_t* offsets_host, uint32_t n, cudaStream_t s)
{
  const uint32_t first = offsets_host[0];
  const uint64_t bytes = static_cast<uint64_t>(offsets_host[n]) - first;
  int rc = begin_upload(c);
  if (rc) return rc;
  VCK(cudaMemcpyAsync(c->d_raw, static_cast<const uint8_t*>(raw_host) + first, bytes, cudaMemcpyHostToDevice, s));
  uint32_t* staged = reinterpret_cast<uint32_t*>(c->h_offsets);
  for (uint32_t i = 0; i <= n; ++i) staged[i] = offsets_host[i] - first;
  VCK(cudaMemcpyAsync(c->d_raw_offsets32, staged, 4ull * (n + 1), cudaMemcpyHostToDevice, s));
  return end_upload(c, s);
}

int velo_run_host_u32(VeloCtx* c, const void* raw_host, const uint32_t* raw_offsets_host, uint32_t n_events,
                      void* stream, VeloOutputs* out)
{
  if (!c || !raw_host || !raw_offsets_host) return VELO_ERR_INVALID;
  if (n_events > c->cfg.max_events) return VELO_ERR_CAPACITY;
  if (static_cast<uint64_t>(raw_offsets_host[n_events]) - raw_offsets_host[0] > c->cfg.max_raw_bytes)
    return VELO_ERR_CAPACITY;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  const int rc = upload_batch_u32(c, raw_host, raw_offsets_host, n_events, s);
  if (rc) return rc;
  return velo_run_u32(c, c->d_raw, c->d_raw_offsets32, n_events, stream, out);
}

int velo_run_host(VeloCtx* c, const void* raw_host, const uint64_t* raw_offsets_host, uint32_t n_events, void* stream,
                  VeloOutputs* out)
{
  if (!c || !raw_host || !raw_offsets_host) return VELO_ERR_INVALID;
  if (n_events > c->cfg.max_events) return VELO_ERR_CAPACITY;
  if (raw_offsets_host[n_events] - raw_offsets_host[0] > c->cfg.max_raw_bytes) return VELO_ERR_CAPACITY;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  int rc = begin_upload(c);
  if (rc == 0) rc = upload_batch(c, raw_host, raw_offsets_host, n_events, c->d_raw, c->d_raw_offsets, s, 0);
  if (rc == 0) rc = end_upload(c, s);
  if (rc) return rc;
  return velo_run(c, c->d_raw, c->d_raw_offsets, n_events, stream, out);
}

int velo_sync(VeloCtx* c, uint32_t* total_tracks, uint32_t* total_track_hits, uint64_t* total_clusters)
{
  if (!c) return VELO_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  cudaStream_t s = c->last_stream;
  const uint32_t N = c->last_n;
  VCK(cudaStreamSynchronize(s));  // the totals were queued behind the run
  if (c->h_totals[2]) return VELO_ERR_DEVICE_TIMEOUT;
  if (total_tracks) *total_tracks = c->h_totals[0];
  if (total_track_hits) *total_track_hits = c->h_totals[1];
  if (total_clusters) {
    std::vector<uint32_t> hits(N);
    if (N) VCK(cudaMemcpy(hits.data(), c->d_event_hits, 4ull * N, cudaMemcpyDeviceToHost));
    uint64_t t = 0;
    for (uint32_t v : hits) t += v;
    *total_clusters = t;
  }
  return 0;
}

int velo_set_mlp(VeloCtx* c, const void* weights_host, size_t bytes)
{
  if (!c || !weights_host || bytes != sizeof(VeloMlpWeights)) return VELO_ERR_INVALID;
  const VeloMlpWeights& w = *static_cast<const VeloMlpWeights*>(weights_host);
  if (!(w.seed_threshold > 0.f && w.seed_threshold < 1.f) || !(w.ext_threshold >= 0.f && w.ext_threshold < 1.f))
    return VELO_ERR_INVALID;
  // bf16 slots: W1 [64][16], W2 [64][80], W3 [16][80], bias in the ones column, zero pads
  std::vector<__nv_bfloat16> slots(kMlpParams, __float2bfloat16_rn(0.f));
  for (int j = 0; j < 64; ++j)
    for (int i = 0; i < 13; ++i) slots[j * kMlpK1 + i] = __float2bfloat16_rn(w.w1[j][i]);
  for (int j = 0; j < 64; ++j)
    for (int i = 0; i < 65; ++i) slots[kMlpW1 + j * kMlpK2 + i] = __float2bfloat16_rn(w.w2[j][i]);
  for (int o = 0; o < 2; ++o)
    for (int i = 0; i < 65; ++i) slots[kMlpW1 + kMlpW2 + o * kMlpK2 + i] = __float2bfloat16_rn(w.w3[o][i]);
  float norm[32] = {};
  for (int k = 0; k < 12; ++k) {
    norm[k] = w.mean[k];
    norm[16 + k] = w.inv_std[k];
  }
  drop_graphs(c);  // the launch parameters change
  VCK(cudaMemcpy(c->d_mlp_w, slots.data(), kMlpParams * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
  VCK(cudaMemcpy(c->d_mlp_norm, norm, sizeof norm, cudaMemcpyHostToDevice));
  auto logit = [](float p) { return std::log(p / (1.f - p)); };
  c->mlp.w = c->d_mlp_w;
  c->mlp.norm = c->d_mlp_norm;
  c->mlp.seed_logit = logit(w.seed_threshold);
  c->mlp.use_ext = w.ext_threshold > 0.f ? 1u : 0u;
  c->mlp.ext_logit = w.ext_threshold > 0.f ? logit(w.ext_threshold) : 0.f;
  c->mlp.max_hits = w.max_event_clusters;
  c->mlp.min_pairs = w.min_pairs;
  c->mlp.min_hits = w.min_event_clusters;
  c->mlp_loaded = true;
  return 0;
}

int velo_capture_labels(VeloCtx* c, int ext, uint32_t max_event_clusters)
{
  if (!c) return VELO_ERR_INVALID;
  if (c->mode != VELO_MODE_PLAIN || c->last_n == 0) return VELO_ERR_STATE;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  if (!c->d_labels) VCK(dalloc(c->d_labels, c->hit_capacity));
  drop_graphs(c);  // the launch parameters of the label mode change
  const ChainPointers P = pointers(c, c->last_n);
  capture_labels_kernel<<<std::min<uint32_t>(c->last_n, 8u * c->sm_count), 256, 0, c->last_stream>>>(
    P, c->d_labels, max_event_clusters);
  VCK(cudaGetLastError());
  VCK(cudaStreamSynchronize(c->last_stream));
  c->labels_ready = true;
  c->labels_ext = ext ? 1u : 0u;
  c->labels_max_hits = max_event_clusters;
  return 0;
}

int velo_set_mode(VeloCtx* c, uint32_t mode)
{
  if (!c || (mode != VELO_MODE_PLAIN && mode != VELO_MODE_PRUNED && mode != VELO_MODE_LABELS)) return VELO_ERR_INVALID;
  if (mode == VELO_MODE_PRUNED) {
    if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
    const int rc = ensure_pruned_buffers(c);
    if (rc) return rc;
  }
  if (mode != c->mode) drop_graphs(c);
  c->mode = mode;
  return 0;
}

int velo_set_pv(VeloCtx* c, int enabled)
{
  if (!c) return VELO_ERR_INVALID;
  if ((enabled != 0) != c->pv) drop_graphs(c);  // the launch sequence changes
  c->pv = enabled != 0;
  return 0;
}

int velo_set_timing(VeloCtx* c, int enabled)
{
  if (!c) return VELO_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  if (enabled && !c->timing) {
    // graphs captured without the stage events are captured again, with them
    bool untimed = false;
    for (auto& kv : c->graphs) untimed |= !kv.second.timed;
    if (untimed) drop_graphs(c);
  }
  while (c->ev_sets.size() < kEventSets) {
    const int rc = add_event_set(c);
    if (rc < 0) return rc;
  }
  std::fill(c->ev_used.begin(), c->ev_used.end(), 0);
  c->timing = enabled != 0;
  return 0;
}

// Sums, over every event set recorded since velo_set_timing, the device time of the six
// stages (the last, the PV stage, is 0 when it is off); ms[6] (when n > 6) receives the
// number of launch sequences summed.
int velo_stage_times(VeloCtx* c, float* ms, int n)
{
  constexpr int kStages = 7;  // six chain stages and the global event cut
  if (!c || !ms || n < kStages) return VELO_ERR_INVALID;
  if (c->ev_sets.empty()) return VELO_ERR_STATE;
  float acc[kStages] = {};
  int runs = 0;
  for (size_t k = 0; k < c->ev_sets.size(); ++k) {
    if (!c->ev_used[k]) continue;
    for (int i = 0; i < kStages; ++i) {
      float t = 0.f;
      const int a = i < kStages - 1 ? i : 7, b = i < kStages - 1 ? i + 1 : 8;
      VCK(cudaEventElapsedTime(&t, c->ev_sets[k][a], c->ev_sets[k][b]));
      acc[i] += t;
    }
    ++runs;
  }
  for (int i = 0; i < kStages; ++i) ms[i] = acc[i];
  if (n > kStages) ms[kStages] = static_cast<float>(runs);
  return 0;
}

int velo_download(VeloCtx* c, void* dst_host, const void* src_device, size_t bytes)
{
  if (!c || (!dst_host && bytes) || (!src_device && bytes)) return VELO_ERR_INVALID;
  if (bytes == 0) return 0;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  VCK(cudaMemcpy(dst_host, src_device, bytes, cudaMemcpyDeviceToHost));
  return 0;
}

int velo_download_async(VeloCtx* c, void* dst_host, const void* src_device, size_t bytes, void* stream)
{
  if (!c || (!dst_host && bytes) || (!src_device && bytes)) return VELO_ERR_INVALID;
  if (bytes == 0) return 0;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  VCK(cudaMemcpyAsync(dst_host, src_device, bytes, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
  return 0;
}

int velo_set_decode_warps(VeloCtx* c, uint32_t warps)
{
  if (!c || (warps != 4 && warps != 8)) return VELO_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  if (static_cast<int>(warps) != c->decode_warps) drop_graphs(c);  // the launch sequence changes
  c->decode_warps = static_cast<int>(warps);
  size_decode_grid(c);
  return cudaGetLastError() == cudaSuccess ? 0 : VELO_ERR_CUDA;
}

int velo_set_block_threshold(VeloCtx* c, uint32_t clusters)
{
  if (!c) return VELO_ERR_INVALID;
  if (clusters != c->block_threshold) drop_graphs(c);  // the launch sequence changes
  c->block_threshold = clusters;
  return 0;
}

int velo_check_wait_timeout(VeloCtx* c, uint32_t polls, void* stream)
{
  if (!c || polls == 0 || polls > (1u << 20)) return VELO_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  c->last_stream = s;
  VCK(cudaMemsetAsync(c->d_queue + 6, 0, sizeof(uint32_t), s));
  wait_timeout_kernel<<<1, 32, 0, s>>>(c->d_queue + 6, polls);
  VCK(cudaGetLastError());
  VCK(cudaMemcpyAsync(c->h_totals + 2, c->d_queue + 6, 4, cudaMemcpyDeviceToHost, s));  // read by velo_sync
  return 0;
}

int velo_graph_count(VeloCtx* c, uint32_t* n)
{
  if (!c || !n) return VELO_ERR_INVALID;
  *n = static_cast<uint32_t>(c->graphs.size());
  return 0;
}

int velo_last_launch_count(VeloCtx* c, uint32_t* n)
{
  if (!c || !n) return VELO_ERR_INVALID;
  *n = c->launches;
  return 0;
}

int velo_destroy(VeloCtx* c)
{
  if (!c) return VELO_ERR_INVALID;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  free_all(c);
  delete c;
  return 0;
}

}  // extern "C"

bool velo_ctx_last_run(VeloCtx* c, ChainPointers* P, cudaStream_t* stream, int* device)
{
  if (!c || !P || c->last_n == 0) return false;
  *P = pointers(c, c->last_n);
  *stream = c->last_stream;
  *device = c->device;
  return true;
}
