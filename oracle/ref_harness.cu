// ORACLE — test infrastructure only. Launch harness for the reference's own VELO kernels
// (Qwicen/cuda_hlt cuda/velo, cuda/utils/prefix_sum), compiled from the reference tree by
// oracle/build.py into oracle/_ref/libvelo_ref_gpu.so. It replays the launch sequence of
// configuration/sequences/Velo.h:5-18 plus velo_kalman_fit_t, with the grid/block shapes,
// buffer sizes and host synchronisation points of the visitors in
// stream/visitors/velo/src/*.cu, so the kernels run exactly as the reference runs them.
// The event list of the VELO chain is the identity (init_event_list, InitEventList.cu:7);
// global_event_cut runs on its own through ref_gec_run.
//
// Every buffer carries a padding tail so that the reference's unchecked writes past an
// event's region (more than 1200 tracks, 500 weak tracklets or 3000 clustering candidates)
// stay inside this harness's allocations; callers only pass events whose per-module
// cluster count fits the reference's 500-entry shared phi buffer, which the harness checks
// on the host before the phi sort runs.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "CalculatePhiAndSort.cuh"
#include "ClusteringCommon.h"
#include "ConsolidateVelo.cuh"
#include "EstimateInputSize.cuh"
#include "GlobalEventCut.cuh"
#include "FillCandidates.cuh"
#include "MaskedVeloClustering.cuh"
#include "PrefixSum.cuh"
#include "SearchByTriplet.cuh"
#include "VeloKalmanFilter.cuh"
#include "WeakTracksAdder.cuh"
#include "pv_beamline_extrapolate.cuh"
#include "pv_beamline_histo.cuh"
#include "pv_beamline_multi_fitter.cuh"
#include "pv_beamline_peak.cuh"

namespace {

constexpr size_t kPad = 8u << 20;  // bytes of padding behind every device buffer

struct Buf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes)
  {
    if (bytes + kPad <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    cap = bytes + kPad;
    cudaError_t e = cudaMalloc(&p, cap);
    if (e != cudaSuccess) {
      p = nullptr;
      cap = 0;
      return e;
    }
    return cudaMemset(p, 0, cap);
  }
  template<class T>
  T* as() const
  {
    return static_cast<T*>(p);
  }
  ~Buf()
  {
    if (p) cudaFree(p);
  }
};

struct Ctx {
  Buf raw, offsets, event_list, event_order, est, mod_num, cand_num, cands, aux1, container, perm, h0, h2, tracks,
    tracklets, ttf, weak, hit_used, atomics, rel, hit_number, aux2, track_hits, states, kalman;
  Buf geometry, module_zs, cand_ks, sp_patterns, sp_fx, sp_fy;
  uint32_t *h_total = nullptr, *h_tracks = nullptr, *h_hits = nullptr;
  cudaStream_t stream = nullptr;
};

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) {                                                                    \
      std::fprintf(stderr, "ref_harness: %s failed: %s\n", #x, cudaGetErrorString(e_));        \
      return -2;                                                                                \
    }                                                                                           \
  } while (0)

size_t aux_size(size_t n)
{
  const size_t s = (n + 511) / 512;
  return s > 0 ? s : 1;
}

// PREFIX_SUM_ALGORITHM invoke (cuda/utils/prefix_sum/include/PrefixSumHandler.cuh:243-267)
void prefix_sum(uint* array, uint* aux, size_t n, cudaStream_t s)
{
  const size_t a = aux_size(n);
  const size_t scan_blocks = a == 1 ? 1 : a - 1;
  prefix_sum_reduce<<<dim3(a), dim3(256), 0, s>>>(array, aux, n);
  prefix_sum_single_block<<<dim3(1), dim3(1024), 0, s>>>(array + n, aux, a);
  prefix_sum_scan<<<dim3(scan_blocks), dim3(512), 0, s>>>(array, aux, n);
}

}  // namespace

extern "C" {

struct RefOutputs {
  uint32_t n_events;
  uint32_t total_estimated;   // container stride (prefix sum of estimates)
  uint32_t total_tracks, total_track_hits;
  uint32_t* module_start;     // [N*52+1]
  uint32_t* module_num;       // [N*52]
  uint32_t* container;        // [6*total_estimated]: Y|Z|ID|stale|phi|X after the sort
  uint32_t* candidate_num;    // [N]
  uint32_t* weak_num;         // [N] weak tracklets per event (before the adder consumed them)
  uint32_t* atomics;          // [2N+1]
  uint32_t* track_hit_number; // [T+1]
  uint8_t* track_hits;        // H*16: SoA x,y,z,id
  uint8_t* states;            // T*sizeof(VeloState): SoA
  uint8_t* kalman;            // T*sizeof(VeloState): SoA
};

void ref_free(RefOutputs* o)
{
  if (!o) return;
  free(o->module_start);
  free(o->module_num);
  free(o->container);
  free(o->candidate_num);
  free(o->weak_num);
  free(o->atomics);
  free(o->track_hit_number);
  free(o->track_hits);
  free(o->states);
  free(o->kalman);
  std::memset(o, 0, sizeof(*o));
}

// Runs the reference sequence `reps` times on the same events (device-resident input after
// the first copy). ms_per_rep: average device time of one full sequence (including its
// host synchronisations and result copies, as the visitors issue them). Returns 0, -1 on
// bad arguments, -2 on a CUDA error, -3 when a module exceeds the 500-entry phi buffer.
int ref_velo_run(const void* raw, const uint32_t* offsets, uint32_t n_events, const void* geometry, int reps,
                 float* ms_per_rep, RefOutputs* out)
{
  if (!raw || !offsets || !geometry || n_events == 0 || reps < 1) return -1;
  Ctx c;
  const uint32_t N = n_events;
  CK(cudaStreamCreate(&c.stream));
  CK(cudaMallocHost(&c.h_total, 4));
  CK(cudaMallocHost(&c.h_tracks, 4));
  CK(cudaMallocHost(&c.h_hits, 4));
  // Constants (stream/sequence/src/Constants.cu:3-53)
  {
    const float zs[52] = {-287.5, -275,  -262.5, -250,  -237.5, -225,  -212.5, -200,  -137.5, -125,  -62.5, -50,   -37.5,
                          -25,    -12.5, 0,      12.5,  25,     37.5,  50,     62.5,  75,     87.5,  100,   112.5, 125,
                          137.5,  150,   162.5,  175,   187.5,  200,   212.5,  225,   237.5,  250,   262.5, 275,   312.5,
                          325,    387.5, 400,    487.5, 500,    587.5, 600,    637.5, 650,    687.5, 700,   737.5, 750};
    const uint8_t ks[9] = {0, 0, 1, 4, 4, 5, 5, 5, 5};
    std::vector<uint8_t> pat(256, 0), sizes(256, 0);
    std::vector<float> fx(512, 0), fy(512, 0);
    cache_sp_patterns(pat, sizes, fx, fy);
    CK(c.geometry.ensure(19456));
    CK(c.module_zs.ensure(sizeof zs));
    CK(c.cand_ks.ensure(9));
    CK(c.sp_patterns.ensure(256));
    CK(c.sp_fx.ensure(2048));
    CK(c.sp_fy.ensure(2048));
    CK(cudaMemcpy(c.geometry.p, geometry, 19456, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.module_zs.p, zs, sizeof zs, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.cand_ks.p, ks, 9, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.sp_patterns.p, pat.data(), 256, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.sp_fx.p, fx.data(), 2048, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.sp_fy.p, fy.data(), 2048, cudaMemcpyHostToDevice));
  }
  const size_t raw_bytes = offsets[N];
  CK(c.raw.ensure(raw_bytes));
  CK(c.offsets.ensure(4ull * (N + 1)));
  CK(cudaMemcpy(c.raw.p, raw, raw_bytes, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.offsets.p, offsets, 4ull * (N + 1), cudaMemcpyHostToDevice));
  {
    std::vector<uint32_t> list(N);
    for (uint32_t i = 0; i < N; ++i) list[i] = i;
    CK(c.event_list.ensure(4ull * N));
    CK(c.event_order.ensure(4ull * N));
    CK(cudaMemcpy(c.event_list.p, list.data(), 4ull * N, cudaMemcpyHostToDevice));
  }
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  float total_ms = 0.f;
  std::vector<uint32_t> h_mod_num(N * 52);
  std::vector<uint32_t> h_weak_atomics;
  const cudaStream_t s = c.stream;

  for (int rep = 0; rep < reps; ++rep) {
    CK(cudaEventRecord(t0, s));
    // velo_estimate_input_size_t (EstimateInputSizeVisitor.cu:8-55)
    CK(c.est.ensure(4ull * (N * 52 + 1)));
    CK(c.mod_num.ensure(4ull * N * 52));
    CK(c.cand_num.ensure(4ull * N));
    CK(c.cands.ensure(4ull * N * 3000));
    estimate_input_size<<<dim3(N), dim3(32, 26), 0, s>>>(
      c.raw.as<char>(), c.offsets.as<uint>(), c.est.as<uint>(), c.mod_num.as<uint>(), c.cand_num.as<uint>(),
      c.cands.as<uint32_t>(), c.event_list.as<uint>(), c.event_order.as<uint>(), c.cand_ks.as<uint8_t>());
    // prefix_sum_velo_clusters_t (PrefixSumVeloClustersVisitor.cu:8-48): host sync 1
    CK(c.aux1.ensure(4ull * aux_size(N * 52)));
    prefix_sum(c.est.as<uint>(), c.aux1.as<uint>(), N * 52, s);
    CK(cudaMemcpyAsync(c.h_total, c.est.as<uint>() + N * 52, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const uint32_t total = *c.h_total;
    // velo_masked_clustering_t
    CK(c.container.ensure(4ull * 6 * total));
    masked_velo_clustering<<<dim3(N), dim3(256), 0, s>>>(
      c.raw.as<char>(), c.offsets.as<uint>(), c.est.as<uint>(), c.mod_num.as<uint>(), c.cand_num.as<uint>(),
      c.cands.as<uint>(), c.container.as<uint32_t>(), c.event_list.as<uint>(), c.event_order.as<uint>(),
      c.geometry.as<char>(), c.sp_patterns.as<uint8_t>(), c.sp_fx.as<float>(), c.sp_fy.as<float>());
    if (rep == 0) {
      // Host check of the shared phi buffer bound before calculate_phi_and_sort runs.
      CK(cudaMemcpyAsync(h_mod_num.data(), c.mod_num.p, 4ull * N * 52, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (uint32_t v : h_mod_num)
        if (v >= 500) return -3;
    }
    // velo_calculate_phi_and_sort_t
    CK(c.perm.ensure(4ull * total));
    calculate_phi_and_sort<<<dim3(N), dim3(64), 0, s>>>(c.est.as<uint>(), c.mod_num.as<uint>(),
                                                         c.container.as<uint32_t>(), c.perm.as<uint>());
    // velo_fill_candidates_t
    CK(c.h0.ensure(2ull * 2 * total));
    CK(c.h2.ensure(2ull * 2 * total));
    fill_candidates<<<dim3(N, 48), dim3(128), 0, s>>>(c.container.as<uint>(), c.est.as<uint>(), c.mod_num.as<uint>(),
                                                       c.h0.as<short>(), c.h2.as<short>());
    // velo_search_by_triplet_t (SearchByTripletVisitor.cu:8-56)
    CK(c.tracks.ensure(sizeof(Velo::TrackHits) * N * 1200));
    CK(c.tracklets.ensure(sizeof(Velo::TrackletHits) * N * 2000));
    CK(c.ttf.ensure(4ull * N * 2000));
    CK(c.weak.ensure(sizeof(Velo::TrackletHits) * N * 500));
    CK(c.hit_used.ensure(total));
    CK(c.atomics.ensure(4ull * N * 5));
    CK(c.rel.ensure(2ull * N * 2 * 500));
    search_by_triplet<<<dim3(N), dim3(32), 32 * sizeof(float), s>>>(
      c.container.as<uint32_t>(), c.est.as<uint>(), c.mod_num.as<uint>(), c.tracks.as<Velo::TrackHits>(),
      c.tracklets.as<Velo::TrackletHits>(), c.ttf.as<uint>(), c.weak.as<Velo::TrackletHits>(), c.hit_used.as<bool>(),
      c.atomics.as<int>(), c.h0.as<short>(), c.h2.as<short>(), c.rel.as<unsigned short>(), c.module_zs.as<float>());
    // velo_weak_tracks_adder_t
    weak_tracks_adder<<<dim3(N), dim3(256), 0, s>>>(c.container.as<uint32_t>(), c.est.as<uint>(),
                                                     c.tracks.as<Velo::TrackHits>(), c.weak.as<Velo::TrackletHits>(),
                                                     c.hit_used.as<bool>(), c.atomics.as<int>());
    if (rep == reps - 1 && out) {
      h_weak_atomics.resize(5ull * N);
      CK(cudaMemcpyAsync(h_weak_atomics.data(), c.atomics.p, 4ull * 5 * N, cudaMemcpyDeviceToHost, s));
    }
    // copy_and_prefix_sum_single_block_velo_t (CopyAndPrefixSumVisitor.cu): host sync 2
    copy_and_prefix_sum_single_block<<<dim3(1), dim3(1024), 0, s>>>(c.atomics.as<uint>() + 2 * N, c.atomics.as<uint>(),
                                                                    c.atomics.as<uint>() + N, N);
    CK(cudaMemcpyAsync(c.h_tracks, c.atomics.as<uint>() + 2 * N, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const uint32_t T = *c.h_tracks;
    // copy_velo_track_hit_number_t
    CK(c.hit_number.ensure(4ull * (T + 1)));
    copy_velo_track_hit_number<<<dim3(N), dim3(512), 0, s>>>(c.tracks.as<Velo::TrackHits>(), c.atomics.as<int>(),
                                                              c.hit_number.as<uint>());
    // prefix_sum_velo_track_hit_number_t: host sync 3
    CK(c.aux2.ensure(4ull * aux_size(T)));
    prefix_sum(c.hit_number.as<uint>(), c.aux2.as<uint>(), T, s);
    CK(cudaMemcpyAsync(c.h_hits, c.hit_number.as<uint>() + T, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const uint32_t H = *c.h_hits;
    // consolidate_velo_tracks_t (ConsolidateVeloVisitor.cu:8-67)
    CK(c.track_hits.ensure(16ull * H));
    CK(c.states.ensure(sizeof(VeloState) * T));
    consolidate_velo_tracks<<<dim3(N), dim3(256), 0, s>>>(c.atomics.as<int>(), c.tracks.as<Velo::TrackHits>(),
                                                           c.hit_number.as<uint>(), c.container.as<uint>(),
                                                           c.est.as<uint>(), c.mod_num.as<uint>(),
                                                           c.track_hits.as<char>(), c.states.as<char>());
    // velo_kalman_fit_t (KalmanFilterVisitor.cu:8-45)
    CK(c.kalman.ensure(sizeof(VeloState) * T));
    velo_kalman_fit<<<dim3(N), dim3(256), 0, s>>>(c.atomics.as<int>(), c.hit_number.as<uint>(),
                                                   c.track_hits.as<char>(), c.states.as<char>(), c.kalman.as<char>());
    CK(cudaGetLastError());
    CK(cudaEventRecord(t1, s));
    CK(cudaEventSynchronize(t1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, t0, t1));
    if (rep > 0 || reps == 1) total_ms += ms;

    if (rep == reps - 1 && out) {
      std::memset(out, 0, sizeof(*out));
      out->n_events = N;
      out->total_estimated = total;
      out->total_tracks = T;
      out->total_track_hits = H;
      out->module_start = static_cast<uint32_t*>(malloc(4ull * (N * 52 + 1)));
      out->module_num = static_cast<uint32_t*>(malloc(4ull * N * 52));
      out->container = static_cast<uint32_t*>(malloc(4ull * 6 * total + 4));
      out->candidate_num = static_cast<uint32_t*>(malloc(4ull * N));
      out->weak_num = static_cast<uint32_t*>(malloc(4ull * N));
      out->atomics = static_cast<uint32_t*>(malloc(4ull * (2 * N + 1)));
      out->track_hit_number = static_cast<uint32_t*>(malloc(4ull * (T + 1)));
      out->track_hits = static_cast<uint8_t*>(malloc(16ull * H + 16));
      out->states = static_cast<uint8_t*>(malloc(sizeof(VeloState) * T + 16));
      out->kalman = static_cast<uint8_t*>(malloc(sizeof(VeloState) * T + 16));
      CK(cudaMemcpy(out->module_start, c.est.p, 4ull * (N * 52 + 1), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(out->module_num, c.mod_num.p, 4ull * N * 52, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(out->container, c.container.p, 4ull * 6 * total, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(out->candidate_num, c.cand_num.p, 4ull * N, cudaMemcpyDeviceToHost));
      for (uint32_t e = 0; e < N; ++e) out->weak_num[e] = h_weak_atomics[N + 4 * e];
      CK(cudaMemcpy(out->atomics, c.atomics.p, 4ull * (2 * N + 1), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(out->track_hit_number, c.hit_number.p, 4ull * (T + 1), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(out->track_hits, c.track_hits.p, 16ull * H, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(out->states, c.states.p, sizeof(VeloState) * T, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(out->kalman, c.kalman.p, sizeof(VeloState) * T, cudaMemcpyDeviceToHost));
    }
  }
  if (ms_per_rep) *ms_per_rep = total_ms / (reps > 1 ? reps - 1 : 1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFreeHost(c.h_total);
  cudaFreeHost(c.h_tracks);
  cudaFreeHost(c.h_hits);
  cudaStreamDestroy(c.stream);
  return 0;
}

int ref_state_size(void) { return static_cast<int>(sizeof(VeloState)); }
int ref_pv_vertex_size(void) { return static_cast<int>(sizeof(PV::Vertex)); }

// The reference's beamline PV finder (cuda/PV/beamlinePV: pv_beamline_extrapolate_t,
// pv_beamline_histo_t, pv_beamline_peak_t, pv_beamline_multi_fitter_t of
// DefaultSequence.h:20-23) on consolidated VELO tracks: atomics[2N+1], track_hit_number[T+1]
// and Kalman beamline states (sizeof(VeloState) * T bytes, the States SoA). Launch shapes
// and the vertex-count memset of stream/visitors/beamlinePV/src/*.cu. Outputs: the z
// histograms [N * Nbins], peaks [N * 32] with counts [N], vertices [N * 32] with counts [N].
int ref_pv_run(const uint32_t* atomics, const uint32_t* track_hit_number, const void* kalman, uint32_t n_events,
               float* zhisto, float* zpeaks, uint32_t* n_peaks, void* vertices, uint32_t* n_vertices, int reps,
               float* ms_per_rep)
{
  if (!atomics || !track_hit_number || !kalman || n_events == 0) return -1;
  const uint32_t N = n_events, T = atomics[2 * N];
  cudaStream_t s;
  CK(cudaStreamCreate(&s));
  Buf d_atomics, d_hn, d_kal, d_trk, d_histo, d_peaks, d_npeaks, d_vtx, d_nvtx;
  CK(d_atomics.ensure(4ull * (2 * N + 1)));
  CK(d_hn.ensure(4ull * (T + 1)));
  CK(d_kal.ensure(sizeof(VeloState) * (T > 0 ? T : 1)));
  CK(d_trk.ensure(sizeof(PVTrack) * (T > 0 ? T : 1)));
  CK(d_histo.ensure(4ull * N * Nbins));
  CK(d_peaks.ensure(4ull * N * PV::max_number_vertices));
  CK(d_npeaks.ensure(4ull * N));
  CK(d_vtx.ensure(sizeof(PV::Vertex) * N * PV::max_number_vertices));
  CK(d_nvtx.ensure(4ull * N));
  CK(cudaMemcpy(d_atomics.p, atomics, 4ull * (2 * N + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_hn.p, track_hit_number, 4ull * (T + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_kal.p, kalman, sizeof(VeloState) * T, cudaMemcpyHostToDevice));
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  float total_ms = 0.f;
  for (int rep = 0; rep < (reps > 0 ? reps : 1); ++rep) {
  CK(cudaEventRecord(t0, s));
  pv_beamline_extrapolate<<<dim3(N), dim3(128), 0, s>>>(static_cast<char*>(d_kal.p), static_cast<int*>(d_atomics.p),
                                                        static_cast<uint*>(d_hn.p), static_cast<PVTrack*>(d_trk.p));
  pv_beamline_histo<<<dim3(N), dim3(128), 0, s>>>(static_cast<int*>(d_atomics.p), static_cast<uint*>(d_hn.p),
                                                  static_cast<PVTrack*>(d_trk.p), static_cast<float*>(d_histo.p));
  pv_beamline_peak<<<dim3((N + PV::num_threads_pv_beamline_peak_t - 1) / PV::num_threads_pv_beamline_peak_t),
                     dim3(PV::num_threads_pv_beamline_peak_t), 0, s>>>(
    static_cast<float*>(d_histo.p), static_cast<float*>(d_peaks.p), static_cast<uint*>(d_npeaks.p), N);
  CK(cudaMemsetAsync(d_nvtx.p, 0, 4ull * N, s));
  pv_beamline_multi_fitter<<<dim3(N), dim3(32), 0, s>>>(
    static_cast<int*>(d_atomics.p), static_cast<uint*>(d_hn.p), static_cast<PVTrack*>(d_trk.p),
    static_cast<float*>(d_peaks.p), static_cast<uint*>(d_npeaks.p), static_cast<PV::Vertex*>(d_vtx.p),
    static_cast<uint*>(d_nvtx.p));
  CK(cudaEventRecord(t1, s));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, t0, t1));
  if (rep > 0 || reps <= 1) total_ms += ms;  // the first of several repetitions warms up
  }
  if (ms_per_rep) *ms_per_rep = total_ms / (reps > 1 ? reps - 1 : 1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (zhisto) CK(cudaMemcpy(zhisto, d_histo.p, 4ull * N * Nbins, cudaMemcpyDeviceToHost));
  if (zpeaks) CK(cudaMemcpy(zpeaks, d_peaks.p, 4ull * N * PV::max_number_vertices, cudaMemcpyDeviceToHost));
  if (n_peaks) CK(cudaMemcpy(n_peaks, d_npeaks.p, 4ull * N, cudaMemcpyDeviceToHost));
  if (vertices)
    CK(cudaMemcpy(vertices, d_vtx.p, sizeof(PV::Vertex) * N * PV::max_number_vertices, cudaMemcpyDeviceToHost));
  if (n_vertices) CK(cudaMemcpy(n_vertices, d_nvtx.p, 4ull * N, cudaMemcpyDeviceToHost));
  cudaStreamDestroy(s);  // the buffers free themselves
  return 0;
}
}

// global_event_cut (GlobalEventCut.cu:3-55) launched as GlobalEventCutVisitor.cu does: one
// block of 32 threads per event, the selected-event counter zeroed first. Offsets are u32, as
// the reference takes them. The kernel returns from some threads before a __syncthreads when
// an event's running UT count reaches the cut; callers pass only events whose UT hit total
// is below the cut, so that every thread of a block reaches every barrier. Outputs: the
// number of selected events and the event list in the kernel's (atomic) order, and the mean
// device time of one counter reset + kernel over reps - 1 repetitions after the first.
extern "C" int ref_gec_run(const void* ut, const uint32_t* ut_offsets, const void* scifi, const uint32_t* scifi_offsets,
                           uint32_t n_events, uint32_t* n_selected, uint32_t* event_list, int reps, float* ms_per_rep)
{
  if (!ut || !ut_offsets || !scifi || !scifi_offsets || !n_selected || !event_list || n_events == 0) return -1;
  const uint32_t N = n_events;
  Buf d_ut, d_ut_off, d_sf, d_sf_off, d_n, d_list;
  CK(d_ut.ensure(ut_offsets[N]));
  CK(d_ut_off.ensure(4ull * (N + 1)));
  CK(d_sf.ensure(scifi_offsets[N]));
  CK(d_sf_off.ensure(4ull * (N + 1)));
  CK(d_n.ensure(4));
  CK(d_list.ensure(4ull * N));
  CK(cudaMemcpy(d_ut.p, ut, ut_offsets[N], cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_ut_off.p, ut_offsets, 4ull * (N + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_sf.p, scifi, scifi_offsets[N], cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_sf_off.p, scifi_offsets, 4ull * (N + 1), cudaMemcpyHostToDevice));
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  const int R = reps > 0 ? reps : 1;
  float total_ms = 0.f;
  for (int rep = 0; rep < R; ++rep) {
    CK(cudaEventRecord(t0));
    CK(cudaMemsetAsync(d_n.p, 0, 4));
    global_event_cut<<<dim3(N), dim3(32)>>>(static_cast<char*>(d_ut.p), static_cast<uint*>(d_ut_off.p),
                                            static_cast<char*>(d_sf.p), static_cast<uint*>(d_sf_off.p),
                                            static_cast<uint*>(d_n.p), static_cast<uint*>(d_list.p));
    CK(cudaGetLastError());
    CK(cudaEventRecord(t1));
    CK(cudaEventSynchronize(t1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, t0, t1));
    if (rep > 0 || R == 1) total_ms += t;
  }
  if (ms_per_rep) *ms_per_rep = total_ms / (R > 1 ? R - 1 : 1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  CK(cudaMemcpy(n_selected, d_n.p, 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(event_list, d_list.p, 4ull * N, cudaMemcpyDeviceToHost));
  return 0;
}
