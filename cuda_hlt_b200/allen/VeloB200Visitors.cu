/*
 * VeloB200Visitors.cu — SequenceVisitor specialisations of the VELO algorithms of
 * VeloB200Sequence.cuh: the visitors of stream/visitors/velo/src/*.cu for the B200 chain.
 *
 * The visitors keep the reference's interface (stream/sequence/include/SequenceVisitor.cuh:
 * set_arguments_size sizes the arguments from host-known counts; visit launches and copies
 * results to the host buffers) and its host buffers: host_number_of_reconstructed_velo_tracks
 * and host_accumulated_number_of_hits_in_velo_tracks (CopyAndPrefixSumVisitor.cu,
 * PrefixSumVeloTrackHitNumberVisitor.cu), host_atomics_velo, host_velo_track_hit_number,
 * host_velo_track_hits (ConsolidateVeloVisitor.cu) and host_kalmanvelo_states
 * (KalmanFilterVisitor.cu). Errors throw StrException, as the reference's memory manager does
 * (cudaCheck throws std::invalid_argument for CUDA errors).
 */
#include <string>
#include <vector>

#include "SequenceVisitor.cuh"
#include "States.cuh"
#include "VeloB200Sequence.cuh"
#include "VeloEventModel.cuh"

namespace {

constexpr size_t kVeloGeometryBytes = 19456;  // the VeloGeometry layout (ClusteringDefinitions.cu:23-53)
constexpr size_t kStateBytes = 12 * sizeof(float) + sizeof(bool);  // Velo::Consolidated::States per track

void velo_b200_check(int rc, const char* what)
{
  if (rc != VELO_OK) throw StrException(std::string("velo_b200: ") + what + " returned " + std::to_string(rc));
}

// Capacity of the calling thread's context.
struct Capacity {
  uint32_t events = 0;
  size_t raw_bytes = 0;
};
thread_local Capacity g_capacity;

}  // namespace

VeloB200StreamState& velo_b200_stream_state()
{
  static thread_local VeloB200StreamState state;
  return state;
}

// ---- velo_estimate_input_size_t: the whole chain on the selected events ----
DEFINE_EMPTY_SET_ARGUMENTS_SIZE(velo_estimate_input_size_t)

template<>
void SequenceVisitor::visit<velo_estimate_input_size_t>(
  velo_estimate_input_size_t&,
  const velo_estimate_input_size_t::arguments_t& arguments,
  const RuntimeOptions& runtime_options,
  const Constants& constants,
  HostBuffers& host_buffers,
  cudaStream_t& cuda_stream,
  cudaEvent_t&)
{
  auto& st = velo_b200_stream_state();
  const uint n_selected = host_buffers.host_number_of_selected_events[0];
  const uint n_raw = runtime_options.number_of_events;
  if (st.ctx && (n_raw > g_capacity.events || runtime_options.host_velopix_events_size > g_capacity.raw_bytes)) {
    velo_destroy(st.ctx);  // a larger batch than the context was made for
    st.ctx = nullptr;
  }
  if (!st.ctx) {
    VeloConfig cfg {};
    cfg.max_events = n_raw;
    cfg.max_raw_bytes = runtime_options.host_velopix_events_size;
    cfg.use_graphs = 1;
    cudaCheck(cudaGetDevice(&cfg.device));
    std::vector<char> geometry(kVeloGeometryBytes);
    cudaCheck(cudaMemcpy(geometry.data(), constants.dev_velo_geometry, geometry.size(), cudaMemcpyDeviceToHost));
    velo_b200_check(velo_create(&cfg, geometry.data(), geometry.size(), &st.ctx), "velo_create");
    g_capacity = Capacity {n_raw, runtime_options.host_velopix_events_size};
  }
  st.n_events = n_selected;
  velo_b200_check(
    velo_run_selected_u32(
      st.ctx,
      arguments.offset<dev_velo_raw_input>(),
      arguments.offset<dev_velo_raw_input_offsets>(),
      n_raw,
      arguments.offset<dev_event_list>(),
      n_selected,
      cuda_stream,
      &st.out),
    "velo_run_selected_u32");
}

// ---- algorithms whose work is inside the chain ----
#define VELO_B200_NOTHING_TO_DO(_TYPE)                                                                           \
  DEFINE_EMPTY_SET_ARGUMENTS_SIZE(_TYPE)                                                                         \
  template<>                                                                                                     \
  void SequenceVisitor::visit<_TYPE>(                                                                            \
    _TYPE&, const _TYPE::arguments_t&, const RuntimeOptions&, const Constants&, HostBuffers&, cudaStream_t&,     \
    cudaEvent_t&)                                                                                                \
  {}

VELO_B200_NOTHING_TO_DO(prefix_sum_velo_clusters_t)
VELO_B200_NOTHING_TO_DO(velo_masked_clustering_t)
VELO_B200_NOTHING_TO_DO(velo_calculate_phi_and_sort_t)
VELO_B200_NOTHING_TO_DO(velo_fill_candidates_t)
VELO_B200_NOTHING_TO_DO(velo_search_by_triplet_t)
VELO_B200_NOTHING_TO_DO(velo_weak_tracks_adder_t)
VELO_B200_NOTHING_TO_DO(copy_velo_track_hit_number_t)

// ---- the host reads of the totals ----
DEFINE_EMPTY_SET_ARGUMENTS_SIZE(copy_and_prefix_sum_single_block_velo_t)

template<>
void SequenceVisitor::visit<copy_and_prefix_sum_single_block_velo_t>(
  copy_and_prefix_sum_single_block_velo_t&,
  const copy_and_prefix_sum_single_block_velo_t::arguments_t&,
  const RuntimeOptions&,
  const Constants&,
  HostBuffers& host_buffers,
  cudaStream_t&,
  cudaEvent_t&)
{
  auto& st = velo_b200_stream_state();
  velo_b200_check(velo_sync(st.ctx, &st.tracks, &st.track_hits, nullptr), "velo_sync");
  host_buffers.host_number_of_reconstructed_velo_tracks[0] = st.tracks;
}

DEFINE_EMPTY_SET_ARGUMENTS_SIZE(prefix_sum_velo_track_hit_number_t)

template<>
void SequenceVisitor::visit<prefix_sum_velo_track_hit_number_t>(
  prefix_sum_velo_track_hit_number_t&,
  const prefix_sum_velo_track_hit_number_t::arguments_t&,
  const RuntimeOptions&,
  const Constants&,
  HostBuffers& host_buffers,
  cudaStream_t&,
  cudaEvent_t&)
{
  host_buffers.host_accumulated_number_of_hits_in_velo_tracks[0] = velo_b200_stream_state().track_hits;
}

// ---- the consolidated outputs into Allen's arguments ----
template<>
void SequenceVisitor::set_arguments_size<consolidate_velo_tracks_t>(
  consolidate_velo_tracks_t::arguments_t arguments,
  const RuntimeOptions&,
  const Constants&,
  const HostBuffers& host_buffers)
{
  const uint n = host_buffers.host_number_of_selected_events[0];
  const uint tracks = host_buffers.host_number_of_reconstructed_velo_tracks[0];
  arguments.set_size<dev_atomics_velo>(2 * n + 1);
  arguments.set_size<dev_velo_track_hit_number>(tracks + 1);
  arguments.set_size<dev_velo_track_hits>(
    host_buffers.host_accumulated_number_of_hits_in_velo_tracks[0] * sizeof(Velo::Hit));
  arguments.set_size<dev_velo_states>(tracks * sizeof(VeloState));
  arguments.set_size<dev_accepted_velo_tracks>(tracks);
}

template<>
void SequenceVisitor::visit<consolidate_velo_tracks_t>(
  consolidate_velo_tracks_t&,
  const consolidate_velo_tracks_t::arguments_t& arguments,
  const RuntimeOptions&,
  const Constants&,
  HostBuffers& host_buffers,
  cudaStream_t& cuda_stream,
  cudaEvent_t&)
{
  const auto& st = velo_b200_stream_state();
  const size_t n = st.n_events, tracks = st.tracks, hits = st.track_hits;
  cudaCheck(cudaMemcpyAsync(
    arguments.offset<dev_atomics_velo>(), st.out.atomics, (2 * n + 1) * sizeof(uint), cudaMemcpyDeviceToDevice,
    cuda_stream));
  cudaCheck(cudaMemcpyAsync(
    arguments.offset<dev_velo_track_hit_number>(), st.out.track_hit_number, (tracks + 1) * sizeof(uint),
    cudaMemcpyDeviceToDevice, cuda_stream));
  cudaCheck(cudaMemcpyAsync(
    arguments.offset<dev_velo_track_hits>(), st.out.track_hits, hits * sizeof(Velo::Hit), cudaMemcpyDeviceToDevice,
    cuda_stream));
  cudaCheck(cudaMemcpyAsync(
    arguments.offset<dev_velo_states>(), st.out.states, tracks * kStateBytes, cudaMemcpyDeviceToDevice, cuda_stream));
  // every track accepted, as ConsolidateVeloVisitor.cu does
  cudaCheck(cudaMemsetAsync(arguments.offset<dev_accepted_velo_tracks>(), 1, tracks, cuda_stream));
  cudaCheck(cudaMemcpyAsync(
    host_buffers.host_atomics_velo, st.out.atomics, (2 * n + 1) * sizeof(uint), cudaMemcpyDeviceToHost, cuda_stream));
  cudaCheck(cudaMemcpyAsync(
    host_buffers.host_velo_track_hit_number, st.out.track_hit_number, (tracks + 1) * sizeof(uint),
    cudaMemcpyDeviceToHost, cuda_stream));
  cudaCheck(cudaMemcpyAsync(
    host_buffers.host_velo_track_hits, st.out.track_hits, hits * sizeof(Velo::Hit), cudaMemcpyDeviceToHost,
    cuda_stream));
}

// ---- the Kalman beamline states ----
template<>
void SequenceVisitor::set_arguments_size<velo_kalman_fit_t>(
  velo_kalman_fit_t::arguments_t arguments,
  const RuntimeOptions&,
  const Constants&,
  const HostBuffers& host_buffers)
{
  arguments.set_size<dev_velo_kalman_beamline_states>(
    host_buffers.host_number_of_reconstructed_velo_tracks[0] * sizeof(VeloState));
}

template<>
void SequenceVisitor::visit<velo_kalman_fit_t>(
  velo_kalman_fit_t&,
  const velo_kalman_fit_t::arguments_t& arguments,
  const RuntimeOptions&,
  const Constants&,
  HostBuffers& host_buffers,
  cudaStream_t& cuda_stream,
  cudaEvent_t&)
{
  const auto& st = velo_b200_stream_state();
  const size_t bytes = st.tracks * kStateBytes;
  cudaCheck(cudaMemcpyAsync(
    arguments.offset<dev_velo_kalman_beamline_states>(), st.out.kalman_states, bytes, cudaMemcpyDeviceToDevice,
    cuda_stream));
  cudaCheck(cudaMemcpyAsync(
    host_buffers.host_kalmanvelo_states, st.out.kalman_states, bytes, cudaMemcpyDeviceToHost, cuda_stream));
}
