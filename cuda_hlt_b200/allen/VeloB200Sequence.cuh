/*
 * VeloB200Sequence.cuh — the VELO algorithms of LHCb Allen's sequences, backed by the B200
 * chain (include/velo_b200.h).
 *
 * A maintainer puts this header on Allen's include path in place of the VELO algorithm
 * declarations (EstimateInputSize.cuh, MaskedVeloClustering.cuh, CalculatePhiAndSort.cuh,
 * SearchByTriplet.cuh, ConsolidateVelo.cuh, VeloKalmanFilter.cuh and the VELO lines of
 * PrefixSum.cuh), compiles VeloB200Visitors.cu in place of stream/visitors/velo/src/*.cu, and
 * links libvelo_b200.so. configuration/sequences/Velo.h and DefaultSequence.h keep their lists
 * of *_t names unchanged: every name below has the shape the ALGORITHM macro gives an
 * algorithm (stream/gear/include/Handler.cuh:12-32: name, Arguments, arguments_t, set_opts,
 * set_arguments, invoke), so the compile-time scheduler (stream/gear/include/Scheduler.cuh)
 * reserves and frees their arguments as before.
 *
 * What runs where:
 *   velo_estimate_input_size_t   the whole chain, asynchronously, on the events of
 *                                dev_event_list (the output of global_event_cut_t), from
 *                                dev_velo_raw_input / dev_velo_raw_input_offsets (u32) as
 *                                init_event_list_t copied them: velo_run_selected_u32
 *   prefix_sum_velo_clusters_t … velo_weak_tracks_adder_t, copy_velo_track_hit_number_t
 *                                nothing (their work is inside the chain)
 *   copy_and_prefix_sum_single_block_velo_t / prefix_sum_velo_track_hit_number_t
 *                                the host reads of the track and track-hit totals that the
 *                                reference's visitors make (velo_sync)
 *   consolidate_velo_tracks_t    the consolidated outputs into Allen's arguments
 *                                dev_atomics_velo, dev_velo_track_hit_number,
 *                                dev_velo_track_hits, dev_velo_states,
 *                                dev_accepted_velo_tracks, and their host copies
 *   velo_kalman_fit_t            dev_velo_kalman_beamline_states
 * The chain's context belongs to the host thread of the Allen Stream that runs the sequence
 * (one context per thread, as Allen runs one Stream per thread: main/src/main.cpp:239-271).
 */
#pragma once

#include <tuple>

#include "Argument.cuh"
#include "ArgumentManager.cuh"
#include "ArgumentsCommon.cuh"
#include "ArgumentsVelo.cuh"
#include "velo_b200.h"

// An algorithm of the sequence without a kernel of its own: the ALGORITHM macro's members,
// with launch options and arguments that the visitor passes to the chain instead.
#define VELO_B200_ALGORITHM(EXPOSED_TYPE_NAME, DEPENDENCIES)                                      \
  struct EXPOSED_TYPE_NAME {                                                                      \
    constexpr static auto name {#EXPOSED_TYPE_NAME};                                              \
    using Arguments = DEPENDENCIES;                                                               \
    using arguments_t = ArgumentRefManager<Arguments>;                                            \
    void set_opts(const dim3&, const dim3&, cudaStream_t&, const unsigned = 0) {}                 \
    template<typename... T>                                                                       \
    void set_arguments(T...)                                                                      \
    {}                                                                                            \
    void invoke() {}                                                                              \
  };

VELO_B200_ALGORITHM(
  velo_estimate_input_size_t,
  ARGUMENTS(dev_velo_raw_input, dev_velo_raw_input_offsets, dev_event_list))
VELO_B200_ALGORITHM(prefix_sum_velo_clusters_t, ARGUMENTS())
VELO_B200_ALGORITHM(velo_masked_clustering_t, ARGUMENTS())
VELO_B200_ALGORITHM(velo_calculate_phi_and_sort_t, ARGUMENTS())
VELO_B200_ALGORITHM(velo_fill_candidates_t, ARGUMENTS())
VELO_B200_ALGORITHM(velo_search_by_triplet_t, ARGUMENTS())
VELO_B200_ALGORITHM(velo_weak_tracks_adder_t, ARGUMENTS())
VELO_B200_ALGORITHM(copy_and_prefix_sum_single_block_velo_t, ARGUMENTS())
VELO_B200_ALGORITHM(copy_velo_track_hit_number_t, ARGUMENTS())
VELO_B200_ALGORITHM(prefix_sum_velo_track_hit_number_t, ARGUMENTS())
VELO_B200_ALGORITHM(
  consolidate_velo_tracks_t,
  ARGUMENTS(
    dev_atomics_velo,
    dev_velo_track_hit_number,
    dev_velo_track_hits,
    dev_velo_states,
    dev_accepted_velo_tracks))
VELO_B200_ALGORITHM(velo_kalman_fit_t, ARGUMENTS(dev_velo_kalman_beamline_states))

// The calling thread's chain context and the outputs of its last run (VeloB200Visitors.cu).
struct VeloB200StreamState {
  VeloCtx* ctx = nullptr;
  VeloOutputs out {};
  uint32_t n_events = 0;
  uint32_t tracks = 0;
  uint32_t track_hits = 0;
};
VeloB200StreamState& velo_b200_stream_state();
