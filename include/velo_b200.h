/*
 * velo_b200.h — C ABI of the B200-native HLT1 VELO reconstruction chain.
 *
 * The chain replaces the VELO stage of LHCb Allen (Qwicen/cuda_hlt): the algorithms
 *   init_event_list            cuda/global_event_cut/src/InitEventList.cu:7
 *   estimate_input_size        cuda/velo/mask_clustering/src/EstimateInputSize.cu:3
 *   prefix_sum_velo_clusters   cuda/utils/prefix_sum/include/PrefixSumHandler.cuh:270
 *   masked_velo_clustering     cuda/velo/mask_clustering/src/MaskedVeloClustering.cu:48
 *   calculate_phi_and_sort     cuda/velo/calculate_phi_and_sort/src/CalculatePhiAndSort.cu:6
 *   fill_candidates            cuda/velo/search_by_triplet/src/FillCandidates.cu:72
 *   search_by_triplet          cuda/velo/search_by_triplet/src/SearchByTriplet.cu:7
 *   weak_tracks_adder          cuda/velo/search_by_triplet/src/WeakTracksAdder.cu:117
 *   copy_and_prefix_sum_single_block_velo / copy_velo_track_hit_number /
 *   prefix_sum_velo_track_hit_number
 *                              cuda/utils/prefix_sum/src/PrefixSumSingleBlock.cu:130-168
 *   consolidate_velo_tracks    cuda/velo/consolidate_tracks/src/ConsolidateVelo.cu:116
 *   velo_kalman_fit            cuda/velo/simplified_kalman_filter/src/VeloKalmanFilter.cu:43
 * as sequenced in configuration/sequences/Velo.h:5-18 (+ velo_kalman_fit_t from
 * DefaultSequence.h:19). Inputs are the raw VP banks of RuntimeOptions
 * (main/include/RuntimeOptions.h:9-55); outputs are the consolidated buffers of
 * stream/setup/include/OutputArguments.cuh:16-34 in the layouts of
 * cuda/event_model/common/include/ConsolidatedTypes.cuh:11-66 and
 * cuda/event_model/velo/include/VeloConsolidated.cuh:12-144.
 *
 * Conventions: every entry point returns 0 or a negative VELO_ERR_* code and never throws.
 * Device pointers are plain addresses; streams are cudaStream_t passed as void*. Nothing
 * blocks except velo_sync (and the host-buffer runs, until the previous run's offsets have
 * left the staging buffer). A context is used by one host thread at a time; separate
 * contexts may run concurrently on separate streams.
 */
#ifndef VELO_B200_H
#define VELO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes (the reference throws instead: main/include/CudaCommon.h:10-18,
 *      stream/gear/include/MemoryManager.cuh:78-80) ---- */
#define VELO_OK 0
#define VELO_ERR_INVALID -1      /* null pointer or bad argument */
#define VELO_ERR_CUDA -2         /* a CUDA runtime call failed */
#define VELO_ERR_CAPACITY -3     /* batch larger than the context was created for */
#define VELO_ERR_BAD_RAW -4      /* malformed raw event */
#define VELO_ERR_BAD_GEOMETRY -5 /* geometry blob has the wrong size */
#define VELO_ERR_BAD_MC -6       /* malformed MC truth blob */
#define VELO_ERR_NO_DEVICE -7    /* no CUDA device visible */
#define VELO_ERR_STATE -8        /* call out of order (e.g. pruned run without weights) */
#define VELO_ERR_DEVICE_TIMEOUT -9 /* a bounded wait in a kernel ran out (tensor core did not answer) */

/* ---- per-event status flags written by velo_run (status[N]) ---- */
#define VELO_STATUS_BAD_RAW (1u << 0)
#define VELO_STATUS_MODULE_OVERFLOW (1u << 1)
#define VELO_STATUS_HIT_OVERFLOW (1u << 2)
#define VELO_STATUS_CANDIDATE_OVERFLOW (1u << 3)
#define VELO_STATUS_TRACK_OVERFLOW (1u << 4)
#define VELO_STATUS_TTF_OVERFLOW (1u << 5)
#define VELO_STATUS_WEAK_OVERFLOW (1u << 6)
#define VELO_STATUS_H1_OVERFLOW (1u << 7)
#define VELO_STATUS_BIG_SP_INDEX (1u << 8)
#define VELO_STATUS_MLP_FALLBACK (1u << 9)
#define VELO_STATUS_PV_OVERFLOW (1u << 13) /* PV stage: peaks, clusters or extrema beyond the
                                              reference's fixed arrays (it writes past them) */
#define VELO_STATUS_NOT_SELECTED (1u << 14) /* velo_run_gec: position at or beyond the number of
                                               selected events (left empty) */

/* ======================================================================
 * Host utilities (libvelo_host.so; no GPU needed)
 * ====================================================================== */

/* SuperPixel pattern tables (same contents as cache_sp_patterns,
 * x86/velo/clustering/src/ClusteringCommon.cpp:3-101; uploaded to the device by
 * Constants::initialize_constants, stream/sequence/src/Constants.cu:45-53).
 * patterns[256], sizes[256], fx[512], fy[512]. */
void velo_build_sp_luts(uint8_t* patterns, uint8_t* sizes, float* fx, float* fy);

/* Checks one raw event in the layout of cuda/velo/readme.md (the reader-side check is
 * main/src/CheckVP.cpp:5-51). Returns 0 or VELO_ERR_BAD_RAW. */
int velo_validate_raw_event(const void* event, uint64_t event_bytes);

/* Seeded synthetic events: straight tracks from Poisson primary vertices through the real
 * VELO geometry, encoded as SuperPixel raw banks, with MC truth in the MC_info layout of
 * checker/tracking/src/MCEvent.cpp:16-92. Event i depends only on (seed, i). */
typedef struct VeloGenConfig {
  uint64_t seed;
  float nu_min, nu_max;         /* pileup per event, uniform in [nu_min, nu_max] */
  float visible_fraction;       /* primary vertices ~ Poisson(nu * visible_fraction) */
  float tracks_per_pv;          /* charged tracks per vertex ~ Poisson(tracks_per_pv) */
  float backward_fraction;      /* eta ~ U(-4,-2) with this probability, else U(2,5) */
  float pv_sigma_xy, pv_sigma_z;/* mm */
  float hit_efficiency;         /* per sensor crossing */
  float p_one_pixel, p_two_pixels; /* cluster size 1/2/3 pixel probabilities (rest = 3) */
  float noise_per_asic_per_nu;  /* random pixels per 256x256 ASIC ~ Poisson(this * nu) */
  float noisy_event_fraction;   /* events with noise scaled by noisy_factor */
  float noisy_factor;
} VeloGenConfig;
typedef struct VeloGenBatch VeloGenBatch;
void velo_gen_default_config(VeloGenConfig* cfg);
int velo_gen_create(const VeloGenConfig* cfg, const void* geometry, uint64_t first_event, uint32_t n_events,
                    int n_threads, VeloGenBatch** out);
uint64_t velo_gen_raw_bytes(const VeloGenBatch* b);
uint64_t velo_gen_mc_bytes(const VeloGenBatch* b);
/* raw_offsets / mc_offsets: n_events+1 byte offsets. truth_clusters: n_events (deposits). */
int velo_gen_copy(const VeloGenBatch* b, void* raw, uint64_t* raw_offsets, void* mc, uint64_t* mc_offsets,
                  uint32_t* truth_clusters);
void velo_gen_destroy(VeloGenBatch* b);

/* MC-truth checker for consolidated VELO tracks: the matching of
 * checker/tracking/src/TrackChecker.cpp:349-405 and checker/tracking/include/MCAssociator.h:166-182
 * (ghost = no MCP with weight >= 0.7), categories "Not electron long eta25"
 * (checker/tracking/src/CategoriesTrackChecker.cpp:120) and "Not electron Velo" (:215). */
typedef struct VeloCheckResult {
  uint64_t events, tracks, ghosts;
  uint64_t long_reconstructible, long_found, long_clones;
  uint64_t velo_reconstructible, velo_found, velo_clones;
  double long_efficiency, velo_efficiency, ghost_rate, ghost_rate_per_event;
} VeloCheckResult;
int velo_check_tracks(const void* mc_blob, const uint64_t* mc_offsets, uint32_t n_events,
                      const uint32_t* event_track_offsets, const uint32_t* track_hit_offsets, const uint32_t* hit_ids,
                      VeloCheckResult* res);

/* MDF reader: the VP raw banks of the events of an LHCb MDF file in the raw layout velo_run
 * takes (number of banks, byte offsets, per bank its source id and body), with the ODIN run
 * and event number of each event. Replaces MDF::read_events (mdf/src/read_mdf.cpp:29-191,
 * driven by MDFReader::read_events, main/src/MDFReader.cpp:15-63) for BankTypes::VP on one
 * file: skips `first_event` events, then reads up to `max_events`. zlib-compressed records
 * (ROOT blocks) are expanded and record checksums verified. Errors: VELO_ERR_INVALID (no
 * file), VELO_ERR_BAD_RAW (bad header, checksum, compressed block or raw bank; the
 * reference prints and stops at the first such record, or, for a bad bank magic, goes on). */
typedef struct VeloMdfEvents VeloMdfEvents;
int velo_mdf_read(const char* path, uint64_t first_event, uint64_t max_events, VeloMdfEvents** out);
/* Same for the banks of another LHCb raw bank type (LHCb::RawBank::BankType numbers,
 * mdf/include/raw_bank.hpp: VP 63, FTCluster 64, UT 66, Muon 13), e.g. the UT and SciFi
 * inputs of velo_run_gec; the layout per event is the same. */
#define VELO_BANK_VP 63u
#define VELO_BANK_FTCLUSTER 64u
#define VELO_BANK_UT 66u
#define VELO_BANK_MUON 13u
int velo_mdf_read_banks(const char* path, uint64_t first_event, uint64_t max_events, uint32_t bank_type,
                        VeloMdfEvents** out);
uint64_t velo_mdf_count(const VeloMdfEvents* events);
uint64_t velo_mdf_raw_bytes(const VeloMdfEvents* events);
/* raw[raw_bytes], offsets[count + 1] (u64 byte offsets), run[count], event[count]; any may be null */
int velo_mdf_copy(const VeloMdfEvents* events, void* raw, uint64_t* offsets, uint32_t* run, uint64_t* event);
void velo_mdf_free(VeloMdfEvents* events);

/* ======================================================================
 * GPU chain (libvelo_b200.so)
 * ====================================================================== */
typedef struct VeloCtx VeloCtx;

#define VELO_MODE_PLAIN 0  /* exhaustive search_by_triplet (reference semantics) */
#define VELO_MODE_PRUNED 1 /* learned seed/extension scorer prunes the search */
#define VELO_MODE_LABELS 2 /* pruned by the plain search's own labels of the same batch
                              (velo_capture_labels): a perfect scorer at no cost, which measures
                              how much pruning can save at most */

/* Search mapping (velo_set_block_threshold sets the boundary directly). */
#define VELO_MAP_AUTO 0    /* search: block per event above 1,536 clusters, warp per event below */
#define VELO_MAP_BLOCK 1   /* search: one block per event */
#define VELO_MAP_WARP 2    /* search: one warp per event */

typedef struct VeloConfig {
  uint32_t max_events;          /* events per velo_run call */
  uint64_t max_raw_bytes;       /* raw input bytes per call */
  uint32_t max_tracks;          /* consolidated tracks per call (0: 400 per event) */
  uint32_t max_track_hits;      /* consolidated track hits per call (0: 16 per track) */
  int32_t device;               /* CUDA device ordinal */
  uint32_t mode;                /* VELO_MODE_* */
  uint32_t mapping;             /* VELO_MAP_* */
  uint32_t use_graphs;          /* capture the launch sequence in CUDA graphs, one per batch-size
                                   bucket (1,024 events x a power of 4, at most max_events), stream
                                   and global event cut on/off; the kernels read each run's inputs
                                   from a device-side parameter block, so a graph serves every
                                   batch of its bucket wherever its buffers are; at most 16 graphs
                                   are kept, the least recently launched evicted first */
} VeloConfig;

/* Output buffers of one velo_run call: device pointers, valid until the next velo_run on
 * the same context. Layouts are the reference's:
 *   atomics[2N+1]        tracks per event [0,N), exclusive offsets [N,2N], T = atomics[2N]
 *   track_hit_number[T+1] exclusive scan of hits per track, H = track_hit_number[T]
 *   track_hits           Velo::Consolidated::Hits SoA: float x[H], y[H], z[H], u32 LHCbID[H]
 *   states / kalman_states Velo::Consolidated::States SoA over T: float x,y,tx,ty,c00,c20,c22,
 *                        c11,c31,c33,chi2,z [T] each, then bool backward[T]
 * Cluster container after the phi sort (for parity checks and downstream use):
 *   module_hit_start[N*52], module_hit_num[N*52] (starts are absolute indices; gaps allowed),
 *   hit_xyzp (4 floats per cluster: x, y, z, phi) and hit_id indexed by those starts,
 *   hit_size (pixels of each cluster, at most 3) and, in VELO_MODE_PRUNED, hit_keep (the
 *   scorer's bits per hit: bit 0 seed keep, bit 1 extension keep; both set on every hit of an
 *   event the scorer does not score, below its event gate or above its trained occupancy;
 *   NULL in the plain mode). */
typedef struct VeloOutputs {
  uint32_t n_events;
  uint32_t* atomics;
  uint32_t* track_hit_number;
  char* track_hits;
  char* states;
  char* kalman_states;
  uint32_t* status;
  uint32_t* module_hit_start;
  uint32_t* module_hit_num;
  float* hit_xyzp;
  uint32_t* hit_id;
  uint64_t hit_capacity;
  uint8_t* hit_size;
  uint8_t* hit_keep;
  /* beamline PV stage (velo_set_pv; null when off) */
  void* pv_vertices;     /* VeloPvVertex[n_events * VELO_PV_MAX_VERTICES], per event in seed order */
  uint32_t* pv_count;    /* [n_events] vertices of each event */
  float* pv_zpeaks;      /* [n_events * VELO_PV_MAX_VERTICES] z of the histogram peaks (seeds) */
  uint32_t* pv_npeaks;   /* [n_events] */
  /* global event cut (velo_run_gec; null after velo_run). Positions 0 .. *n_selected - 1 of
   * every per-event output above hold the selected raw events event_list[0 ..], in ascending
   * order; later positions are empty (VELO_STATUS_NOT_SELECTED). */
  uint32_t* event_list;  /* [n_events] dev_event_list */
  uint32_t* n_selected;  /* [1] dev_number_of_selected_events */
  uint32_t* gec_counts;  /* [2 * n_events] per raw event: SciFi cluster estimate, UT hits
                            (0xFFFFFFFF: malformed bank table) */
  uint8_t* gec_flags;    /* [n_events] per raw event: VELO_GEC_PASS | VELO_GEC_MALFORMED */
  /* fill_candidates output (dev_h0_candidates / dev_h2_candidates of FillCandidates.cu:72):
   * per hit of modules 2..49, indexed like hit_xyzp, two u32 {first | last << 16} of its h0
   * window (module + 2) and h2 window (module - 2), event-relative, 0xFFFF: none; in
   * VELO_MODE_PRUNED a pruned seed has no h0 window */
  uint32_t* hit_windows;
} VeloOutputs;

/* A primary vertex, in the layout of PV::Vertex (cuda/PV/beamlinePV/include/PV_Definitions.cuh:64-109). */
#define VELO_PV_MAX_VERTICES 32
typedef struct VeloPvVertex {
  float x, y, z;
  float chi2;
  int32_t ndof;      /* left unset by the reference; 0 */
  uint32_t n_tracks; /* as the reference counts them: every track of the event */
  float cov00, cov10, cov11, cov20, cov21, cov22;
  int32_t n_tracks_unused;
} VeloPvVertex;

/* Creates a context: device buffers for cfg->max_events events, device constants from the
 * 19456-byte geometry blob (cuda/velo/common/src/ClusteringDefinitions.cu:23-53). */
int velo_create(const VeloConfig* cfg, const void* geometry, size_t geometry_bytes, VeloCtx** out);

/* Runs the chain on n_events raw events already in device memory: raw (byte buffer) and
 * raw_offsets[n_events+1] (u64 byte offsets of each event in raw). Asynchronous on stream. */
int velo_run(VeloCtx* ctx, const void* raw, const uint64_t* raw_offsets, uint32_t n_events, void* stream,
             VeloOutputs* out);

/* Same, from host buffers: copies the input to the context's device buffers on the stream,
 * then runs. The raw bytes are copied straight from raw_host (pin or register it for the copy
 * to overlap other work); the offsets go through a pinned staging buffer of the context,
 * rebased to the batch's first byte on the way, so their copy is asynchronous whatever memory
 * they are in. The call waits only if the previous host run's offsets have not yet left that
 * buffer. */
int velo_run_host(VeloCtx* ctx, const void* raw_host, const uint64_t* raw_offsets_host, uint32_t n_events,
                  void* stream, VeloOutputs* out);

/* velo_run and velo_run_host with u32 byte offsets, the reference's own input format
 * (RuntimeOptions::host_velopix_offsets, main/include/RuntimeOptions.h:9-55, filled by
 * main/src/InputReader.cpp:28-57): no widening pass on the caller's side. */
int velo_run_u32(VeloCtx* ctx, const void* raw, const uint32_t* raw_offsets, uint32_t n_events, void* stream,
                 VeloOutputs* out);
int velo_run_host_u32(VeloCtx* ctx, const void* raw_host, const uint32_t* raw_offsets_host, uint32_t n_events,
                      void* stream, VeloOutputs* out);

/* The chain on a selection of the batch's n_raw events (device inputs, u32 offsets[n_raw + 1]):
 * position e (< n_events) decodes raw event event_list[e] (device array), as the reference's
 * VELO kernels read dev_event_list after global_event_cut_t (EstimateInputSize.cu:14-19 and
 * the other kernels of the sequence). An entry at or beyond n_raw leaves its position empty
 * with VELO_STATUS_BAD_RAW. */
int velo_run_selected_u32(VeloCtx* ctx, const void* raw, const uint32_t* raw_offsets, uint32_t n_raw,
                          const uint32_t* event_list, uint32_t n_events, void* stream, VeloOutputs* out);

/* Global event cut in front of the chain: global_event_cut_t
 * (cuda/global_event_cut/src/GlobalEventCut.cu:3-55, configuration/sequences/Velo.h:7).
 * An event passes when its SciFi cluster estimate, (sum over FTCluster banks of (bank bytes
 * - 4)) / 2 - 2 in 32-bit unsigned arithmetic, is below max_clusters and that plus its UT
 * hit count (sum over UT banks of the low 16 bits of the bank's second word) is below
 * max_clusters too. UT and SciFi raw events have the layout of UTRaw.cuh / SciFiRaw.cuh:
 * u32 number of banks, u32 bank byte offsets [banks + 1], the banks. The chain then runs on
 * the selected events without a host synchronisation (the reference reads the selected
 * count back before its next kernel). */
#define VELO_GEC_MAX_CLUSTERS 9750u /* maxSciFiUTClusters, GlobalEventCut.cuh:9 */
#define VELO_GEC_PASS 1u
#define VELO_GEC_MALFORMED 2u       /* bank table or a UT bank header outside the event: fails */
typedef struct VeloGecInput {
  const void* ut_raw;             /* UT raw events, back to back */
  const uint64_t* ut_offsets;     /* [n_events + 1] byte offsets */
  const void* scifi_raw;          /* FTCluster raw events */
  const uint64_t* scifi_offsets;  /* [n_events + 1] */
  uint32_t max_clusters;          /* VELO_GEC_MAX_CLUSTERS */
} VeloGecInput;
/* Device inputs (all pointers device-resident). */
int velo_run_gec(VeloCtx* ctx, const void* raw, const uint64_t* raw_offsets, const VeloGecInput* gec,
                 uint32_t n_events, void* stream, VeloOutputs* out);
/* Host inputs: copies the three detectors' batches to device buffers of the context first. */
int velo_run_gec_host(VeloCtx* ctx, const void* raw_host, const uint64_t* raw_offsets_host,
                      const VeloGecInput* gec_host, uint32_t n_events, void* stream, VeloOutputs* out);

/* Waits for the context's last run (its stream); fills totals (tracks, track hits, clusters).
 * The track and track-hit totals are read into pinned memory at the end of every run, so the
 * wait does not queue behind copies issued on the stream's copy engine since. */
int velo_sync(VeloCtx* ctx, uint32_t* total_tracks, uint32_t* total_track_hits, uint64_t* total_clusters);

/* ---- learned seed/extension scorer (no counterpart in the reference) ----
 * A 12 -> 64 -> 64 -> 2 MLP scores each seeding candidate h1 of search_by_triplet
 * (TrackSeeding.cu:7-200) from one proxy triplet: the hits bracketing phi(h1) in its h0
 * and h2 windows, the pair with the smallest seeding scatter. Features, in order: tx, ty
 * of h0->h2, log(1 + 1000 * scatter), phi(h0) - phi(h1), phi(h1) - phi(h2), module index,
 * h0 window size, h2 window size, radius of h1, pixels of h1, h0, h2 (at most 3).
 * Output 0 ("seed keep") predicts that the plain search keeps h1 on a final track; output
 * 1 ("extension keep") that h1 is the fourth or a later hit of one. In VELO_MODE_PRUNED the
 * search seeds only from h1 with p0 >= seed_threshold and, when ext_threshold > 0,
 * forwards only onto hits with p1 >= ext_threshold; events with more than
 * max_event_clusters clusters run the plain search (VELO_STATUS_MLP_FALLBACK). Seeds with
 * fewer than min_pairs (h0, h2) combinations to test are kept without scoring: the scorer
 * costs the same for every candidate, the search only for the combinations it tests.
 * Inference and training run on the tensor cores in bf16 with fp32 accumulation. */
typedef struct VeloMlpWeights {
  float mean[12];               /* feature normalisation: (f - mean) * inv_std */
  float inv_std[12];
  float w1[64][13];             /* hidden 1 x (12 features, bias) */
  float w2[64][65];             /* hidden 2 x (64, bias) */
  float w3[2][65];              /* outputs x (64, bias) */
  float seed_threshold;         /* probability */
  float ext_threshold;          /* probability; 0 disables extension pruning */
  uint32_t max_event_clusters;  /* occupancy limit of the trained range */
  uint32_t min_pairs;           /* score only seeds with |h0 window| x |h2 window| >= this */
  uint32_t min_event_clusters;  /* score only in events with at least this many clusters (0: all);
                                   smaller events keep every seed, as in the plain search */
} VeloMlpWeights;

/* Loads the scorer (weights_host -> VeloMlpWeights, bytes == sizeof(VeloMlpWeights));
 * required before a run in VELO_MODE_PRUNED. */
int velo_set_mlp(VeloCtx* ctx, const void* weights_host, size_t bytes);

/* Keeps, for every hit of the last run (plain mode, after velo_sync), the labels the scorer
 * is trained on: bit 0 "on a final track", bit 1 "fourth or later hit of a final track".
 * A following run in VELO_MODE_LABELS on the same batch (same raw events and offsets, so
 * that the hits land in the same slots) seeds only from hits with bit 0 and, when ext is
 * nonzero, forwards only onto hits with bit 1; events with more than max_event_clusters
 * clusters are not pruned (VELO_STATUS_MLP_FALLBACK), as in VELO_MODE_PRUNED. Blocks until
 * the labels are written. No counterpart in the reference: a measurement of the ceiling of
 * learned pruning (the scorer's decisions replaced by the right answers, at no cost). */
int velo_capture_labels(VeloCtx* ctx, int ext, uint32_t max_event_clusters);

/* Switches the context between VELO_MODE_PLAIN, VELO_MODE_PRUNED and VELO_MODE_LABELS. */
int velo_set_mode(VeloCtx* ctx, uint32_t mode);

/* Trainer of the scorer on one device. Samples are the seeding candidates of plain runs,
 * labelled by the tracks of that run. */
typedef struct VeloMlpTrainer VeloMlpTrainer;
int velo_mlp_trainer_create(int device, uint64_t max_samples, uint64_t seed, VeloMlpTrainer** out);
int velo_mlp_trainer_destroy(VeloMlpTrainer* t);
/* Appends the candidates of the last velo_run of ctx (plain mode, after velo_sync) until
 * max_samples are held; *n_total receives the number held. */
int velo_mlp_collect(VeloMlpTrainer* t, VeloCtx* ctx, uint64_t* n_total);
/* Copies held samples [first, first+n): features[n][12], label bits[n] (bit 0 seed keep,
 * bit 1 extension keep). */
int velo_mlp_samples(VeloMlpTrainer* t, uint64_t first, uint32_t n, float* features, uint8_t* labels);
/* Sets the feature normalisation from the held samples (mean and 1/std). */
int velo_mlp_normalize(VeloMlpTrainer* t);
/* Minibatch Adam (beta 0.9 / 0.999) over the held samples, reshuffled every epoch;
 * *last_loss = mean cross-entropy of the last epoch. */
int velo_mlp_train(VeloMlpTrainer* t, uint32_t epochs, uint32_t batch, float lr, float* last_loss);
int velo_mlp_get_weights(VeloMlpTrainer* t, VeloMlpWeights* w);
int velo_mlp_set_weights(VeloMlpTrainer* t, const VeloMlpWeights* w);
/* Gradient of the mean cross-entropy over n host samples at the trainer's weights, from
 * the training kernels (w1/w2/w3 of *grad; the rest zero). */
int velo_mlp_gradient(VeloMlpTrainer* t, const float* features, const uint8_t* labels, uint32_t n,
                      VeloMlpWeights* grad, float* loss);
/* Logits [n][2] of n host feature rows from the inference kernel code. */
int velo_mlp_infer(VeloMlpTrainer* t, const float* features, uint32_t n, float* logits);

/* Device time of each stage of the runs recorded since velo_set_timing, milliseconds:
 * ms[0] decode+cluster+sort, ms[1] fill_candidates (windows, scorer), ms[2] search,
 * ms[3] scan, ms[4] consolidate+fit, ms[5] beamline PV (0 when off), ms[6] global event cut
 * (0 without velo_run_gec), ms[7] (n > 7) number of runs summed. */
int velo_stage_times(VeloCtx* ctx, float* ms, int n);
int velo_set_timing(VeloCtx* ctx, int enabled);

int velo_destroy(VeloCtx* ctx);

/* Blocking copy of device memory of the context's device into host memory (for callers
 * without their own CUDA runtime, e.g. FFI bindings reading the outputs). */
int velo_download(VeloCtx* ctx, void* dst_host, const void* src_device, size_t bytes);
/* Asynchronous variant on `stream` (dst_host should be pinned). */
int velo_download_async(VeloCtx* ctx, void* dst_host, const void* src_device, size_t bytes, void* stream);

/* Appends the beamline primary-vertex finder (cuda/PV/beamlinePV: pv_beamline_extrapolate,
 * pv_beamline_histo, pv_beamline_peak, pv_beamline_multi_fitter of DefaultSequence.h:20-23)
 * to every run, on the Kalman beamline states; its outputs are VeloOutputs.pv_*. Off by
 * default. */
int velo_set_pv(VeloCtx* ctx, int enabled);

/* Search mapping: events with more than `clusters` clusters run the block-per-event search,
 * the others the warp-per-event search (0: all block, >= 16384: all warp). Set by the
 * autotuner (cuda_hlt_b200/autotune.py) from timings per hit-count bucket. */
int velo_set_block_threshold(VeloCtx* ctx, uint32_t clusters);

/* Decode block size: 4 or 8 warps per event (default 8); set by the autotuner
 * (cuda_hlt_b200/autotune.py) from decode timings on a sample batch. */
int velo_set_decode_warps(VeloCtx* ctx, uint32_t warps);

/* Diagnostics of the error path of the bounded device waits: runs one kernel that waits, for
 * `polls` polls (1 .. 2^20), on a barrier that nothing completes, with the wait function of
 * the scorer kernels; the wait runs out, the kernel records the timeout and returns, and the
 * next velo_sync returns VELO_ERR_DEVICE_TIMEOUT. The context stays usable: the next run
 * clears the error. No counterpart in the reference (its kernels report nothing). */
int velo_check_wait_timeout(VeloCtx* ctx, uint32_t polls, void* stream);

/* Kernel launch count of the last run (all kernels of this library). */
int velo_last_launch_count(VeloCtx* ctx, uint32_t* n);

/* CUDA graphs the context holds (VeloConfig.use_graphs). */
int velo_graph_count(VeloCtx* ctx, uint32_t* n);

/* Search without allocation, for callers that cannot allocate device memory (for example a
 * host framework that reserves the device up front and hands out fixed slices). No
 * counterpart in the reference. Runs search_by_triplet on a cluster container produced by
 * velo_run (VeloOutputs hit_xyzp, module_hit_start, module_hit_num, status) and writes the
 * tracks of each event in the reference's Velo::TrackHits terms: track_n[n * 1200] hit
 * counts and track_hits[n * 1200 * 26] event-relative hit indices, event_tracks[n] and
 * status_out[n]. Its scratch is a fixed ~23 MB __device__ array, resident on every device
 * that loads the library: at most 512 events per call (more: VELO_ERR_CAPACITY), all calls
 * share it (calls overlapping on a device race), and the first call on a device looks up
 * its address, so that first call should come before any stream capture. Calls no
 * allocator. */
int velo_search_static(const float* hit_xyzp, const uint32_t* module_hit_start, const uint32_t* module_hit_num,
                       const uint32_t* status_in, uint32_t n_events, uint16_t* track_n, uint16_t* track_hits,
                       uint32_t* event_tracks, uint32_t* status_out, void* stream);

const char* velo_version(void);

#ifdef __cplusplus
}
#endif
#endif /* VELO_B200_H */
