// The learned scorer's kernels between decode and search (pruned mode). The decode kernel
// computes the phi windows of every h1 (fill_candidates, FillCandidates.cu:8-70) and, in the
// pruned mode, appends every seeding candidate (both windows non-empty) that the scoring gate
// admits to a compact list as an 8-byte record (event hit base, h1, module; queue slot 7
// counts them). Then:
//   candidate_features     a thread per listed candidate (all lanes busy, full occupancy)
//                          computes its twelve proxy-triplet features and writes them,
//                          normalised and in bf16, as a row of 128-row tiles laid out for
//                          the tensor core, with the candidate's hit slot alongside;
//   score_candidates       a persistent tcgen05 kernel: each CTA bulk-copies 4 KB tiles of
//                          those rows into a four-slot shared-memory ring, runs the MLP and
//                          writes the verdict per candidate: a pruned seed gets its h0 window
//                          cleared, so the search never sees it; keep bits per hit (bit 0
//                          seed keep, bit 1 extension keep) are kept for the outputs.
// Events above the scorer's occupancy range append no candidates (the plain search) and get
// VELO_STATUS_MLP_FALLBACK. Seeds with fewer than min_pairs (h0, h2) combinations are not
// appended either: they stay seeds, as scoring them would cost more than their pair loop;
// nor are the seeds of events below min_hits clusters, whose whole search is cheap.
#pragma once
#include "velo_mlp.cuh"

namespace velo {

constexpr uint32_t kErrorMlpTimeout = 1u;  // queue[6]: the tensor core did not answer in time
constexpr uint32_t kFillThreads = 256;
constexpr uint32_t kCandTileBytes = kMlpTile * kMlpK1 * 2;  // 4096

// Features of the listed candidates: a thread per row, grid-stride over queue slot 7's rows.
__global__ void __launch_bounds__(kFillThreads) candidate_features_kernel(ChainPointers P)
{
  __shared__ float s_norm[32];
  if (threadIdx.x < 32) s_norm[threadIdx.x] = P.mlp.norm[threadIdx.x];
  __syncthreads();
  const uint32_t rows = P.queue[7];
  for (uint32_t r = blockIdx.x * kFillThreads + threadIdx.x; r < rows; r += gridDim.x * kFillThreads) {
    const uint2 c = P.cand_rec[r];
    const uint32_t base = c.x, h = c.y & 0xFFFFu, m = c.y >> 16;
    const uint2 w = P.windows[base + h];
    float f[kMlpFeatures];
    seed_features(P.hits.xyzp + base, P.hit_size + base, h, m, static_cast<int>(w.x & 0xFFFFu),
                  static_cast<int>(w.x >> 16), static_cast<int>(w.y & 0xFFFFu), static_cast<int>(w.y >> 16), f);
    store_feature_row(P.cand_feat + static_cast<size_t>(r / kMlpTile) * kCandTileBytes, r % kMlpTile, f, s_norm);
    P.cand_slot[r] = base + h;
  }
}

// Shared memory of score_candidates: the inference tile buffers (whose X tile is slot 0 of
// the copy ring) plus kScoreRing - 1 more X tiles, each slot with its barrier. Tiles are
// prefetched kScoreRing - 1 ahead, so every CTA keeps several 4 KB copies in flight.
constexpr uint32_t kScoreRing = 4;
struct __align__(128) ScoreSmem {
  MlpInferSmem mlp;
  uint8_t x[kScoreRing - 1][kCandTileBytes];
  uint64_t load_bar[kScoreRing];
};
constexpr uint32_t kScoreSmem = sizeof(ScoreSmem) + 128;

__global__ void __launch_bounds__(kMlpTile) score_candidates_kernel(ChainPointers P)
{
  extern __shared__ uint8_t s_dyn[];
  ScoreSmem& s = *reinterpret_cast<ScoreSmem*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
  const uint32_t rows = P.queue[7];
  const uint32_t tiles = (rows + kMlpTile - 1) / kMlpTile;
  if (blockIdx.x >= tiles) return;  // uniform: this CTA has no tile
  if (threadIdx.x == 0)
    for (uint32_t i = 0; i < kScoreRing; ++i) mbar_init1(&s.load_bar[i]);
  mlp_infer_setup(s.mlp, P.mlp);  // includes the barrier that publishes the inits
  uint8_t* xbuf[kScoreRing];
  xbuf[0] = s.mlp.x;
  for (uint32_t i = 1; i < kScoreRing; ++i) xbuf[i] = s.x[i - 1];
  uint32_t mma_phase = 0, load_phase = 0;  // load_phase: bit i = parity of slot i
  bool ok = true;
  // this CTA's tiles are blockIdx.x + k * gridDim.x, k = 0, 1, ...; tile k goes to slot k % ring
  if (threadIdx.x == 0)
    for (uint32_t k = 0; k + 1 < kScoreRing; ++k) {
      const uint32_t t = blockIdx.x + k * gridDim.x;
      if (t < tiles)
        bulk_load_smem(xbuf[k], P.cand_feat + static_cast<size_t>(t) * kCandTileBytes, kCandTileBytes,
                       &s.load_bar[k]);
    }
  uint32_t k = 0;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
    const uint32_t slot = k % kScoreRing;
    // refill the slot used by tile k - 1 (its MMAs are complete) with tile k + ring - 1
    const uint32_t ahead = tile + (kScoreRing - 1) * gridDim.x;
    if (threadIdx.x == 0 && ahead < tiles) {
      const uint32_t as = (k + kScoreRing - 1) % kScoreRing;
      bulk_load_smem(xbuf[as], P.cand_feat + static_cast<size_t>(ahead) * kCandTileBytes, kCandTileBytes,
                     &s.load_bar[as]);
    }
    const uint32_t r = tile * kMlpTile + threadIdx.x;
    const uint32_t hit = r < rows ? P.cand_slot[r] : 0u;  // issued early: used after the MMAs
    const bool loaded = mbar_wait_parity(&s.load_bar[slot], (load_phase >> slot) & 1u);
    load_phase ^= 1u << slot;
    if (!__syncthreads_and(loaded)) {
      ok = false;
      break;
    }
    float z0 = 0.f, z1 = 0.f;
    if (!mlp_tile_forward(s.mlp, mma_phase, z0, z1, xbuf[slot])) {
      ok = false;
      break;
    }
    if (r < rows) {
      const bool seed = z0 >= P.mlp.seed_logit;
      const bool ext = !P.mlp.use_ext || z1 >= P.mlp.ext_logit;
      if (!seed) P.windows[hit].x = 0xFFFFu;  // no h0 window: the search skips this h1
      P.keep[hit] = static_cast<uint8_t>((seed ? 1u : 0u) | (ext ? 2u : 0u));
    }
  }
  if (!ok && threadIdx.x == 0) {
    atomicOr(P.queue + 6, kErrorMlpTimeout);
    // copies still in flight must land before the CTA exits: wait (bounded) on every slot
    // whose issued copy has not been consumed
    for (uint32_t j = 0; j < kScoreRing; ++j) mbar_wait_parity(&s.load_bar[j], (load_phase >> j) & 1u);
  }
  mlp_infer_teardown(s.mlp);
}

}  // namespace velo
