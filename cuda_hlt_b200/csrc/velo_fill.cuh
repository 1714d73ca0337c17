// The learned scorer's kernels between decode and search (pruned mode). The decode kernel
// computes the phi windows of every h1 (fill_candidates, FillCandidates.cu:8-70) and, in the
// pruned mode, appends every seeding candidate (both windows non-empty) that the scoring gate
// admits to a compact list as an 8-byte record (event hit base, h1, module; queue slot 7
// counts them). Then:
//   candidate_features     a thread per listed candidate (all lanes busy, full occupancy)
//                          computes its twelve proxy-triplet features and writes them,
//                          normalised and in bf16, as a row of 128-row tiles laid out for
//                          the tensor core, with the candidate's hit slot alongside;
//   score_candidates       a persistent tcgen05 kernel: each CTA bulk-copies pairs of 4 KB
//                          tiles of those rows into a shared-memory ring, runs the MLP's
//                          three layers on the tensor core for both tiles at once and writes
//                          the verdict per candidate: a pruned seed gets its h0 window
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

// score_candidates: 256 threads in two independent halves of 128 that share the weights in
// shared memory and one tensor-memory allocation. Half h (warps 4h .. 4h + 3; a warp reads
// the TMEM lanes 32 * (warp % 4) onwards) scores its own stream of 128-row tiles with its own
// 64 TMEM columns, load ring, MMA barrier and named barrier (1 + h), so one half runs its
// epilogues while the other waits on the tensor core. All three layers run on the tensor
// core, in the training kernel's layouts: hidden tiles 80 wide with a ones column, so the
// layer-2 and head biases come out of the MMAs, and each epilogue is ReLU, round to bf16 and
// store; the logits are the first two columns of the head's accumulators. Tiles are
// bulk-copied into a two-deep ring per half, one tile ahead; the epilogues take their
// accumulators 16 columns at a time, so three CTAs fit on an SM without spilling.
constexpr uint32_t kScorePair = 2;                                  // halves per CTA
constexpr uint32_t kScoreThreads = kMlpTile * kScorePair;           // 256
constexpr uint32_t kScoreRing = 2;                                  // tiles in a half's ring
constexpr uint32_t kScoreTmemCols = kMlpHidden * kScorePair;        // 128
struct __align__(128) ScoreSmem {
  uint8_t w1[kMlpW1 * 2];                          // W1 [64][16]
  uint8_t w2[kMlpW2 * 2];                          // W2 [64][80], bias in column 64
  uint8_t w3[kMlpW3 * 2];                          // W3 [16][80], rows 2..15 zero
  uint8_t x[kScorePair][kScoreRing][kCandTileBytes];
  uint8_t h[kScorePair][kMlpTile * kMlpK2 * 2];    // H1, then H2: [128][80], 1.0 in column 64
  uint64_t load_bar[kScorePair][kScoreRing];
  uint64_t mbar[kScorePair];
  uint32_t tmem;
};
constexpr uint32_t kScoreSmem = sizeof(ScoreSmem) + 128;

// This thread's half (0/1) and its row in the half's tile.
__device__ __forceinline__ uint32_t score_half() { return threadIdx.x >> 7; }
__device__ __forceinline__ uint32_t score_row() { return threadIdx.x & (kMlpTile - 1); }

// Epilogue of a hidden layer for this thread's row: ReLU of the 64 accumulators, rounded to
// bf16 into columns 0..63 of the row of H (the ones column stays).
__device__ __forceinline__ void score_hidden_epilogue(uint8_t* h, uint32_t taddr_row, uint32_t row)
{
#pragma unroll
  for (uint32_t c = 0; c < 4; ++c) {
    float v[16];
    tmem_ld16(taddr_row + 16 * c, v);
    tmem_ld_wait();
#pragma unroll
    for (uint32_t u = 0; u < 2; ++u) {
      uint4 q;
      q.x = pack_bf16x2(fmaxf(v[8 * u + 0], 0.f), fmaxf(v[8 * u + 1], 0.f));
      q.y = pack_bf16x2(fmaxf(v[8 * u + 2], 0.f), fmaxf(v[8 * u + 3], 0.f));
      q.z = pack_bf16x2(fmaxf(v[8 * u + 4], 0.f), fmaxf(v[8 * u + 5], 0.f));
      q.w = pack_bf16x2(fmaxf(v[8 * u + 6], 0.f), fmaxf(v[8 * u + 7], 0.f));
      *reinterpret_cast<uint4*>(h + canon_off(row, 2 * c + u, kSbo2)) = q;
    }
  }
}

// Named barrier of one half (barrier 1 + half, its 128 threads); the ids are immediates, so
// the kernel holds three barriers (the half is the same for all threads of a half).
__device__ __forceinline__ void half_sync(uint32_t half)
{
  if (half == 0) asm volatile("bar.sync 1, 128;" ::: "memory");
  else asm volatile("bar.sync 2, 128;" ::: "memory");
}

// AND of `v` over the threads of one half, at its named barrier.
__device__ __forceinline__ bool half_and(uint32_t half, bool v)
{
  uint32_t r;
  if (half == 0)
    asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(v ? 1u : 0u)
      : "memory");
  else
    asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(v ? 1u : 0u)
      : "memory");
  return r != 0;
}

// One layer on this half's tile: D = A * B^T into the half's 64 TMEM columns, then wait.
// False (uniformly over the half) on timeout.
__device__ __forceinline__ bool score_layer(ScoreSmem& s, uint32_t half, uint32_t& phase, const uint8_t* a,
                                            uint32_t a_sbo, const uint8_t* b, uint32_t b_sbo, uint32_t k, uint32_t n)
{
  fence_async_smem();  // this half's shared-memory writes, visible to the tensor core
  tc_fence_before();
  half_sync(half);
  tc_fence_after();
  if (score_row() == 0) {
    umma_issue(s.tmem + half * kMlpHidden, a, a_sbo, b, b_sbo, k, n, false);
    umma_commit(&s.mbar[half]);
  }
  const bool ok = mbar_wait_parity(&s.mbar[half], phase);
  phase ^= 1u;
  tc_fence_after();
  return half_and(half, ok);
}

__global__ void __launch_bounds__(kScoreThreads, 3) score_candidates_kernel(ChainPointers P)
{
  extern __shared__ uint8_t s_dyn[];
  ScoreSmem& s = *reinterpret_cast<ScoreSmem*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
  const uint32_t rows = P.queue[7];
  const uint32_t tiles = (rows + kMlpTile - 1) / kMlpTile;
  if (blockIdx.x * kScorePair >= tiles) return;  // uniform: neither half has a tile
  // set-up: tensor memory, barriers, weights (as mlp_infer_setup, for the three-layer layout)
  if (threadIdx.x < 32) tmem_alloc(&s.tmem, kScoreTmemCols);
  if (threadIdx.x == 0)
    for (uint32_t h = 0; h < kScorePair; ++h) {
      mbar_init1(&s.mbar[h]);
      for (uint32_t i = 0; i < kScoreRing; ++i) mbar_init1(&s.load_bar[h][i]);
    }
  load_canon(s.w1, P.mlp.w, kMlpHidden, kMlpK1);
  load_canon(s.w2, P.mlp.w + kMlpW1, kMlpHidden, kMlpK2);
  load_canon(s.w3, P.mlp.w + kMlpW1 + kMlpW2, kMlpOutPad, kMlpK2);
  // columns 64..79 of both H tiles: 1.0 (the bias column), then zeros; never overwritten
  for (uint32_t c = threadIdx.x; c < kScorePair * kMlpTile * 2; c += blockDim.x) {
    const uint32_t t = c / (2 * kMlpTile), row = (c / 2) % kMlpTile, kb = 8 + c % 2;
    const uint4 v = kb == 8 ? make_uint4(pack_bf16x2(1.f, 0.f), 0u, 0u, 0u) : make_uint4(0u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(s.h[t] + canon_off(row, kb, kSbo2)) = v;
  }
  umma_stage_barrier();  // publishes the barrier inits, the weights and the TMEM address

  const uint32_t half = score_half(), row = score_row();
  const uint32_t taddr_row = s.tmem + (((threadIdx.x >> 5) & 3u) * 32u << 16) + half * kMlpHidden;
  // this half's tiles: first, first + workers, ...; its k-th tile goes to ring slot k % ring
  const uint32_t workers = kScorePair * gridDim.x, first = kScorePair * blockIdx.x + half;
  auto issue_load = [&](uint32_t t, uint32_t slot) {
    bulk_load_smem(s.x[half][slot], P.cand_feat + static_cast<size_t>(t) * kCandTileBytes, kCandTileBytes,
                   &s.load_bar[half][slot]);
  };
  uint32_t mma_phase = 0, load_phase = 0;  // load_phase: bit i = parity of slot i
  bool ok = true;
  if (row == 0)
    for (uint32_t k = 0; k + 1 < kScoreRing; ++k) {
      const uint32_t t = first + k * workers;
      if (t < tiles) issue_load(t, k);
    }
  uint32_t k = 0;
  for (uint32_t t = first; t < tiles; t += workers, ++k) {
    const uint32_t slot = k % kScoreRing;
    // refill the slot that tile k - 1 used (its MMAs are complete) with tile k + ring - 1
    const uint32_t ahead = t + (kScoreRing - 1) * workers;
    if (row == 0 && ahead < tiles) issue_load(ahead, (k + kScoreRing - 1) % kScoreRing);
    const uint32_t r = t * kMlpTile + row;
    const uint32_t hit = r < rows ? P.cand_slot[r] : 0u;  // issued early: used after the MMAs
    const bool loaded = mbar_wait_parity(&s.load_bar[half][slot], (load_phase >> slot) & 1u);
    load_phase ^= 1u << slot;
    if (!half_and(half, loaded)) {
      ok = false;
      break;
    }
    if (!score_layer(s, half, mma_phase, s.x[half][slot], kSbo1, s.w1, kSbo1, kMlpK1, kMlpHidden)) {
      ok = false;
      break;
    }
    score_hidden_epilogue(s.h[half], taddr_row, row);  // H1
    if (!score_layer(s, half, mma_phase, s.h[half], kSbo2, s.w2, kSbo2, kMlpK2, kMlpHidden)) {
      ok = false;
      break;
    }
    score_hidden_epilogue(s.h[half], taddr_row, row);  // H2, over H1 (layer 2 has read it)
    if (!score_layer(s, half, mma_phase, s.h[half], kSbo2, s.w3, kSbo2, kMlpK2, kMlpOutPad)) {
      ok = false;
      break;
    }
    float z[16];
    tmem_ld16(taddr_row, z);
    tmem_ld_wait();
    const float z0 = z[0], z1 = z[1];
    if (r < rows) {
      const bool seed = z0 >= P.mlp.seed_logit;
      const bool ext = !P.mlp.use_ext || z1 >= P.mlp.ext_logit;
      if (!seed) P.windows[hit].x = 0xFFFFu;  // no h0 window: the search skips this h1
      P.keep[hit] = static_cast<uint8_t>((seed ? 1u : 0u) | (ext ? 2u : 0u));
    }
  }
  if (!ok && row == 0) {
    atomicOr(P.queue + 6, kErrorMlpTimeout);
    // this half's copies still in flight must land before the CTA exits: wait (bounded) on
    // every slot whose issued copy has not been consumed
    for (uint32_t j = 0; j < kScoreRing; ++j) mbar_wait_parity(&s.load_bar[half][j], (load_phase >> j) & 1u);
  }
  tc_fence_before();
  __syncthreads();  // both halves
  tc_fence_after();
  if (threadIdx.x < 32) tmem_dealloc(s.tmem, kScoreTmemCols);
}

}  // namespace velo
