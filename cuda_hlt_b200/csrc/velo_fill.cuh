// Kernel 2 of the chain: fill_candidates. For every hit h1 of modules 2..49 the phi windows
// of h0 (module m+2) and h2 (module m-2) with the reference's searches and tolerance
// (FillCandidates.cu:8-70, VeloTools.cuh:6-42). The reference computes them in a kernel of
// their own too; here one thread per hit (a 256-thread CTA per event, persistent, queue slot
// 3) writes them as event-relative u16 pairs {first, last} (0xFFFF = none), so the search
// kernel reads a window instead of binary-searching inside its serial module loop.
//
// Pruned mode, two kernels:
//   fill_candidates<true>  also computes the twelve proxy-triplet features of every seeding
//                          candidate (both windows non-empty) and appends them, normalised
//                          and in bf16, to a compact list of 128-row tiles laid out for the
//                          tensor core (queue slot 7 counts the rows), with the candidate's
//                          hit slot alongside;
//   score_candidates       a persistent tcgen05 kernel: each CTA bulk-copies 4 KB tiles of
//                          that list into shared memory (double-buffered), runs the MLP and
//                          writes the verdict per candidate: a pruned seed gets its h0 window
//                          cleared, so the search never sees it; keep bits per hit (bit 0
//                          seed keep, bit 1 extension keep) are kept for the outputs.
// Events above the scorer's occupancy range append no candidates (the plain search) and get
// VELO_STATUS_MLP_FALLBACK.
#pragma once
#include "velo_mlp.cuh"

namespace velo {

constexpr uint32_t kErrorMlpTimeout = 1u;  // queue[6]: the tensor core did not answer in time
constexpr uint32_t kFillThreads = 256;
constexpr uint32_t kCandTileBytes = kMlpTile * kMlpK1 * 2;  // 4096

__device__ __forceinline__ uint2 pack_windows(int f0, int l0, int f2, int l2)
{
  return make_uint2((static_cast<uint32_t>(f0) & 0xFFFFu) | (static_cast<uint32_t>(l0) << 16),
                    (static_cast<uint32_t>(f2) & 0xFFFFu) | (static_cast<uint32_t>(l2) << 16));
}

template<bool kPruned>
__global__ void __launch_bounds__(kFillThreads) fill_candidates_kernel(ChainPointers P)
{
  __shared__ uint32_t s_ms[kModules + 1];
  __shared__ uint32_t s_event;
  __shared__ float s_norm[32];
  const uint32_t lane = threadIdx.x & 31u;
  if (kPruned && threadIdx.x < 32) s_norm[threadIdx.x] = P.mlp.norm[threadIdx.x];

  for (;;) {
    if (threadIdx.x == 0) s_event = atomicAdd(P.queue + 3, 1u);
    __syncthreads();
    const uint32_t e = s_event;
    if (e >= P.n_events) break;
    const uint32_t nhits = P.event_hits[e];
    const uint32_t base = P.event_hit_base[e];
    const uint32_t status = P.status[e];
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (threadIdx.x < kModules) s_ms[threadIdx.x] = P.module_start[e * kModules + threadIdx.x] - base;
    if (threadIdx.x == 0) s_ms[kModules] = nhits;
    __syncthreads();
    if (runnable) {
      const float4* H = P.hits.xyzp + base;
      uint2* W = P.windows + base;
      const bool fallback = kPruned && nhits > P.mlp.max_hits;
      if (kPruned && fallback && threadIdx.x == 0) P.status[e] = status | kStatusMlpFallback;
      const uint32_t lo = s_ms[2], hi = s_ms[50];
      if (kPruned) {
        // modules 0, 1, 50, 51 hold no h1: extension candidates only
        uint8_t* K = P.keep + base;
        for (uint32_t h = threadIdx.x; h < lo; h += kFillThreads) K[h] = 2;
        for (uint32_t h = hi + threadIdx.x; h < nhits; h += kFillThreads) K[h] = 2;
      }
      for (uint32_t t0 = lo; t0 < hi; t0 += kFillThreads) {
        const uint32_t h = t0 + threadIdx.x;
        const bool valid = h < hi;
        int f0 = -1, l0 = -1, f2 = -1, l2 = -1;
        uint32_t m = 2;
        if (valid) {
          uint32_t a = 2, b = 50;  // last module with start <= h
          while (b - a > 1) {
            const uint32_t mid = (a + b) >> 1;
            if (s_ms[mid] <= h) a = mid; else b = mid;
          }
          m = a;
          const float p = H[h].w;
          const uint32_t n0 = s_ms[m + 3] - s_ms[m + 2], n2 = s_ms[m - 1] - s_ms[m - 2];
          if (n0 > 0) phi_window4(H, s_ms[m + 2], n0, p, kPhiExtrapolation, f0, l0);
          if (n2 > 0) phi_window4(H, s_ms[m - 2], n2, p, kPhiExtrapolation, f2, l2);
          W[h] = pack_windows(f0, l0, f2, l2);
        }
        if (kPruned) {
          const bool cand = valid && f0 != -1 && f2 != -1;
          if (valid) P.keep[base + h] = cand ? 3u : 2u;  // candidates: verdict from score_candidates
          const bool append = cand && !fallback;
          // one atomic per warp for the rows of its candidates
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, append);
          uint32_t row0 = 0;
          if (lane == 0 && bal) row0 = atomicAdd(P.queue + 7, static_cast<uint32_t>(__popc(bal)));
          row0 = __shfl_sync(0xFFFFFFFFu, row0, 0);
          if (append) {
            const uint32_t r = row0 + __popc(bal & ((1u << lane) - 1u));
            float f[kMlpFeatures];
            seed_features(H, P.hit_size + base, h, m, f0, l0, f2, l2, f);
            store_feature_row(P.cand_feat + static_cast<size_t>(r / kMlpTile) * kCandTileBytes, r % kMlpTile, f,
                              s_norm);
            P.cand_slot[r] = base + h;
          }
        }
      }
    }
    __syncthreads();
  }
}


// score_candidates processes kScoreTiles tiles per iteration with the same 128 threads
// (thread t owns row t of each): the MMAs of all of them go out under one barrier and one
// commit, so the fixed cost of a layer (barriers, commit round trip, tensor-memory loads)
// is shared. Accumulators of tile i sit in tensor-memory columns [64 i, 64 i + 64).
constexpr uint32_t kScoreTiles = 2;
constexpr uint32_t kScoreTmemCols = 64 * kScoreTiles;

struct __align__(128) ScoreSmem {
  uint8_t w1[kMlpW1 * 2];
  uint8_t w2[kMlpW2 * 2];
  uint8_t w3[kMlpW3 * 2];
  uint8_t h[kScoreTiles][kMlpTile * kMlpK2 * 2];
  uint8_t x[2][kScoreTiles][kCandTileBytes];  // double-buffered X tiles
  uint64_t mma_bar;
  uint64_t load_bar[2];
  uint32_t tmem;
};
constexpr uint32_t kScoreSmem = sizeof(ScoreSmem) + 128;

// Issues the copies of the X tiles of group g (tiles g*kScoreTiles ...) into buffer `buf`.
__device__ __forceinline__ void score_load_group(ScoreSmem& s, const ChainPointers& P, uint32_t g, uint32_t tiles,
                                                 uint32_t buf)
{
  const uint32_t t0 = g * kScoreTiles;
  const uint32_t n = min(kScoreTiles, tiles - t0);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&s.load_bar[buf])),
               "r"(n * kCandTileBytes)
               : "memory");
  for (uint32_t i = 0; i < n; ++i)
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(s.x[buf][i])),
                 "l"(P.cand_feat + static_cast<size_t>(t0 + i) * kCandTileBytes), "r"(kCandTileBytes),
                 "r"(smem_u32(&s.load_bar[buf]))
                 : "memory");
}

// One layer for all tiles of the group: D_i = A_i * B^T into columns 64 i, then wait.
__device__ __forceinline__ bool score_layer(ScoreSmem& s, uint32_t& phase, const uint8_t* const* a, uint32_t a_sbo,
                                            const uint8_t* b, uint32_t b_sbo, uint32_t k, uint32_t n)
{
  umma_stage_barrier();
  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < kScoreTiles; ++i) umma_issue(s.tmem + 64 * i, a[i], a_sbo, b, b_sbo, k, n, false);
    umma_commit(&s.mma_bar);
  }
  return umma_wait(&s.mma_bar, phase);
}

__global__ void __launch_bounds__(kMlpTile) score_candidates_kernel(ChainPointers P)
{
  extern __shared__ uint8_t s_dyn[];
  ScoreSmem& s = *reinterpret_cast<ScoreSmem*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
  const uint32_t rows = P.queue[7];
  const uint32_t tiles = (rows + kMlpTile - 1) / kMlpTile;
  const uint32_t groups = (tiles + kScoreTiles - 1) / kScoreTiles;
  if (blockIdx.x >= groups) return;  // uniform: this CTA has no work
  if (threadIdx.x < 32) tmem_alloc(&s.tmem, kScoreTmemCols);
  if (threadIdx.x == 0) {
    mbar_init1(&s.mma_bar);
    mbar_init1(&s.load_bar[0]);
    mbar_init1(&s.load_bar[1]);
  }
  load_canon(s.w1, P.mlp.w, kMlpHidden, kMlpK1);
  load_canon(s.w2, P.mlp.w + kMlpW1, kMlpHidden, kMlpK2);
  load_canon(s.w3, P.mlp.w + kMlpW1 + kMlpW2, kMlpOutPad, kMlpK2);
  umma_stage_barrier();
  if (threadIdx.x == 0) score_load_group(s, P, blockIdx.x, tiles, 0);
  const uint32_t lane_addr = s.tmem + ((threadIdx.x & ~31u) << 16);
  const uint8_t* const hp[kScoreTiles] = {s.h[0], s.h[1]};
  uint32_t mma_phase = 0, load_phase[2] = {0u, 0u}, buf = 0;
  bool ok = true;
  for (uint32_t g = blockIdx.x; g < groups; g += gridDim.x, buf ^= 1u) {
    // prefetch the next group into the other buffer (its MMAs are complete)
    if (threadIdx.x == 0 && g + gridDim.x < groups) score_load_group(s, P, g + gridDim.x, tiles, buf ^ 1u);
    const bool loaded = mbar_wait_parity(&s.load_bar[buf], load_phase[buf]);
    load_phase[buf] ^= 1u;
    if (!__syncthreads_and(loaded)) {
      ok = false;
      break;
    }
    const uint8_t* const xp[kScoreTiles] = {s.x[buf][0], s.x[buf][1]};
    if (!(ok = score_layer(s, mma_phase, xp, kSbo1, s.w1, kSbo1, kMlpK1, kMlpHidden))) break;
    for (uint32_t i = 0; i < kScoreTiles; ++i) mlp_hidden_epilogue(s.h[i], lane_addr + 64 * i);
    if (!(ok = score_layer(s, mma_phase, hp, kSbo2, s.w2, kSbo2, kMlpK2, kMlpHidden))) break;
    for (uint32_t i = 0; i < kScoreTiles; ++i) mlp_hidden_epilogue(s.h[i], lane_addr + 64 * i);
    if (!(ok = score_layer(s, mma_phase, hp, kSbo2, s.w3, kSbo2, kMlpK2, kMlpOutPad))) break;
    for (uint32_t i = 0; i < kScoreTiles; ++i) {
      float v[16];
      tmem_ld16(lane_addr + 64 * i, v);
      tmem_ld_wait();
      const uint32_t r = (g * kScoreTiles + i) * kMlpTile + threadIdx.x;
      if (r < rows) {
        const uint32_t slot = P.cand_slot[r];
        const bool seed = v[0] >= P.mlp.seed_logit;
        const bool ext = !P.mlp.use_ext || v[1] >= P.mlp.ext_logit;
        if (!seed) P.windows[slot].x = 0xFFFFu;  // no h0 window: the search skips this h1
        P.keep[slot] = static_cast<uint8_t>((seed ? 1u : 0u) | (ext ? 2u : 0u));
      }
    }
  }
  if (!ok && threadIdx.x == 0) {
    atomicOr(P.queue + 6, kErrorMlpTimeout);
    // a bulk copy still in flight must land before the CTA exits
    mbar_wait_parity(&s.load_bar[buf ^ 1u], load_phase[buf ^ 1u]);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) tmem_dealloc(s.tmem, kScoreTmemCols);
}

}  // namespace velo
