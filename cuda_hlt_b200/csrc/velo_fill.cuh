// Kernel 2 of the chain: fill_candidates. For every hit h1 of modules 2..49 the phi windows
// of h0 (module m+2) and h2 (module m-2) with the reference's searches and tolerance
// (FillCandidates.cu:8-70, VeloTools.cuh:6-42). The reference computes them in a kernel of
// their own too; here one 128-thread CTA per event (persistent, queue slot 3) writes them
// as event-relative u16 pairs {first, last} (0xFFFF = none), so the search kernel reads a
// window instead of binary-searching inside its serial module loop.
//
// In the pruned mode the same CTA computes the twelve proxy-triplet features of each h1,
// runs the learned scorer on the tensor cores (128 hits per tile) and writes a keep byte
// per hit: bit 0 seed keep, bit 1 extension keep. Events above the scorer's occupancy range
// keep every hit (the plain search) and get VELO_STATUS_MLP_FALLBACK.
#pragma once
#include "velo_mlp.cuh"

namespace velo {

constexpr uint32_t kErrorMlpTimeout = 1u;  // queue[6]: the tensor core did not answer in time

__device__ __forceinline__ uint2 pack_windows(int f0, int l0, int f2, int l2)
{
  return make_uint2((static_cast<uint32_t>(f0) & 0xFFFFu) | (static_cast<uint32_t>(l0) << 16),
                    (static_cast<uint32_t>(f2) & 0xFFFFu) | (static_cast<uint32_t>(l2) << 16));
}

// Dynamic shared memory of the pruned form: one MlpInferSmem, 128-byte aligned.
constexpr uint32_t kFillPrunedSmem = sizeof(MlpInferSmem) + 128;

template<bool kPruned>
__global__ void __launch_bounds__(kMlpTile) fill_candidates_kernel(ChainPointers P)
{
  __shared__ uint32_t s_ms[kModules + 1];
  __shared__ uint32_t s_event;
  extern __shared__ uint8_t s_dyn[];
  MlpInferSmem& sm = *reinterpret_cast<MlpInferSmem*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
  uint32_t phase = 0;
  bool mlp_ok = true;
  if (kPruned) mlp_infer_setup(sm, P.mlp);

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
      const bool fallback = kPruned && (nhits > P.mlp.max_hits || !mlp_ok);
      if (kPruned && fallback && threadIdx.x == 0) P.status[e] = status | kStatusMlpFallback;
      const uint32_t lo = s_ms[2], hi = s_ms[50];
      if (kPruned) {
        // modules 0, 1, 50, 51 hold no h1; their hits stay extension candidates
        uint8_t* K = P.keep + base;
        for (uint32_t h = threadIdx.x; h < lo; h += kMlpTile) K[h] = 2;
        for (uint32_t h = hi + threadIdx.x; h < nhits; h += kMlpTile) K[h] = 2;
      }
      for (uint32_t t0 = lo; t0 < hi; t0 += kMlpTile) {
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
          uint32_t keep = 3;
          if (!fallback) {  // uniform over the CTA
            float f[kMlpFeatures];
            if (cand) seed_features(H, P.hit_size + base, h, m, f0, l0, f2, l2, f);
            mlp_store_features(sm, f, cand);
            float z0 = 0.f, z1 = 0.f;
            if (!mlp_tile_forward(sm, phase, z0, z1)) {
              mlp_ok = false;
              if (threadIdx.x == 0) atomicOr(P.queue + 6, kErrorMlpTimeout);
            }
            if (mlp_ok)
              keep = cand ? ((z0 >= P.mlp.seed_logit ? 1u : 0u) | ((!P.mlp.use_ext || z1 >= P.mlp.ext_logit) ? 2u : 0u))
                          : 2u;
          }
          if (valid) P.keep[base + h] = static_cast<uint8_t>(keep);
        }
      }
    }
    __syncthreads();
  }
  if (kPruned) mlp_infer_teardown(sm);
}

}  // namespace velo
