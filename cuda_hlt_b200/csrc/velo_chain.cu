// B200 VELO chain: kernels and the C-ABI context (include/velo_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <array>
#include <map>
#include <vector>

#include "../../include/velo_b200.h"
#include "velo_kernels.cuh"

#include "velo_decode.cuh"

namespace velo {

// ============================================================================
// Kernel 2: search_by_triplet, one warp per event.
// ============================================================================
struct EventHits {
  const float* x;
  const float* y;
  const float* z;
  const float* phi;
};

struct WarpState {
  uint32_t n_tracks, tracklet_ptr, ttf_ptr, weak_ptr;
  uint32_t flags;
};

__device__ __forceinline__ bool test_used(const uint32_t* used, uint32_t h) { return (used[h >> 5] >> (h & 31)) & 1u; }
__device__ __forceinline__ void set_used(uint32_t* used, uint32_t h) { atomicOr(used + (h >> 5), 1u << (h & 31)); }

__device__ __forceinline__ uint32_t ballot_rank(bool pred, uint32_t& total)
{
  const uint32_t b = __ballot_sync(0xFFFFFFFFu, pred);
  total = __popc(b);
  return __popc(b & ((1u << lane_id()) - 1u));
}

// Best (h0, h2) for one h1 over its phi windows (TrackSeeding.cu:110-164); minimal scatter,
// first in (h0, h2) order on exact ties.
__device__ __forceinline__ float seed_best(const EventHits& H, const uint32_t* used, uint32_t h1i, int h0f, int h0l,
                                           int h2f, int h2l, uint16_t& best_h0, uint16_t& best_h2, bool& tie)
{
  float best_fit = 3.402823466e+38f;
  const float h1x = H.x[h1i], h1y = H.y[h1i], h1z = H.z[h1i];
  for (int h0i = h0f; h0i < h0l; ++h0i) {
    if (test_used(used, h0i)) continue;
    const float h0x = H.x[h0i], h0y = H.y[h0i], h0z = H.z[h0i];
    for (int h2i = h2f; h2i < h2l; ++h2i) {
      if (test_used(used, h2i)) continue;
      const float h2x = H.x[h2i], h2y = H.y[h2i], h2z = H.z[h2i];
      const float dmax = kMaxSlope * (h0z - h1z);
      const float scatterDenom2 = 1.f / ((h2z - h1z) * (h2z - h1z));
      const float z2_tz = (h2z - h0z) / (h1z - h0z);
      const float x = h0x + (h1x - h0x) * z2_tz;
      const float y = h0y + (h1y - h0y) * z2_tz;
      const float dx = x - h2x;
      const float dy = y - h2y;
      const float scatterNum = (dx * dx) + (dy * dy);
      const float scatter = scatterNum * scatterDenom2;
      const bool pass = fabsf(h1x - h0x) < dmax && fabsf(h1y - h0y) < dmax && fabsf(dx) < kTolerance &&
                        fabsf(dy) < kTolerance && scatter < kMaxScatterSeeding;
      if (pass && scatter == best_fit) tie = true;
      if (pass && scatter < best_fit) {
        best_fit = scatter;
        best_h0 = static_cast<uint16_t>(h0i);
        best_h2 = static_cast<uint16_t>(h2i);
      }
    }
  }
  return best_fit;
}

// Forwarding fit of one candidate (TrackForwarding.cu:12-35).
__device__ __forceinline__ float forward_fit(float h0x, float h0y, float h2x, float h2y, float predx, float predy,
                                             float scatterDenom2)
{
  const float x_prediction = h0x + predx;
  const float dx = fabsf(x_prediction - h2x);
  const bool tolx_condition = dx < kTolerance;
  const float y_prediction = h0y + predy;
  const float dy = fabsf(y_prediction - h2y);
  const bool toly_condition = dy < kTolerance;
  const float scatterNum = (dx * dx) + (dy * dy);
  const float scatter = scatterNum * scatterDenom2;
  const bool scatter_condition = scatter < kMaxScatterForwarding;
  const bool condition = tolx_condition && toly_condition && scatter_condition;
  return condition * scatter + !condition * 3.402823466e+38f;
}

// Candidate window of a forwarded track in one module (TrackForwarding.cuh:28-59).
__device__ __forceinline__ void forward_window(const float* phis, uint32_t mstart, uint32_t mnum, float mz, float tx,
                                               float ty, float h0x, float h0y, float h0z, bool odd, int& first,
                                               int& last, uint32_t& flags)
{
  const float dz = mz - h0z;
  const float predx = tx * dz;
  const float predy = ty * dz;
  const float x_prediction = h0x + predx;
  const float y_prediction = h0y + predy;
  const float phi = odd ? phi_odd_side(x_prediction, y_prediction) : phi_even_side(x_prediction, y_prediction);
  first = -1;
  last = -1;
  if (mnum == 0) {
    // The reference binary-searches an empty range here and reads the element at the
    // module start, outside the module; this implementation takes no candidates.
    flags |= kStatusEmptyModuleRead;
    return;
  }
  phi_window(phis, mstart, mnum, phi, kForwardPhiTolerance, first, last);
}

// 3-hit straight-line chi2 of weak_tracks_adder (WeakTracksAdder.cu:9-86).
__device__ __forceinline__ float weak_chi2(const EventHits& H, const uint16_t* h)
{
  float s0, sx, sz, sxz, sz2;
  float u0, uy, uz, uyz, uz2;
  s0 = sx = sz = sxz = sz2 = 0.0f;
  u0 = uy = uz = uyz = uz2 = 0.0f;
  for (int k = 0; k < 3; ++k) {
    const uint32_t hitno = h[k];
    const float x = H.x[hitno], y = H.y[hitno], z = H.z[hitno];
    const float wx = kParamW;
    const float wx_t_x = wx * x;
    const float wx_t_z = wx * z;
    s0 += wx;
    sx += wx_t_x;
    sz += wx_t_z;
    sxz += wx_t_x * z;
    sz2 += wx_t_z * z;
    const float wy = kParamW;
    const float wy_t_y = wy * y;
    const float wy_t_z = wy * z;
    u0 += wy;
    uy += wy_t_y;
    uz += wy_t_z;
    uyz += wy_t_y * z;
    uz2 += wy_t_z * z;
  }
  float tx, x0, ty, y0;
  {
    const float dens = 1.0f / (sz2 * s0 - sz * sz);
    tx = (sxz * s0 - sx * sz) * dens;
    x0 = (sx * sz2 - sxz * sz) * dens;
    const float denu = 1.0f / (uz2 * u0 - uz * uz);
    ty = (uyz * u0 - uy * uz) * denu;
    y0 = (uy * uz2 - uyz * uz) * denu;
  }
  float ch = 0.0f;
  int nDoF = -4;
  for (int k = 0; k < 3; ++k) {
    const uint32_t hitno = h[k];
    const float z = H.z[hitno];
    const float x = x0 + tx * z;
    const float y = y0 + ty * z;
    const float dx = x - H.x[hitno];
    const float dy = y - H.y[hitno];
    ch += dx * dx * kParamW + dy * dy * kParamW;
    nDoF += 2;
  }
  return ch / nDoF;
}

template<int WPB>
__global__ void __launch_bounds__(WPB * 32) search_kernel(ChainPointers P)
{
  __shared__ uint32_t s_used[WPB][kEventHitCap / 32];
  __shared__ uint32_t s_mstart[WPB][kModules];
  __shared__ uint32_t s_mnum[WPB][kModules];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  uint32_t* used = s_used[warp];
  uint32_t* mstart = s_mstart[warp];
  uint32_t* mnum = s_mnum[warp];

  for (;;) {
    uint32_t e = 0;
    if (lane == 0) e = atomicAdd(P.queue + 1, 1u);
    e = __shfl_sync(0xFFFFFFFFu, e, 0);
    if (e >= P.n_events) break;
    const uint32_t nhits = P.event_hits[e];
    uint32_t status = P.status[e];
    const uint32_t base = P.event_hit_base[e];
    WarpState st{0, 0, 0, 0, 0};
    uint32_t total_hits_on_tracks = 0;
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (nhits > kEventHitCap) st.flags |= kStatusHitOverflow;
    if (runnable) {
      for (uint32_t i = lane; i < (nhits + 31) / 32; i += 32) used[i] = 0u;
      for (uint32_t m = lane; m < kModules; m += 32) {
        mstart[m] = P.module_start[e * kModules + m] - base;
        mnum[m] = P.module_num[e * kModules + m];
      }
      __syncwarp();
      EventHits H{P.hits.x + base, P.hits.y + base, P.hits.z + base, P.hits.phi + base};
      uint16_t* track_n = P.scratch.track_n + static_cast<size_t>(e) * kMaxTracks;
      uint16_t* track_hits = P.scratch.track_hits + static_cast<size_t>(e) * kMaxTracks * kMaxTrackSize;
      uint16_t* tracklets = P.scratch.tracklets + static_cast<size_t>(e) * kTrackletRing * 3;
      uint32_t* ttf = P.scratch.ttf + static_cast<size_t>(e) * kTtfModulo;
      uint16_t* weak = P.scratch.weak + static_cast<size_t>(e) * kWeakCap * 3;
      uint32_t last_seeded = 0;

      // ---- seeding on modules (first-2, first-3) with h0 in first-0/1, h2 in first-4/5 ----
      auto seeding = [&](uint32_t first) {
        uint32_t n_h1 = 0;
        const uint32_t tracklets_before = st.tracklet_ptr;
        for (int side = 2; side <= 3; ++side) {
          const uint32_t m = first - side;
          const uint32_t start = mstart[m], num = mnum[m];
          const uint32_t m0s = mstart[m + 2], m0n = mnum[m + 2], m2s = mstart[m - 2], m2n = mnum[m - 2];
          for (uint32_t r0 = 0; r0 < num; r0 += 32) {
            const uint32_t r = r0 + lane;
            bool has = false;
            float best = 3.402823466e+38f;
            uint16_t bh0 = 0, bh2 = 0;
            uint32_t h1 = start + r;
            bool tie = false;
            if (r < num && !test_used(used, h1)) {
              // fill_candidates windows (FillCandidates.cu:31-68)
              const float p = H.phi[h1];
              int f0 = -1, l0 = -1, f2 = -1, l2 = -1;
              if (m0n > 0) phi_window(H.phi, m0s, m0n, p, kPhiExtrapolation, f0, l0);
              if (m2n > 0) phi_window(H.phi, m2s, m2n, p, kPhiExtrapolation, f2, l2);
              if (f0 != -1 && f2 != -1) {
                has = true;
                best = seed_best(H, used, h1, f0, l0, f2, l2, bh0, bh2, tie);
              }
            }
            if (tie) st.flags |= kStatusSeedTie;
            uint32_t nh;
            ballot_rank(has, nh);
            n_h1 += nh;
            const bool win = best < 3.402823466e+38f;
            uint32_t nwin;
            const uint32_t rank = ballot_rank(win, nwin);
            if (win) {
              const uint32_t tp = (st.tracklet_ptr + rank) % kTrackletRing;
              tracklets[3 * tp] = bh0;
              tracklets[3 * tp + 1] = static_cast<uint16_t>(h1);
              tracklets[3 * tp + 2] = bh2;
              ttf[(st.ttf_ptr + rank) % kTtfModulo] = 0x80000000u | tp;
            }
            st.tracklet_ptr += nwin;
            st.ttf_ptr += nwin;
          }
        }
        if (n_h1 > kMaxHitsPerModule) st.flags |= kStatusH1Overflow;
        const uint32_t seeded = st.tracklet_ptr - tracklets_before;
        if (seeded + last_seeded > kTrackletRing) st.flags |= kStatusTtfOverflow;
        last_seeded = seeded;
        __syncwarp();
      };

      // ---- forwarding of the tracks to follow into modules first-4 (odd) / first-5 (even) ----
      auto forwarding = [&](uint32_t first, uint32_t prev_ttf, uint32_t diff) {
        const uint32_t mo = first - 4, me = first - 5;
        const uint32_t mos = mstart[mo], mon = mnum[mo], mes = mstart[me], men = mnum[me];
        const float moz = c_module_z[mo], mez = c_module_z[me];
        for (uint32_t i0 = 0; i0 < diff; i0 += 32) {
          const uint32_t i = i0 + lane;
          int action = 0;  // 1 extend, 2 keep with a skipped module, 3 demote to weak
          uint32_t full = 0, trackno = 0, nhit = 0;
          uint16_t t0 = 0, t1 = 0, t2 = 0, best_h2 = 0;
          if (i < diff) {
            full = ttf[(prev_ttf + i) % kTtfModulo];
            const bool flag = (full & 0x80000000u) == 0x80000000u;
            const uint32_t skipped = (full & 0x70000000u) >> 28;
            trackno = full & 0x0FFFFFFFu;
            uint16_t ha, hb;
            if (flag) {
              t0 = tracklets[3 * trackno];
              t1 = tracklets[3 * trackno + 1];
              t2 = tracklets[3 * trackno + 2];
              nhit = 3;
              ha = t1;
              hb = t2;
            } else {
              nhit = track_n[trackno];
              ha = track_hits[trackno * kMaxTrackSize + nhit - 2];
              hb = track_hits[trackno * kMaxTrackSize + nhit - 1];
            }
            const float h0x = H.x[ha], h0y = H.y[ha], h0z = H.z[ha];
            const float h1x = H.x[hb], h1y = H.y[hb], h1z = H.z[hb];
            const float td = 1.0f / (h1z - h0z);
            const float txn = (h1x - h0x);
            const float tyn = (h1y - h0y);
            const float tx = txn * td;
            const float ty = tyn * td;
            float best_fit = 3.402823466e+38f;
            int of, ol, ef, el;
            forward_window(H.phi, mos, mon, moz, tx, ty, h0x, h0y, h0z, true, of, ol, st.flags);
            forward_window(H.phi, mes, men, mez, tx, ty, h0x, h0y, h0z, false, ef, el, st.flags);
            const int n_odd = ol - of, n_even = el - ef;
            for (int j = 0; j < n_odd + n_even; ++j) {
              const int h2i = j < n_odd ? of + j : ef + j - n_odd;
              const float h2x = H.x[h2i], h2y = H.y[h2i], h2z = H.z[h2i];
              const float dz = h2z - h0z;
              const float predx = tx * dz;
              const float predy = ty * dz;
              const float scatterDenom2 = 1.f / ((h2z - h1z) * (h2z - h1z));
              const float fit = forward_fit(h0x, h0y, h2x, h2y, predx, predy, scatterDenom2);
              if (fit < best_fit) {
                best_fit = fit;
                best_h2 = static_cast<uint16_t>(h2i);
              }
            }
            // a track holds at most one hit per module pair: 26 hits (VeloDefinitions.cuh:26)
            if (best_fit != 3.402823466e+38f && nhit < kMaxTrackSize) action = 1;
            else if (skipped < kMaxSkippedModules) action = 2;
            else if (nhit == 3) action = 3;
          }
          // extensions: mark used, allocate new tracks in lane order
          if (action == 1) {
            set_used(used, best_h2);
            if (nhit == 3) {
              set_used(used, t0);
              set_used(used, t1);
              set_used(used, t2);
            }
          }
          uint32_t n_new;
          const uint32_t new_rank = ballot_rank(action == 1 && nhit == 3, n_new);
          bool stored = action == 1;
          if (action == 1 && nhit == 3) {
            const uint32_t slot = st.n_tracks + new_rank;
            if (slot < kMaxTracks) {
              uint16_t* th = track_hits + slot * kMaxTrackSize;
              th[0] = t0;
              th[1] = t1;
              th[2] = t2;
              th[3] = best_h2;
              track_n[slot] = 4;
              trackno = slot;
            } else {
              stored = false;
            }
          } else if (action == 1) {
            track_hits[trackno * kMaxTrackSize + nhit] = best_h2;
            track_n[trackno] = static_cast<uint16_t>(nhit + 1);
          }
          if (st.n_tracks + n_new > kMaxTracks) st.flags |= kStatusTrackOverflow;
          st.n_tracks = min(st.n_tracks + n_new, kMaxTracks);
          // tracks to follow of the next step
          const bool push = stored || action == 2;
          uint32_t n_push;
          const uint32_t push_rank = ballot_rank(push, n_push);
          if (push) {
            const uint32_t value = action == 2 ? ((((full & 0x70000000u) >> 28) + 1) << 28) | (full & 0x8FFFFFFFu)
                                               : trackno;
            ttf[(st.ttf_ptr + push_rank) % kTtfModulo] = value;
          }
          st.ttf_ptr += n_push;
          // demotions to weak
          uint32_t n_weak;
          const uint32_t weak_rank = ballot_rank(action == 3, n_weak);
          if (action == 3 && st.weak_ptr + weak_rank < kWeakCap) {
            uint16_t* w = weak + 3 * (st.weak_ptr + weak_rank);
            w[0] = t0;
            w[1] = t1;
            w[2] = t2;
          }
          st.weak_ptr += n_weak;
        }
        __syncwarp();
      };

      // ---- module loop (ProcessModules.cu:37-162) ----
      uint32_t first = kModules - 1;
      seeding(first);
      uint32_t last_ttf = 0;
      first -= 2;
      while (first >= 4) {
        const uint32_t prev = last_ttf;
        last_ttf = st.ttf_ptr;
        if (last_ttf - prev > kTtfModulo) st.flags |= kStatusTtfOverflow;
        forwarding(first, prev, last_ttf - prev);
        if (st.ttf_ptr - prev > kTtfModulo) st.flags |= kStatusTtfOverflow;
        seeding(first);
        first -= 2;
      }
      {
        // tracklets still waiting become weak (ProcessModules.cu:146-162)
        const uint32_t prev = last_ttf;
        const uint32_t diff = st.ttf_ptr - prev;
        for (uint32_t i0 = 0; i0 < diff; i0 += 32) {
          const uint32_t i = i0 + lane;
          uint32_t full = 0;
          if (i < diff) full = ttf[(prev + i) % kTtfModulo];
          const bool is_weak = i < diff && (full & 0x80000000u);
          uint32_t n_weak;
          const uint32_t rank = ballot_rank(is_weak, n_weak);
          if (is_weak && st.weak_ptr + rank < kWeakCap) {
            const uint32_t tp = full & 0x0FFFFFFFu;
            uint16_t* w = weak + 3 * (st.weak_ptr + rank);
            w[0] = tracklets[3 * tp];
            w[1] = tracklets[3 * tp + 1];
            w[2] = tracklets[3 * tp + 2];
          }
          st.weak_ptr += n_weak;
        }
      }
      if (st.weak_ptr > kMaxWeakTracks) st.flags |= kStatusWeakOverflow;
      __syncwarp();
      // ---- weak_tracks_adder (WeakTracksAdder.cu:88-115) ----
      const uint32_t n_weak = min(st.weak_ptr, kWeakCap);
      for (uint32_t i0 = 0; i0 < n_weak; i0 += 32) {
        const uint32_t i = i0 + lane;
        bool accept = false;
        uint16_t h[3] = {0, 0, 0};
        if (i < n_weak) {
          h[0] = weak[3 * i];
          h[1] = weak[3 * i + 1];
          h[2] = weak[3 * i + 2];
          const bool any_used = test_used(used, h[0]) || test_used(used, h[1]) || test_used(used, h[2]);
          const float chi2 = weak_chi2(H, h);
          accept = !any_used && chi2 < kMaxChi2;
        }
        uint32_t n_acc;
        const uint32_t rank = ballot_rank(accept, n_acc);
        if (accept) {
          const uint32_t slot = st.n_tracks + rank;
          if (slot < kMaxTracks) {
            uint16_t* th = track_hits + slot * kMaxTrackSize;
            th[0] = h[0];
            th[1] = h[1];
            th[2] = h[2];
            track_n[slot] = 3;
          }
        }
        if (st.n_tracks + n_acc > kMaxTracks) st.flags |= kStatusTrackOverflow;
        st.n_tracks = min(st.n_tracks + n_acc, kMaxTracks);
      }
      __syncwarp();
      uint32_t sum = 0;
      for (uint32_t t = lane; t < st.n_tracks; t += 32) sum += track_n[t];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
      total_hits_on_tracks = sum;
    }
    // merge lane flags
    uint32_t f = st.flags;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) f |= __shfl_xor_sync(0xFFFFFFFFu, f, o);
    if (lane == 0) {
      P.event_tracks[e] = runnable ? st.n_tracks : 0;
      P.event_track_hits[e] = runnable ? total_hits_on_tracks : 0;
      P.status[e] = status | f;
    }
    __syncwarp();
  }
}

// ============================================================================
// Kernel 3: exclusive scans over events (single block).
// ============================================================================
__global__ void __launch_bounds__(1024) event_scan_kernel(ChainPointers P)
{
  __shared__ uint32_t s_warp_t[32], s_warp_h[32];
  const uint32_t N = P.n_events;
  const uint32_t per = (N + blockDim.x - 1) / blockDim.x;
  const uint32_t a = min(N, threadIdx.x * per), b = min(N, a + per);
  uint32_t t = 0, h = 0;
  for (uint32_t e = a; e < b; ++e) {
    t += P.event_tracks[e];
    h += P.event_track_hits[e];
  }
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t it = t, ih = h;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t vt = __shfl_up_sync(0xFFFFFFFFu, it, o), vh = __shfl_up_sync(0xFFFFFFFFu, ih, o);
    if (lane >= static_cast<uint32_t>(o)) {
      it += vt;
      ih += vh;
    }
  }
  if (lane == 31) {
    s_warp_t[warp] = it;
    s_warp_h[warp] = ih;
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t wt = lane < (blockDim.x >> 5) ? s_warp_t[lane] : 0, wh = lane < (blockDim.x >> 5) ? s_warp_h[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t vt = __shfl_up_sync(0xFFFFFFFFu, wt, o), vh = __shfl_up_sync(0xFFFFFFFFu, wh, o);
      if (lane >= static_cast<uint32_t>(o)) {
        wt += vt;
        wh += vh;
      }
    }
    s_warp_t[lane] = wt;
    s_warp_h[lane] = wh;
  }
  __syncthreads();
  uint32_t ot = it - t + (warp ? s_warp_t[warp - 1] : 0);
  uint32_t oh = ih - h + (warp ? s_warp_h[warp - 1] : 0);
  for (uint32_t e = a; e < b; ++e) {
    uint32_t nt = P.event_tracks[e];
    uint32_t nh = P.event_track_hits[e];
    if (ot + nt > P.max_tracks_total || oh + nh > P.max_track_hits_total) {
      // consolidated output capacity exhausted: the event keeps no tracks
      P.status[e] |= kStatusTrackOverflow;
      nt = 0;
      nh = 0;
      P.event_tracks[e] = 0;
      P.event_track_hits[e] = 0;
    }
    P.atomics[e] = nt;
    P.atomics[N + e] = ot;
    P.event_hit_offset[e] = oh;
    ot += nt;
    oh += nh;
  }
  // the last thread that owns events (or thread 0 when N == 0) writes the totals
  if (b == N && (a < b || (N == 0 && threadIdx.x == 0))) {
    P.atomics[2 * N] = ot;
    P.event_hit_offset[N] = oh;
    P.track_hit_number[ot] = oh;
  }
}

// ============================================================================
// Kernel 4: consolidation + beamline LSQ state + simplified Kalman (warp per event).
// ============================================================================
struct FitState {
  float x, y, tx, ty, c00, c20, c22, c11, c31, c33, chi2, z;
  bool backward;
};

// means_square_fit (ConsolidateVelo.cu:6-114)
__device__ __forceinline__ FitState beamline_fit(const float* hx, const float* hy, const float* hz, uint32_t n)
{
  FitState state;
  float s0, sx, sz, sxz, sz2;
  float u0, uy, uz, uyz, uz2;
  s0 = sx = sz = sxz = sz2 = 0.0f;
  u0 = uy = uz = uyz = uz2 = 0.0f;
  for (uint32_t h = 0; h < n; ++h) {
    const float x = hx[h];
    const float y = hy[h];
    const float z = hz[h];
    const float wx = kParamW;
    const float wx_t_x = wx * x;
    const float wx_t_z = wx * z;
    s0 += wx;
    sx += wx_t_x;
    sz += wx_t_z;
    sxz += wx_t_x * z;
    sz2 += wx_t_z * z;
    const float wy = kParamW;
    const float wy_t_y = wy * y;
    const float wy_t_z = wy * z;
    u0 += wy;
    uy += wy_t_y;
    uz += wy_t_z;
    uyz += wy_t_y * z;
    uz2 += wy_t_z * z;
  }
  {
    const float dens = 1.0f / (sz2 * s0 - sz * sz);
    state.tx = (sxz * s0 - sx * sz) * dens;
    state.x = (sx * sz2 - sxz * sz) * dens;
    const float denu = 1.0f / (uz2 * u0 - uz * uz);
    state.ty = (uyz * u0 - uy * uz) * denu;
    state.y = (uy * uz2 - uyz * uz) * denu;
    state.z = -(state.x * state.tx + state.y * state.ty) / (state.tx * state.tx + state.ty * state.ty);
    state.backward = state.z > hz[0];
  }
  {
    const float m00 = s0;
    const float m11 = u0;
    const float m20 = sz - state.z * s0;
    const float m31 = uz - state.z * u0;
    const float m22 = sz2 - 2 * state.z * sz + state.z * state.z * s0;
    const float m33 = uz2 - 2 * state.z * uz + state.z * state.z * u0;
    const float den20 = 1.0f / (m22 * m00 - m20 * m20);
    const float den31 = 1.0f / (m33 * m11 - m31 * m31);
    state.c00 = m22 * den20;
    state.c20 = -m20 * den20;
    state.c22 = m00 * den20;
    state.c11 = m33 * den31;
    state.c31 = -m31 * den31;
    state.c33 = m11 * den31;
  }
  {
    float ch = 0.0f;
    int nDoF = -4;
    for (uint32_t h = 0; h < n; ++h) {
      const float z = hz[h];
      const float x = state.x + state.tx * z;
      const float y = state.y + state.ty * z;
      const float dx = x - hx[h];
      const float dy = y - hy[h];
      ch += dx * dx * kParamW + dy * dy * kParamW;
      nDoF += 2;
    }
    state.chi2 = ch / nDoF;
  }
  state.x = state.x + state.tx * state.z;
  state.y = state.y + state.ty * state.z;
  return state;
}

// velo_kalman_filter_step (VeloKalmanFilter.cu:6-41)
__device__ __forceinline__ float kalman_step(const float z, const float zhit, const float xhit, const float whit,
                                             float& x, float& tx, float& covXX, float& covXTx, float& covTxTx)
{
  const float dz = zhit - z;
  const float predx = x + dz * tx;
  const float dz_t_covTxTx = dz * covTxTx;
  const float predcovXTx = covXTx + dz_t_covTxTx;
  const float dx_t_covXTx = dz * covXTx;
  const float predcovXX = covXX + 2 * dx_t_covXTx + dz * dz_t_covTxTx;
  const float predcovTxTx = covTxTx;
  const float R = 1.0f / ((1.0f / whit) + predcovXX);
  const float Kx = predcovXX * R;
  const float KTx = predcovXTx * R;
  const float r = xhit - predx;
  x = predx + Kx * r;
  tx = tx + KTx * r;
  covXX = (1 - Kx) * predcovXX;
  covXTx = (1 - Kx) * predcovXTx;
  covTxTx = predcovTxTx - KTx * predcovXTx;
  return r * r * R;
}

// simplified_fit<true> (VeloKalmanFilter.cuh:27-93)
__device__ __forceinline__ FitState kalman_fit(const float* hx, const float* hy, const float* hz, uint32_t nhits,
                                               const FitState& beam)
{
  const bool backward = beam.z > hz[0];
  const int direction = (backward ? 1 : -1) * 1;
  const float noise2PerLayer = 1e-8 + 7e-6 * (beam.tx * beam.tx + beam.ty * beam.ty);
  int firsthit = 0;
  int lasthit = nhits - 1;
  int dhit = 1;
  if ((hz[lasthit] - hz[firsthit]) * direction < 0) {
    const int temp = firsthit;
    firsthit = lasthit;
    lasthit = temp;
    dhit = -1;
  }
  FitState state;
  state.x = hx[firsthit];
  state.y = hy[firsthit];
  state.z = hz[firsthit];
  state.tx = beam.tx;
  state.ty = beam.ty;
  state.c00 = kParamWInverted;
  state.c11 = kParamWInverted;
  state.c20 = 0.f;
  state.c31 = 0.f;
  state.c22 = 1.f;
  state.c33 = 1.f;
  state.chi2 = 0.0f;
  for (uint32_t i = firsthit + dhit; i != static_cast<uint32_t>(lasthit + dhit); i += dhit) {
    const int hitindex = i;
    const float hit_x = hx[hitindex];
    const float hit_y = hy[hitindex];
    const float hit_z = hz[hitindex];
    state.c22 += noise2PerLayer;
    state.c33 += noise2PerLayer;
    state.chi2 += kalman_step(state.z, hit_z, hit_x, kParamW, state.x, state.tx, state.c00, state.c20, state.c22);
    state.chi2 += kalman_step(state.z, hit_z, hit_y, kParamW, state.y, state.ty, state.c11, state.c31, state.c33);
    state.z = hit_z;
  }
  state.c22 += noise2PerLayer;
  state.c33 += noise2PerLayer;
  state.backward = backward;  // not set by the reference's fit
  return state;
}

__device__ __forceinline__ void store_state(char* base, uint32_t T, uint32_t i, const FitState& s)
{
  float* f = reinterpret_cast<float*>(base);
  f[i] = s.x;
  f[T + i] = s.y;
  f[2 * T + i] = s.tx;
  f[3 * T + i] = s.ty;
  f[4 * T + i] = s.c00;
  f[5 * T + i] = s.c20;
  f[6 * T + i] = s.c22;
  f[7 * T + i] = s.c11;
  f[8 * T + i] = s.c31;
  f[9 * T + i] = s.c33;
  f[10 * T + i] = s.chi2;
  f[11 * T + i] = s.z;
  reinterpret_cast<bool*>(base + sizeof(float) * 12 * T)[i] = s.backward;
}

template<int WPB>
__global__ void __launch_bounds__(WPB * 32) consolidate_fit_kernel(ChainPointers P)
{
  const uint32_t lane = lane_id();
  const uint32_t e = blockIdx.x * WPB + (threadIdx.x >> 5);
  if (e >= P.n_events) return;
  const uint32_t N = P.n_events;
  const uint32_t T = P.atomics[2 * N];
  const uint32_t Htot = P.event_hit_offset[N];
  const uint32_t nt = P.atomics[e];
  const uint32_t t0 = P.atomics[N + e];
  const uint32_t base = P.event_hit_base[e];
  float* ox = reinterpret_cast<float*>(P.track_hits_out);
  float* oy = ox + Htot;
  float* oz = ox + 2 * static_cast<size_t>(Htot);
  uint32_t* oid = reinterpret_cast<uint32_t*>(ox + 3 * static_cast<size_t>(Htot));
  const uint16_t* track_n = P.scratch.track_n + static_cast<size_t>(e) * kMaxTracks;
  const uint16_t* track_hits = P.scratch.track_hits + static_cast<size_t>(e) * kMaxTracks * kMaxTrackSize;
  uint32_t carry = P.event_hit_offset[e];
  for (uint32_t i0 = 0; i0 < nt; i0 += 32) {
    const uint32_t i = i0 + lane;
    const uint32_t n = i < nt ? track_n[i] : 0;
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= static_cast<uint32_t>(o)) incl += v;
    }
    const uint32_t hoff = carry + incl - n;
    carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (i < nt) {
      float hx[kMaxTrackSize], hy[kMaxTrackSize], hz[kMaxTrackSize];
      for (uint32_t k = 0; k < n; ++k) {
        const uint32_t h = base + track_hits[i * kMaxTrackSize + k];
        hx[k] = P.hits.x[h];
        hy[k] = P.hits.y[h];
        hz[k] = P.hits.z[h];
        ox[hoff + k] = hx[k];
        oy[hoff + k] = hy[k];
        oz[hoff + k] = hz[k];
        oid[hoff + k] = P.hits.id[h];
      }
      P.track_hit_number[t0 + i] = hoff;
      const FitState beam = beamline_fit(hx, hy, hz, n);
      store_state(P.states, T, t0 + i, beam);
      const FitState kal = kalman_fit(hx, hy, hz, n, beam);
      store_state(P.kalman_states, T, t0 + i, kal);
    }
  }
}

}  // namespace velo

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
  // input staging (for velo_run_host)
  uint8_t* d_raw = nullptr;
  uint64_t* d_raw_offsets = nullptr;
  // work buffers
  float *d_hx = nullptr, *d_hy = nullptr, *d_hz = nullptr, *d_hphi = nullptr;
  uint32_t* d_hid = nullptr;
  uint64_t hit_capacity = 0;
  uint32_t *d_module_start = nullptr, *d_module_num = nullptr, *d_event_hit_base = nullptr, *d_event_hits = nullptr,
           *d_status = nullptr;
  uint16_t *d_track_n = nullptr, *d_track_hits = nullptr, *d_tracklets = nullptr, *d_weak = nullptr;
  uint32_t* d_ttf = nullptr;
  uint32_t *d_event_tracks = nullptr, *d_event_track_hits = nullptr;
  uint32_t *d_atomics = nullptr, *d_track_hit_number = nullptr, *d_event_hit_offset = nullptr;
  char *d_track_hits_out = nullptr, *d_states = nullptr, *d_kalman = nullptr;
  uint32_t* d_queue = nullptr;
  uint32_t* h_totals = nullptr;  // pinned [4]
  cudaStream_t last_stream = nullptr;
  uint32_t last_n = 0;
  uint32_t launches = 0;
  bool timing = false;
  // Stage timing: one set of 5 events per launch sequence; a graph keeps the set it was
  // captured with, plain launches cycle through the sets.
  std::vector<std::array<cudaEvent_t, 5>> ev_sets;
  std::vector<uint8_t> ev_used;
  uint32_t ev_next = 0;
  int ev_current = -1;
  int decode_warps = 4;
  int search_wpb = 4;
  uint32_t decode_blocks = 0, search_blocks = 0;
  // CUDA graphs per (n_events, raw, offsets)
  struct GraphKey {
    uint32_t n;
    const void* raw;
    const void* offsets;
    cudaStream_t stream;
    bool operator<(const GraphKey& o) const
    {
      if (n != o.n) return n < o.n;
      if (raw != o.raw) return raw < o.raw;
      if (offsets != o.offsets) return offsets < o.offsets;
      return stream < o.stream;
    }
  };
  struct GraphEntry {
    cudaGraphExec_t exec;
    int ev_set;  // event set recorded by the graph, -1 without timing
  };
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
  void* ptrs[] = {c->d_geometry, c->d_sp_patterns, c->d_sp_fx, c->d_sp_fy, c->d_raw, c->d_raw_offsets, c->d_hx,
                  c->d_hy, c->d_hz, c->d_hphi, c->d_hid, c->d_module_start, c->d_module_num, c->d_event_hit_base,
                  c->d_event_hits, c->d_status, c->d_track_n, c->d_track_hits, c->d_tracklets, c->d_weak, c->d_ttf,
                  c->d_event_tracks, c->d_event_track_hits, c->d_atomics, c->d_track_hit_number,
                  c->d_event_hit_offset, c->d_track_hits_out, c->d_states, c->d_kalman, c->d_queue};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->h_totals) cudaFreeHost(c->h_totals);
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
  for (auto& set : c->ev_sets)
    for (auto& e : set)
      if (e) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
}

constexpr uint32_t kPlainEventSets = 8;

int add_event_set(VeloCtx* c)
{
  std::array<cudaEvent_t, 5> set{};
  for (auto& e : set)
    if (cudaEventCreate(&e) != cudaSuccess) return VELO_ERR_CUDA;
  c->ev_sets.push_back(set);
  c->ev_used.push_back(0);
  return static_cast<int>(c->ev_sets.size() - 1);
}

ChainPointers pointers(VeloCtx* c, const void* raw, const uint64_t* offsets, uint32_t n)
{
  ChainPointers P{};
  P.raw = static_cast<const uint8_t*>(raw);
  P.raw_offsets = offsets;
  P.n_events = n;
  P.k = DeviceConstants{reinterpret_cast<const float*>(c->d_geometry), c->d_sp_patterns, c->d_sp_fx, c->d_sp_fy};
  P.hits = HitsSoA{c->d_hx, c->d_hy, c->d_hz, c->d_hphi, c->d_hid};
  P.module_start = c->d_module_start;
  P.module_num = c->d_module_num;
  P.event_hit_base = c->d_event_hit_base;
  P.event_hits = c->d_event_hits;
  P.status = c->d_status;
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
  P.mlp = nullptr;
  return P;
}

// Inside a stream capture an event record must be marked external to become a node that
// records when the graph runs (a plain record only orders the capture).
cudaError_t record(cudaEvent_t e, cudaStream_t s, bool capturing)
{
  return capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s);
}

int launch_chain(VeloCtx* c, const ChainPointers& P, cudaStream_t s, bool capturing = false)
{
  const uint32_t n = P.n_events;
  c->launches = 0;
  VCK(cudaMemsetAsync(c->d_queue, 0, 4 * sizeof(uint32_t), s));
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][0], s, capturing));
  {
    const uint32_t blocks = std::min<uint32_t>(n, c->decode_blocks);
    if (c->decode_warps == 8)
      decode_cluster_sort_kernel<8><<<blocks, 256, 0, s>>>(P);
    else
      decode_cluster_sort_kernel<4><<<blocks, 128, 0, s>>>(P);
    VCK(cudaGetLastError());
    ++c->launches;
  }
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][1], s, capturing));
  {
    const uint32_t warps = n;
    const uint32_t blocks = std::min<uint32_t>((warps + 3) / 4, c->search_blocks);
    search_kernel<4><<<blocks, 128, 0, s>>>(P);
    VCK(cudaGetLastError());
    ++c->launches;
  }
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][2], s, capturing));
  event_scan_kernel<<<1, 1024, 0, s>>>(P);
  VCK(cudaGetLastError());
  ++c->launches;
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][3], s, capturing));
  consolidate_fit_kernel<4><<<(n + 3) / 4, 128, 0, s>>>(P);
  VCK(cudaGetLastError());
  ++c->launches;
  if (c->timing && c->ev_current >= 0) VCK(record(c->ev_sets[c->ev_current][4], s, capturing));
  return 0;
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
  ok &= dalloc(c->d_raw, cfg->max_raw_bytes + 16) == cudaSuccess;
  ok &= dalloc(c->d_raw_offsets, N + 1) == cudaSuccess;
  ok &= dalloc(c->d_hx, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_hy, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_hz, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_hphi, c->hit_capacity) == cudaSuccess;
  ok &= dalloc(c->d_hid, c->hit_capacity) == cudaSuccess;
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
  ok &= dalloc(c->d_queue, 4) == cudaSuccess;
  ok &= cudaMallocHost(reinterpret_cast<void**>(&c->h_totals), 4 * sizeof(uint32_t) + 8) == cudaSuccess;
  if (!ok) return fail(VELO_ERR_CUDA);
  uint8_t pat[256], sizes[256];
  float fx[512], fy[512];
  velo_build_sp_luts(pat, sizes, fx, fy);
  if (cudaMemcpy(c->d_geometry, geometry, kGeometryBytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_sp_patterns, pat, 256, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_sp_fx, fx, sizeof fx, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_sp_fy, fy, sizeof fy, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(VELO_ERR_CUDA);
  int occ = 0;
  if (c->decode_warps == 8)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, decode_cluster_sort_kernel<8>, 256, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, decode_cluster_sort_kernel<4>, 128, 0);
  c->decode_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, search_kernel<4>, 128, 0);
  c->search_blocks = static_cast<uint32_t>(std::max(1, occ) * c->sm_count);
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
  out->hit_x = c->d_hx;
  out->hit_y = c->d_hy;
  out->hit_z = c->d_hz;
  out->hit_phi = c->d_hphi;
  out->hit_id = c->d_hid;
  out->hit_capacity = c->hit_capacity;
  return 0;
}

int velo_run(VeloCtx* c, const void* raw, const uint64_t* raw_offsets, uint32_t n_events, void* stream,
             VeloOutputs* out)
{
  if (!c || (!raw && n_events) || (!raw_offsets && n_events)) return VELO_ERR_INVALID;
  if (n_events > c->cfg.max_events) return VELO_ERR_CAPACITY;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  c->last_stream = s;
  c->last_n = n_events;
  fill_outputs(c, n_events, out);
  if (n_events == 0) {
    VCK(cudaMemsetAsync(c->d_atomics, 0, sizeof(uint32_t), s));
    VCK(cudaMemsetAsync(c->d_track_hit_number, 0, sizeof(uint32_t), s));
    VCK(cudaMemsetAsync(c->d_event_hit_offset, 0, sizeof(uint32_t), s));
    return 0;
  }
  const ChainPointers P = pointers(c, raw, raw_offsets, n_events);
  if (c->cfg.use_graphs) {
    const VeloCtx::GraphKey key{n_events, raw, raw_offsets, s};
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
      cudaStream_t cap = s;
      bool tmp = false;
      if (cap == nullptr) {  // the legacy default stream cannot be captured
        VCK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        tmp = true;
      }
      int set = -1;
      if (c->timing) {
        const int rc = add_event_set(c);
        if (rc < 0) return rc;
        set = rc;
      }
      c->ev_current = set;
      cudaGraph_t g;
      VCK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
      const int rc = launch_chain(c, P, cap, true);
      cudaError_t ce = cudaStreamEndCapture(cap, &g);
      if (tmp) cudaStreamDestroy(cap);
      if (rc != 0) return rc;
      VCK(ce);
      cudaGraphExec_t exec;
      VCK(cudaGraphInstantiate(&exec, g, 0));
      cudaGraphDestroy(g);
      it = c->graphs.emplace(key, VeloCtx::GraphEntry{exec, set}).first;
    }
    VCK(cudaGraphLaunch(it->second.exec, s));
    if (it->second.ev_set >= 0) c->ev_used[it->second.ev_set] = 1;
    c->launches = 4;
    return 0;
  }
  c->ev_current = -1;
  if (c->timing) {
    // plain launches cycle through the first kPlainEventSets sets
    c->ev_current = static_cast<int>(c->ev_next++ % kPlainEventSets);
    c->ev_used[c->ev_current] = 1;
  }
  return launch_chain(c, P, s);
}

int velo_run_host(VeloCtx* c, const void* raw_host, const uint64_t* raw_offsets_host, uint32_t n_events, void* stream,
                  VeloOutputs* out)
{
  if (!c || !raw_host || !raw_offsets_host) return VELO_ERR_INVALID;
  if (n_events > c->cfg.max_events) return VELO_ERR_CAPACITY;
  const uint64_t first = raw_offsets_host[0];
  const uint64_t bytes = raw_offsets_host[n_events] - first;
  if (bytes > c->cfg.max_raw_bytes) return VELO_ERR_CAPACITY;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  VCK(cudaMemcpyAsync(c->d_raw, static_cast<const uint8_t*>(raw_host) + first, bytes, cudaMemcpyHostToDevice, s));
  if (first == 0) {
    VCK(cudaMemcpyAsync(c->d_raw_offsets, raw_offsets_host, 8ull * (n_events + 1), cudaMemcpyHostToDevice, s));
  } else {
    // rebase the offsets on the host only when the caller passed a slice
    std::vector<uint64_t> rebased(raw_offsets_host, raw_offsets_host + n_events + 1);
    for (auto& v : rebased) v -= first;
    VCK(cudaMemcpyAsync(c->d_raw_offsets, rebased.data(), 8ull * (n_events + 1), cudaMemcpyHostToDevice, s));
    VCK(cudaStreamSynchronize(s));
  }
  return velo_run(c, c->d_raw, c->d_raw_offsets, n_events, stream, out);
}

int velo_sync(VeloCtx* c, uint32_t* total_tracks, uint32_t* total_track_hits, uint64_t* total_clusters)
{
  if (!c) return VELO_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  cudaStream_t s = c->last_stream;
  const uint32_t N = c->last_n;
  if (total_tracks || total_track_hits) {
    VCK(cudaMemcpyAsync(c->h_totals, c->d_atomics + 2 * N, 4, cudaMemcpyDeviceToHost, s));
    VCK(cudaMemcpyAsync(c->h_totals + 1, c->d_event_hit_offset + N, 4, cudaMemcpyDeviceToHost, s));
  }
  VCK(cudaStreamSynchronize(s));
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
  if (!c || !weights_host || bytes == 0) return VELO_ERR_INVALID;
  return VELO_ERR_STATE;
}

int velo_set_timing(VeloCtx* c, int enabled)
{
  if (!c) return VELO_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return VELO_ERR_CUDA;
  while (c->ev_sets.size() < kPlainEventSets) {
    const int rc = add_event_set(c);
    if (rc < 0) return rc;
  }
  std::fill(c->ev_used.begin(), c->ev_used.end(), 0);
  c->timing = enabled != 0;
  return 0;
}

// Sums, over every event set recorded since velo_set_timing, the device time of the four
// stages; ms[4] (when n > 4) receives the number of launch sequences summed.
int velo_stage_times(VeloCtx* c, float* ms, int n)
{
  if (!c || !ms || n < 4) return VELO_ERR_INVALID;
  if (c->ev_sets.empty()) return VELO_ERR_STATE;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  int runs = 0;
  for (size_t k = 0; k < c->ev_sets.size(); ++k) {
    if (!c->ev_used[k]) continue;
    for (int i = 0; i < 4; ++i) {
      float t = 0.f;
      VCK(cudaEventElapsedTime(&t, c->ev_sets[k][i], c->ev_sets[k][i + 1]));
      acc[i] += t;
    }
    ++runs;
  }
  for (int i = 0; i < 4; ++i) ms[i] = acc[i];
  if (n > 4) ms[4] = static_cast<float>(runs);
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
