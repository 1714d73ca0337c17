// Kernel 3 of the chain: search_by_triplet, one warp per event (persistent, queue), events
// handed out largest first (order_events_kernel, velo_order.cuh).
//
// The module loop, forwarding and weak-track rules are those of the reference
// (ProcessModules.cu:8-163, TrackForwarding.cu:41-181, TrackSeeding.cu:7-200,
// WeakTracksAdder.cu:88-115). What changes is the mapping onto the warp:
//   * seeding: the phi windows of every h1 come precomputed from fill_candidates (in the
//     pruned mode the scorer has cleared the windows of pruned seeds, and forwarding skips
//     candidates without the extension-keep bit when that pruning is on);
//     the h1 candidates of a step are compacted into a shared list, their
//     (h1, h0) pairs are flattened over the lanes, and each h1 keeps its best triplet in a
//     shared 64-bit key (scatter bits, h0 offset, h2 offset) reduced with atomicMin. The
//     winner is the minimal scatter, first in (h0, h2) order; an atomicMax twin with the
//     scatter bits inverted finds the last candidate of equal scatter, so exact ties (which
//     the reference resolves by thread scheduling) are flagged;
//   * hit_used is a bitmask in shared memory; appends to the ring buffers go in lane order
//     through ballots, so the result does not depend on scheduling.
#pragma once
#include "velo_kernels.cuh"

namespace velo {

// h1 candidates per seeding pass (multiple of 32). The per-warp shared state is small so
// that L1, which shares the SM's 256 KB with shared memory, keeps more of the events' hit
// records: 64 measured faster than 128 (4.46 vs 4.60 ms per 16,384 events).
constexpr uint32_t kSeedChunk = 64;

__device__ __forceinline__ bool test_used(const uint32_t* used, uint32_t h) { return (used[h >> 5] >> (h & 31)) & 1u; }
__device__ __forceinline__ void set_used(uint32_t* used, uint32_t h) { atomicOr(used + (h >> 5), 1u << (h & 31)); }

__device__ __forceinline__ uint32_t ballot_rank(bool pred, uint32_t& total)
{
  const uint32_t b = __ballot_sync(0xFFFFFFFFu, pred);
  total = __popc(b);
  return __popc(b & ((1u << lane_id()) - 1u));
}

// Scatter of the triplet (h0, h1, h2) and whether it passes the seeding cuts
// (TrackSeeding.cu:137-152).
__device__ __forceinline__ bool seed_scatter(const float4 h0, const float4 h1, const float4 h2, float& scatter)
{
  const float dmax = kMaxSlope * (h0.z - h1.z);
  const float scatterDenom2 = 1.f / ((h2.z - h1.z) * (h2.z - h1.z));
  const float z2_tz = (h2.z - h0.z) / (h1.z - h0.z);
  const float x = h0.x + (h1.x - h0.x) * z2_tz;
  const float y = h0.y + (h1.y - h0.y) * z2_tz;
  const float dx = x - h2.x;
  const float dy = y - h2.y;
  const float scatterNum = (dx * dx) + (dy * dy);
  scatter = scatterNum * scatterDenom2;
  return fabsf(h1.x - h0.x) < dmax && fabsf(h1.y - h0.y) < dmax && fabsf(dx) < kTolerance && fabsf(dy) < kTolerance &&
         scatter < kMaxScatterSeeding;
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

// phi window of a forwarded track in one module (TrackForwarding.cuh:28-59).
__device__ __forceinline__ void forward_window(const float4* H, uint32_t mstart, uint32_t mnum, float mz, float tx,
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
  phi_window4(H, mstart, mnum, phi, kForwardPhiTolerance, first, last);
}

// 3-hit straight-line chi2 of weak_tracks_adder (WeakTracksAdder.cu:9-86).
__device__ __forceinline__ float weak_chi2(const float4* H, const uint16_t* h)
{
  float s0, sx, sz, sxz, sz2;
  float u0, uy, uz, uyz, uz2;
  s0 = sx = sz = sxz = sz2 = 0.0f;
  u0 = uy = uz = uyz = uz2 = 0.0f;
  float4 p[3];
  for (int k = 0; k < 3; ++k) {
    p[k] = H[h[k]];
    const float x = p[k].x, y = p[k].y, z = p[k].z;
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
    const float z = p[k].z;
    const float x = x0 + tx * z;
    const float y = y0 + ty * z;
    const float dx = x - p[k].x;
    const float dy = y - p[k].y;
    ch += dx * dx * kParamW + dy * dy * kParamW;
    nDoF += 2;
  }
  return ch / nDoF;
}

struct SeedSlots {
  uint16_t h1[kSeedChunk];
  uint16_t f0[kSeedChunk];
  uint16_t f2[kSeedChunk];
  uint16_t l2[kSeedChunk];
  uint16_t np[kSeedChunk];
  uint32_t pair_start[kSeedChunk];
  unsigned long long best[kSeedChunk];
  unsigned long long last[kSeedChunk];
};

// Forwarding reads the phi of its two target modules from shared memory; the staging
// area reuses the seeding slots (the two phases never overlap).
constexpr uint32_t kFwdStage = sizeof(SeedSlots) / (2 * sizeof(float));

struct SearchWarpShared {
  uint32_t used[kEventHitCap / 32];
  uint32_t mstart[kModules];
  uint32_t mnum[kModules];
  union {
    SeedSlots seed;
    float fphi[2][kFwdStage];
  } u;
};

// phi window of a forwarded track in one module (TrackForwarding.cuh:28-59), with the
// module's phi staged in shared memory (`sphi`, null when the module did not fit): the
// same probes on the same values as phi_window4 over the cluster records.
__device__ __forceinline__ void forward_window_staged(const float4* H, const float* sphi, uint32_t mstart,
                                                      uint32_t mnum, float mz, float tx, float ty, float h0x,
                                                      float h0y, float h0z, bool odd, int& first, int& last,
                                                      uint32_t& flags)
{
  if (!sphi) {
    forward_window(H, mstart, mnum, mz, tx, ty, h0x, h0y, h0z, odd, first, last, flags);
    return;
  }
  const float dz = mz - h0z;
  const float predx = tx * dz;
  const float predy = ty * dz;
  const float x_prediction = h0x + predx;
  const float y_prediction = h0y + predy;
  const float phi = odd ? phi_odd_side(x_prediction, y_prediction) : phi_even_side(x_prediction, y_prediction);
  first = -1;
  last = -1;
  if (mnum == 0) {
    flags |= kStatusEmptyModuleRead;
    return;
  }
  phi_window(sphi, 0, mnum, phi, kForwardPhiTolerance, first, last);
  if (first != -1) {
    first += static_cast<int>(mstart);
    last += static_cast<int>(mstart);
  }
}

// Per-event scratch of the warp search: the reference's Velo::TrackHits slots and the rings
// of tracklets, of tracks to follow and of weak tracklets (SearchByTripletVisitor.cu:11-18).
struct EventScratch {
  uint16_t* track_n;     // [kMaxTracks]
  uint16_t* track_hits;  // [kMaxTracks * kMaxTrackSize]
  uint16_t* tracklets;   // [kTrackletRing * 3]
  uint32_t* ttf;         // [kTtfModulo]
  uint16_t* weak;        // [kWeakCap * 3]
};

// Seeding windows read from the fill_candidates output: {h0 first | last << 16, h2 first |
// last << 16} per hit, event-relative (0xFFFF: no window). Each is read once per event, so
// it is loaded evict-first: the cache keeps the cluster records, which the search rereads.
struct StoredWindows {
  const uint2* w;
  __device__ __forceinline__ uint2 operator()(uint32_t h1, uint32_t) const { return __ldcs(w + h1); }
};

// Seeding windows computed where they are needed, with the searches of fill_candidates
// (FillCandidates.cu:31-68): h0 window in module m + 2, h2 window in module m - 2.
struct ComputedWindows {
  const float4* H;
  const uint32_t* mstart;
  const uint32_t* mnum;
  __device__ __forceinline__ uint2 operator()(uint32_t h1, uint32_t m) const
  {
    const float p = H[h1].w;
    int f0 = -1, l0 = -1, f2 = -1, l2 = -1;
    if (mnum[m + 2] > 0) phi_window4(H, mstart[m + 2], mnum[m + 2], p, kPhiExtrapolation, f0, l0);
    if (mnum[m - 2] > 0) phi_window4(H, mstart[m - 2], mnum[m - 2], p, kPhiExtrapolation, f2, l2);
    return make_uint2((static_cast<uint32_t>(f0) & 0xFFFFu) | (static_cast<uint32_t>(l0) << 16),
                      (static_cast<uint32_t>(f2) & 0xFFFFu) | (static_cast<uint32_t>(l2) << 16));
  }
};

// Loads the module table of one event into the warp's shared state and clears its used-hit
// bitmask. module_start holds absolute hit indices; base is the event's first hit.
__device__ __forceinline__ void search_event_setup(SearchWarpShared& sw, const uint32_t* module_start,
                                                   const uint32_t* module_num, uint32_t base, uint32_t nhits)
{
  const uint32_t lane = lane_id();
  for (uint32_t i = lane; i < (nhits + 31) / 32; i += 32) sw.used[i] = 0u;
  for (uint32_t m = lane; m < kModules; m += 32) {
    sw.mstart[m] = module_start[m] - base;
    sw.mnum[m] = module_num[m];
  }
  __syncwarp();
}

// search_by_triplet and weak_tracks_adder of one event by one warp (ProcessModules.cu:37-162,
// TrackSeeding.cu:7-200, TrackForwarding.cu:41-181, WeakTracksAdder.cu:88-115), after
// search_event_setup. H: the event's phi-sorted cluster records; windows(h1, module): the
// seeding windows of h1; KE: extension-keep bits per hit (bit 1), or null. Returns the
// number of tracks written to sc.track_n / sc.track_hits; status bits go to `flags` (per
// lane: OR-reduce them over the warp).
template<class Windows>
__device__ __forceinline__ uint32_t search_event_warp(SearchWarpShared& sw, const float4* H, const Windows& windows,
                                                      const uint8_t* KE, const EventScratch& sc, uint32_t& flags)
{
  const uint32_t lane = lane_id();
  uint32_t* used = sw.used;
  uint32_t* mstart = sw.mstart;
  uint32_t* mnum = sw.mnum;
  SeedSlots& sl = sw.u.seed;
  uint16_t* track_n = sc.track_n;
  uint16_t* track_hits = sc.track_hits;
  uint16_t* tracklets = sc.tracklets;
  uint32_t* ttf = sc.ttf;
  uint16_t* weak = sc.weak;
  uint32_t n_tracks = 0, tracklet_ptr = 0, ttf_ptr = 0, weak_ptr = 0;
  uint32_t last_seeded = 0;

  // ---- seeding: h1 in modules first-2 / first-3, h0 in h1+2, h2 in h1-2 ----
  auto seeding = [&](uint32_t first) {
    uint32_t n_h1 = 0;
    const uint32_t tracklets_before = tracklet_ptr;
    // Candidates of both modules (first - 2, then first - 3) are queued in the slots and
    // processed kSeedChunk at a time: a module's last few hits share a pass with the next
    // module's first ones. The two modules' seeds are independent (seeding marks no hit
    // used), and winners are appended in queue order, the order of a pass per module.
    uint32_t nc = 0;  // candidates queued
    // (b)-(d) on the queued candidates
    auto flush = [&]() {
      __syncwarp();
      // (b) exclusive scan of the h0 counts
      uint32_t total_pairs = 0;
      for (uint32_t k0 = 0; k0 < nc; k0 += 32) {
        const uint32_t k = k0 + lane;
        const uint32_t v = k < nc ? sl.np[k] : 0;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
          if (lane >= static_cast<uint32_t>(o)) incl += t;
        }
        if (k < nc) sl.pair_start[k] = total_pairs + incl - v;
        total_pairs += __shfl_sync(0xFFFFFFFFu, incl, 31);
      }
      __syncwarp();
      // (c) (h1, h0) pairs over the lanes, each scanning its h2 window. Every candidate
      // has at least one pair (a non-empty window ends past its first hit), so the
      // candidates starting inside a group of 32 pairs are k_lo + 1 .. k_lo + 32 and
      // each lane's candidate is k_lo plus the starts at or before it (one shared
      // load, an OR across the warp and a popcount instead of a binary search).
      uint32_t k_lo = 0;  // candidate of pair p0
      for (uint32_t p0 = 0; p0 < total_pairs; p0 += 32) {
        const uint32_t p = p0 + lane;
        uint32_t head = 0;
        if (k_lo + 1 + lane < nc) {
          const uint32_t s = sl.pair_start[k_lo + 1 + lane];
          if (s >= p0 && s <= p0 + 31) head = 1u << (s - p0);
        }
        const uint32_t heads = __reduce_or_sync(0xFFFFFFFFu, head);
        const uint32_t k = k_lo + __popc(heads & (0xFFFFFFFFu >> (31 - lane)));
        k_lo = __shfl_sync(0xFFFFFFFFu, k, 31);
        if (p < total_pairs) {
          const uint32_t h0rel = p - sl.pair_start[k];
          const uint32_t h0i = sl.f0[k] + h0rel;
          if (!test_used(used, h0i)) {
            const float4 h0 = H[h0i];
            const float4 h1 = H[sl.h1[k]];
            const uint32_t f2 = sl.f2[k], l2 = sl.l2[k];
            unsigned long long best = ~0ull, last = 0ull;
            for (uint32_t h2i = f2; h2i < l2; ++h2i) {
              if (test_used(used, h2i)) continue;
              float scatter;
              if (seed_scatter(h0, h1, H[h2i], scatter)) {
                const uint32_t idx = (h0rel << 16) | (h2i - f2);
                const uint32_t sb = __float_as_uint(scatter);
                const unsigned long long key = (static_cast<unsigned long long>(sb) << 32) | idx;
                const unsigned long long key_last = (static_cast<unsigned long long>(~sb) << 32) | idx;
                best = min(best, key);
                last = max(last, key_last);
              }
            }
            if (best != ~0ull) {
              atomicMin(&sl.best[k], best);
              atomicMax(&sl.last[k], last);
            }
          }
        }
      }
      __syncwarp();
      // (d) winners, appended in candidate order (TrackSeeding.cu:185-195)
      for (uint32_t k0 = 0; k0 < nc; k0 += 32) {
        const uint32_t k = k0 + lane;
        const bool win = k < nc && sl.best[k] != ~0ull;
        uint32_t nwin;
        const uint32_t rank = ballot_rank(win, nwin);
        if (win) {
          const unsigned long long key = sl.best[k];
          if ((key & 0xFFFFFFFFull) != (sl.last[k] & 0xFFFFFFFFull)) flags |= kStatusSeedTie;
          const uint32_t tp = (tracklet_ptr + rank) % kTrackletRing;
          tracklets[3 * tp] = static_cast<uint16_t>(sl.f0[k] + ((key >> 16) & 0xFFFFu));
          tracklets[3 * tp + 1] = sl.h1[k];
          tracklets[3 * tp + 2] = static_cast<uint16_t>(sl.f2[k] + (key & 0xFFFFu));
          ttf[(ttf_ptr + rank) % kTtfModulo] = 0x80000000u | tp;
        }
        tracklet_ptr += nwin;
        ttf_ptr += nwin;
      }
      __syncwarp();
      nc = 0;
    };
    int side = 2;
    uint32_t r0 = 0;
    for (;;) {
      while (side <= 3 && r0 >= mnum[first - side]) {
        ++side;
        r0 = 0;
      }
      const bool have = side <= 3;
      // (a) unused h1 with both phi windows (FillCandidates.cu:31-68, TrackSeeding.cu:24-49)
      // among the next (up to) kSeedChunk hits; the windows of their 32-hit groups are
      // loaded together so that their latencies overlap
      uint32_t start = 0, r_end = 0, n_new = 0;
      uint2 wv[kSeedChunk / 32];
      bool hv[kSeedChunk / 32];
#pragma unroll
      for (uint32_t j = 0; j < kSeedChunk / 32; ++j) {
        wv[j] = make_uint2(0xFFFFu, 0xFFFFu);
        hv[j] = false;
      }
      if (have) {
        const uint32_t m = first - side;
        start = mstart[m];
        r_end = min(mnum[m], r0 + kSeedChunk);
#pragma unroll
        for (uint32_t j = 0; j < kSeedChunk / 32; ++j) {
          const uint32_t r = r0 + 32 * j + lane;
          if (r < r_end && !test_used(used, start + r)) wv[j] = windows(start + r, m);
        }
#pragma unroll
        for (uint32_t j = 0; j < kSeedChunk / 32; ++j) {
          const uint32_t r = r0 + 32 * j + lane;
          hv[j] = r < r_end && (wv[j].x & 0xFFFFu) != 0xFFFFu && (wv[j].y & 0xFFFFu) != 0xFFFFu;
          n_new += __popc(__ballot_sync(0xFFFFFFFFu, hv[j]));
        }
      }
      if (nc > 0 && (!have || nc + n_new > kSeedChunk)) flush();
      if (!have) break;
#pragma unroll
      for (uint32_t j = 0; j < kSeedChunk / 32; ++j) {
        const uint32_t h1 = start + r0 + 32 * j + lane;
        const uint2 w = wv[j];
        uint32_t cnt;
        const uint32_t rank = ballot_rank(hv[j], cnt);
        if (hv[j]) {
          const uint32_t k = nc + rank;
          const uint32_t f0 = w.x & 0xFFFFu, l0 = w.x >> 16, f2 = w.y & 0xFFFFu, l2 = w.y >> 16;
          sl.h1[k] = static_cast<uint16_t>(h1);
          sl.f0[k] = static_cast<uint16_t>(f0);
          sl.np[k] = static_cast<uint16_t>(l0 - f0);
          sl.f2[k] = static_cast<uint16_t>(f2);
          sl.l2[k] = static_cast<uint16_t>(l2);
          sl.best[k] = ~0ull;
          sl.last[k] = 0ull;
        }
        nc += cnt;
      }
      n_h1 += n_new;
      r0 += kSeedChunk;
    }
    if (n_h1 > kMaxHitsPerModule) flags |= kStatusH1Overflow;
    const uint32_t seeded = tracklet_ptr - tracklets_before;
    if (seeded + last_seeded > kTrackletRing) flags |= kStatusTtfOverflow;
    last_seeded = seeded;
  };

  // ---- forwarding of the tracks to follow into modules first-4 (odd) / first-5 (even) ----
  auto forwarding = [&](uint32_t first, uint32_t prev_ttf, uint32_t diff) {
    const uint32_t mo = first - 4, me = first - 5;
    const uint32_t mos = mstart[mo], mon = mnum[mo], mes = mstart[me], men = mnum[me];
    const float moz = c_module_z[mo], mez = c_module_z[me];
    // stage the phi of both target modules (their binary searches then stay in shared
    // memory); a module above the staging size is searched in global memory
    const float* sphi_o = mon <= kFwdStage ? sw.u.fphi[0] : nullptr;
    const float* sphi_e = men <= kFwdStage ? sw.u.fphi[1] : nullptr;
    if (diff > 0) {
      if (sphi_o)
        for (uint32_t i = lane; i < mon; i += 32) sw.u.fphi[0][i] = H[mos + i].w;
      if (sphi_e)
        for (uint32_t i = lane; i < men; i += 32) sw.u.fphi[1][i] = H[mes + i].w;
    }
    __syncwarp();
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
        const float4 h0 = H[ha];
        const float4 h1 = H[hb];
        const float td = 1.0f / (h1.z - h0.z);
        const float txn = (h1.x - h0.x);
        const float tyn = (h1.y - h0.y);
        const float tx = txn * td;
        const float ty = tyn * td;
        float best_fit = 3.402823466e+38f;
        int of, ol, ef, el;
        forward_window_staged(H, sphi_o, mos, mon, moz, tx, ty, h0.x, h0.y, h0.z, true, of, ol, flags);
        forward_window_staged(H, sphi_e, mes, men, mez, tx, ty, h0.x, h0.y, h0.z, false, ef, el, flags);
        const int n_odd = ol - of, n_even = el - ef;
        for (int j = 0; j < n_odd + n_even; ++j) {
          const int h2i = j < n_odd ? of + j : ef + j - n_odd;
          if (KE && !(KE[h2i] & 2u)) continue;
          const float4 h2 = H[h2i];
          const float dz = h2.z - h0.z;
          const float predx = tx * dz;
          const float predy = ty * dz;
          const float scatterDenom2 = 1.f / ((h2.z - h1.z) * (h2.z - h1.z));
          const float fit = forward_fit(h0.x, h0.y, h2.x, h2.y, predx, predy, scatterDenom2);
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
        const uint32_t slot = n_tracks + new_rank;
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
      if (n_tracks + n_new > kMaxTracks) flags |= kStatusTrackOverflow;
      n_tracks = min(n_tracks + n_new, kMaxTracks);
      const bool push = stored || action == 2;
      uint32_t n_push;
      const uint32_t push_rank = ballot_rank(push, n_push);
      if (push) {
        const uint32_t value =
          action == 2 ? ((((full & 0x70000000u) >> 28) + 1) << 28) | (full & 0x8FFFFFFFu) : trackno;
        ttf[(ttf_ptr + push_rank) % kTtfModulo] = value;
      }
      ttf_ptr += n_push;
      uint32_t n_weak;
      const uint32_t weak_rank = ballot_rank(action == 3, n_weak);
      if (action == 3 && weak_ptr + weak_rank < kWeakCap) {
        uint16_t* w = weak + 3 * (weak_ptr + weak_rank);
        w[0] = t0;
        w[1] = t1;
        w[2] = t2;
      }
      weak_ptr += n_weak;
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
    last_ttf = ttf_ptr;
    if (last_ttf - prev > kTtfModulo) flags |= kStatusTtfOverflow;
    forwarding(first, prev, last_ttf - prev);
    if (ttf_ptr - prev > kTtfModulo) flags |= kStatusTtfOverflow;
    seeding(first);
    first -= 2;
  }
  {
    // tracklets still waiting become weak (ProcessModules.cu:146-162)
    const uint32_t prev = last_ttf;
    const uint32_t diff = ttf_ptr - prev;
    for (uint32_t i0 = 0; i0 < diff; i0 += 32) {
      const uint32_t i = i0 + lane;
      uint32_t full = 0;
      if (i < diff) full = ttf[(prev + i) % kTtfModulo];
      const bool is_weak = i < diff && (full & 0x80000000u);
      uint32_t n_weak;
      const uint32_t rank = ballot_rank(is_weak, n_weak);
      if (is_weak && weak_ptr + rank < kWeakCap) {
        const uint32_t tp = full & 0x0FFFFFFFu;
        uint16_t* w = weak + 3 * (weak_ptr + rank);
        w[0] = tracklets[3 * tp];
        w[1] = tracklets[3 * tp + 1];
        w[2] = tracklets[3 * tp + 2];
      }
      weak_ptr += n_weak;
    }
  }
  if (weak_ptr > kMaxWeakTracks) flags |= kStatusWeakOverflow;
  __syncwarp();
  // ---- weak_tracks_adder (WeakTracksAdder.cu:88-115) ----
  const uint32_t n_weak = min(weak_ptr, kWeakCap);
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
      const uint32_t slot = n_tracks + rank;
      if (slot < kMaxTracks) {
        uint16_t* th = track_hits + slot * kMaxTrackSize;
        th[0] = h[0];
        th[1] = h[1];
        th[2] = h[2];
        track_n[slot] = 3;
      }
    }
    if (n_tracks + n_acc > kMaxTracks) flags |= kStatusTrackOverflow;
    n_tracks = min(n_tracks + n_acc, kMaxTracks);
  }
  __syncwarp();
  return n_tracks;
}

// 8 blocks of 4 warps per SM at 64 registers: more resident events (10 or 12 blocks at 48 or
// 40 registers) measured slower, their hit records competing for L1.
template<int WPB>
__global__ void __launch_bounds__(WPB * 32, 8) search_kernel(ChainPointers P)
{
  __shared__ SearchWarpShared s_warp[WPB];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  SearchWarpShared& sw = s_warp[warp];

  for (;;) {
    uint32_t q = 0;
    if (lane == 0) q = atomicAdd(P.queue + 1, 1u);
    q = __shfl_sync(0xFFFFFFFFu, q, 0);
    if (q >= P.queue[4]) break;
    const uint32_t e = P.event_order[q];
    const uint32_t nhits = P.event_hits[e];
    const uint32_t status = P.status[e];
    const uint32_t base = P.event_hit_base[e];
    uint32_t flags = 0;  // per lane, OR-reduced at the end
    uint32_t n_tracks = 0, total_hits_on_tracks = 0;
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (nhits > kEventHitCap) flags |= kStatusHitOverflow;
    if (runnable) {
      search_event_setup(sw, P.module_start + e * kModules, P.module_num + e * kModules, base, nhits);
      const EventScratch sc{P.scratch.track_n + static_cast<size_t>(e) * kMaxTracks,
                            P.scratch.track_hits + static_cast<size_t>(e) * kMaxTracks * kMaxTrackSize,
                            P.scratch.tracklets + static_cast<size_t>(e) * kTrackletRing * 3,
                            P.scratch.ttf + static_cast<size_t>(e) * kTtfModulo,
                            P.scratch.weak + static_cast<size_t>(e) * kWeakCap * 3};
      const uint8_t* KE = (P.keep && P.mlp.use_ext) ? P.keep + base : nullptr;  // extension pruning
      n_tracks = search_event_warp(sw, P.hits.xyzp + base, StoredWindows{P.windows + base}, KE, sc, flags);
      uint32_t sum = 0;
      for (uint32_t t = lane; t < n_tracks; t += 32) sum += sc.track_n[t];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
      total_hits_on_tracks = sum;
    }
    uint32_t f = flags;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) f |= __shfl_xor_sync(0xFFFFFFFFu, f, o);
    if (lane == 0) {
      P.event_tracks[e] = runnable ? n_tracks : 0;
      P.event_track_hits[e] = runnable ? total_hits_on_tracks : 0;
      P.status[e] = status | f;
    }
    __syncwarp();
  }
}

}  // namespace velo
