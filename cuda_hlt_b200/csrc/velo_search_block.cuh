// search_by_triplet with one block (8 warps) per event.
//
// The event's phi-sorted clusters (float4 x, y, z, phi) are copied into shared memory by
// one TMA bulk copy (cp.async.bulk, completion on an mbarrier, bounded wait); events
// larger than the staging area read global memory instead. Seeding and forwarding follow
// the reference rules exactly as the warp-per-event kernel does, with the work of a step
// spread over 256 threads and every append to a ring buffer ranked in (iteration, warp,
// lane) order, so results are independent of scheduling and equal to the warp kernel's.
#pragma once
#include "velo_search.cuh"

namespace velo {

constexpr uint32_t kBlockWarps = 8;
constexpr uint32_t kBlockThreads = 32 * kBlockWarps;
constexpr uint32_t kStageCap = 4096;             // clusters staged in shared memory per event
constexpr uint32_t kBulkWaitLimit = 1u << 24;    // polls of the copy barrier before giving up
constexpr uint32_t kStatusStageTimeout = 1u << 12;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One thread: expect `bytes` on the barrier and start the global -> shared bulk copy.
__device__ __forceinline__ void bulk_copy_to_shared(void* dst, const void* src, uint32_t bytes,
                                                    unsigned long long* bar)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
    "l"(src), "r"(bytes), "r"(smem_addr(bar))
    : "memory");
}

// Bounded wait for the barrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity)
{
  for (uint32_t it = 0; it < kBulkWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
    if (done) return true;
  }
  return false;
}

struct BlockSeedSlots {
  uint16_t h1[kBlockThreads];
  uint16_t f0[kBlockThreads];
  uint16_t f2[kBlockThreads];
  uint16_t l2[kBlockThreads];
  uint16_t np[kBlockThreads];
  uint32_t pair_start[kBlockThreads];
  unsigned long long best[kBlockThreads];
  unsigned long long last[kBlockThreads];
};

struct BlockSearchShared {
  uint32_t used[kEventHitCap / 32];
  uint32_t mstart[kModules];
  uint32_t mnum[kModules];
  BlockSeedSlots seed;
  uint32_t warp_cnt[kBlockWarps];
  uint32_t event;
  uint32_t flags;
  unsigned long long bar;
};

// Exclusive block ranks of up to three predicates at once (each count <= 256 fits 10 bits).
__device__ __forceinline__ void block_rank3(uint32_t* warp_cnt, bool p0, bool p1, bool p2, uint32_t r[3],
                                            uint32_t tot[3])
{
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, p0), b1 = __ballot_sync(0xFFFFFFFFu, p1),
                 b2 = __ballot_sync(0xFFFFFFFFu, p2);
  if (lane == 0) warp_cnt[warp] = __popc(b0) | (__popc(b1) << 10) | (__popc(b2) << 20);
  __syncthreads();
  uint32_t pre = 0, all = 0;
#pragma unroll
  for (uint32_t w = 0; w < kBlockWarps; ++w) {
    const uint32_t v = warp_cnt[w];
    pre += w < warp ? v : 0u;
    all += v;
  }
  __syncthreads();
  r[0] = (pre & 0x3FFu) + __popc(b0 & lt);
  r[1] = ((pre >> 10) & 0x3FFu) + __popc(b1 & lt);
  r[2] = ((pre >> 20) & 0x3FFu) + __popc(b2 & lt);
  tot[0] = all & 0x3FFu;
  tot[1] = (all >> 10) & 0x3FFu;
  tot[2] = (all >> 20) & 0x3FFu;
}

// Exclusive block scan of one value per thread; returns the exclusive prefix and the total.
__device__ __forceinline__ uint32_t block_scan(uint32_t* warp_cnt, uint32_t v, uint32_t& total)
{
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= static_cast<uint32_t>(o)) incl += t;
  }
  if (lane == 31) warp_cnt[warp] = incl;
  __syncthreads();
  uint32_t pre = 0, all = 0;
#pragma unroll
  for (uint32_t w = 0; w < kBlockWarps; ++w) {
    const uint32_t c = warp_cnt[w];
    pre += w < warp ? c : 0u;
    all += c;
  }
  __syncthreads();
  total = all;
  return pre + incl - v;
}

__global__ void __launch_bounds__(kBlockThreads) search_block_kernel(ChainPointers P)
{
  extern __shared__ __align__(16) uint8_t dyn[];
  float4* stage = reinterpret_cast<float4*>(dyn);
  __shared__ BlockSearchShared sb;
  const uint32_t tid = threadIdx.x;
  uint32_t* used = sb.used;
  uint32_t* mstart = sb.mstart;
  uint32_t* mnum = sb.mnum;
  BlockSeedSlots& sl = sb.seed;
  if (tid == 0) mbar_init(&sb.bar, 1);
  __syncthreads();
  uint32_t phase = 0;

  for (;;) {
    if (tid == 0) {
      sb.event = atomicAdd(P.queue + 2, 1u);
      sb.flags = 0;
    }
    __syncthreads();
    const uint32_t e = sb.event;
    if (e >= P.queue[5]) break;
    const uint32_t ev = P.block_events[e];
    const uint32_t nhits = P.event_hits[ev];
    const uint32_t status = P.status[ev];
    const uint32_t base = P.event_hit_base[ev];
    uint32_t flags = 0;
    uint32_t n_tracks = 0, tracklet_ptr = 0, ttf_ptr = 0, weak_ptr = 0;
    uint32_t total_hits_on_tracks = 0;
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (nhits > kEventHitCap) flags |= kStatusHitOverflow;
    if (runnable) {
      const bool staged = nhits <= kStageCap;
      if (staged && tid == 0) {
        // order earlier generic reads of the staging area before the async-proxy writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        bulk_copy_to_shared(stage, P.hits.xyzp + base, nhits * sizeof(float4), &sb.bar);
      }
      for (uint32_t i = tid; i < (nhits + 31) / 32; i += kBlockThreads) used[i] = 0u;
      for (uint32_t m = tid; m < kModules; m += kBlockThreads) {
        mstart[m] = P.module_start[ev * kModules + m] - base;
        mnum[m] = P.module_num[ev * kModules + m];
      }
      bool ok = true;
      if (staged) {
        ok = mbar_wait(&sb.bar, phase);
        phase ^= 1u;
        if (!ok) atomicOr(&sb.flags, kStatusStageTimeout);
      }
      __syncthreads();
      if (sb.flags & kStatusStageTimeout) {
        // The copy did not complete within the limit: report and stop this block; its
        // staging area may still be written, so it takes no further events.
        if (tid == 0) atomicOr(P.status + ev, kStatusStageTimeout);
        return;
      }
      const float4* H = staged ? stage : P.hits.xyzp + base;
      const uint2* Wn = P.windows + base;  // phi windows of every h1 (fill_candidates)
      const uint8_t* KE = (P.keep && P.mlp.use_ext) ? P.keep + base : nullptr;
      uint16_t* track_n = P.scratch.track_n + static_cast<size_t>(ev) * kMaxTracks;
      uint16_t* track_hits = P.scratch.track_hits + static_cast<size_t>(ev) * kMaxTracks * kMaxTrackSize;
      uint16_t* tracklets = P.scratch.tracklets + static_cast<size_t>(ev) * kTrackletRing * 3;
      uint32_t* ttf = P.scratch.ttf + static_cast<size_t>(ev) * kTtfModulo;
      uint16_t* weak = P.scratch.weak + static_cast<size_t>(ev) * kWeakCap * 3;
      uint32_t last_seeded = 0;

      // ---- seeding over the hits of modules first-2 and first-3 taken together ----
      auto seeding = [&](uint32_t first) {
        uint32_t n_h1 = 0;
        const uint32_t tracklets_before = tracklet_ptr;
        const uint32_t ma = first - 2, mb = first - 3;
        const uint32_t na = mnum[ma], total_h1 = na + mnum[mb];
        for (uint32_t r0 = 0; r0 < total_h1; r0 += kBlockThreads) {
          // (a) unused h1 with both phi windows (FillCandidates.cu:31-68, TrackSeeding.cu:24-49)
          const uint32_t r = r0 + tid;
          int f0 = -1, l0 = -1, f2 = -1, l2 = -1;
          bool has = false;
          uint32_t h1 = 0;
          if (r < total_h1) {
            const uint32_t m = r < na ? ma : mb;
            h1 = mstart[m] + (r < na ? r : r - na);
            if (!test_used(used, h1)) {
              const uint2 w = Wn[h1];
              f0 = static_cast<int>(w.x & 0xFFFFu);
              l0 = static_cast<int>(w.x >> 16);
              f2 = static_cast<int>(w.y & 0xFFFFu);
              l2 = static_cast<int>(w.y >> 16);
              has = f0 != 0xFFFF && f2 != 0xFFFF;
            }
          }
          uint32_t rk[3], tot[3];
          block_rank3(sb.warp_cnt, has, false, false, rk, tot);
          const uint32_t nc = tot[0];
          if (has) {
            const uint32_t k = rk[0];
            sl.h1[k] = static_cast<uint16_t>(h1);
            sl.f0[k] = static_cast<uint16_t>(f0);
            sl.np[k] = static_cast<uint16_t>(l0 - f0);
            sl.f2[k] = static_cast<uint16_t>(f2);
            sl.l2[k] = static_cast<uint16_t>(l2);
            sl.best[k] = ~0ull;
            sl.last[k] = 0ull;
          }
          n_h1 += nc;
          __syncthreads();
          // (b) exclusive scan of the h0 counts
          uint32_t total_pairs;
          const uint32_t ps = block_scan(sb.warp_cnt, tid < nc ? sl.np[tid] : 0u, total_pairs);
          if (tid < nc) sl.pair_start[tid] = ps;
          __syncthreads();
          // (c) (h1, h0) pairs over the threads, each scanning its h2 window
          for (uint32_t p = tid; p < total_pairs; p += kBlockThreads) {
            uint32_t lo = 0, hi = nc;  // last k with pair_start[k] <= p
            while (hi - lo > 1) {
              const uint32_t mid = (lo + hi) >> 1;
              if (sl.pair_start[mid] <= p) lo = mid; else hi = mid;
            }
            const uint32_t k = lo;
            const uint32_t h0rel = p - sl.pair_start[k];
            const uint32_t h0i = sl.f0[k] + h0rel;
            if (test_used(used, h0i)) continue;
            const float4 h0 = H[h0i];
            const float4 hh1 = H[sl.h1[k]];
            const uint32_t f2k = sl.f2[k], l2k = sl.l2[k];
            unsigned long long best = ~0ull, last = 0ull;
            for (uint32_t h2i = f2k; h2i < l2k; ++h2i) {
              if (test_used(used, h2i)) continue;
              float scatter;
              if (seed_scatter(h0, hh1, H[h2i], scatter)) {
                const uint32_t idx = (h0rel << 16) | (h2i - f2k);
                const uint32_t sbits = __float_as_uint(scatter);
                best = min(best, (static_cast<unsigned long long>(sbits) << 32) | idx);
                last = max(last, (static_cast<unsigned long long>(~sbits) << 32) | idx);
              }
            }
            if (best != ~0ull) {
              atomicMin(&sl.best[k], best);
              atomicMax(&sl.last[k], last);
            }
          }
          __syncthreads();
          // (d) winners, appended in candidate order (TrackSeeding.cu:185-195)
          const bool win = tid < nc && sl.best[tid] != ~0ull;
          block_rank3(sb.warp_cnt, win, false, false, rk, tot);
          if (win) {
            const unsigned long long key = sl.best[tid];
            if ((key & 0xFFFFFFFFull) != (sl.last[tid] & 0xFFFFFFFFull)) flags |= kStatusSeedTie;
            const uint32_t tp = (tracklet_ptr + rk[0]) % kTrackletRing;
            tracklets[3 * tp] = static_cast<uint16_t>(sl.f0[tid] + ((key >> 16) & 0xFFFFu));
            tracklets[3 * tp + 1] = sl.h1[tid];
            tracklets[3 * tp + 2] = static_cast<uint16_t>(sl.f2[tid] + (key & 0xFFFFu));
            ttf[(ttf_ptr + rk[0]) % kTtfModulo] = 0x80000000u | tp;
          }
          tracklet_ptr += tot[0];
          ttf_ptr += tot[0];
          __syncthreads();
        }
        if (n_h1 > kMaxHitsPerModule) flags |= kStatusH1Overflow;
        const uint32_t seeded = tracklet_ptr - tracklets_before;
        if (seeded + last_seeded > kTrackletRing) flags |= kStatusTtfOverflow;
        last_seeded = seeded;
      };

      // ---- forwarding into modules first-4 (odd) / first-5 (even) ----
      auto forwarding = [&](uint32_t first, uint32_t prev_ttf, uint32_t diff) {
        const uint32_t mo = first - 4, me = first - 5;
        const uint32_t mos = mstart[mo], mon = mnum[mo], mes = mstart[me], men = mnum[me];
        const float moz = c_module_z[mo], mez = c_module_z[me];
        for (uint32_t i0 = 0; i0 < diff; i0 += kBlockThreads) {
          const uint32_t i = i0 + tid;
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
            forward_window(H, mos, mon, moz, tx, ty, h0.x, h0.y, h0.z, true, of, ol, flags);
            forward_window(H, mes, men, mez, tx, ty, h0.x, h0.y, h0.z, false, ef, el, flags);
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
          const bool is_new = action == 1 && nhit == 3;
          uint32_t rk[3], tot[3];
          // new-track slots first; the pushes depend on whether a new track got a slot
          block_rank3(sb.warp_cnt, is_new, false, action == 3, rk, tot);
          bool stored = action == 1;
          if (is_new) {
            const uint32_t slot = n_tracks + rk[0];
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
          if (n_tracks + tot[0] > kMaxTracks) flags |= kStatusTrackOverflow;
          n_tracks = min(n_tracks + tot[0], kMaxTracks);
          if (action == 3 && weak_ptr + rk[2] < kWeakCap) {
            uint16_t* w = weak + 3 * (weak_ptr + rk[2]);
            w[0] = t0;
            w[1] = t1;
            w[2] = t2;
          }
          weak_ptr += tot[2];
          const bool push = stored || action == 2;
          uint32_t rk2[3], tot2[3];
          block_rank3(sb.warp_cnt, push, false, false, rk2, tot2);
          if (push) {
            const uint32_t value =
              action == 2 ? ((((full & 0x70000000u) >> 28) + 1) << 28) | (full & 0x8FFFFFFFu) : trackno;
            ttf[(ttf_ptr + rk2[0]) % kTtfModulo] = value;
          }
          ttf_ptr += tot2[0];
        }
        __syncthreads();
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
        const uint32_t prev = last_ttf;
        const uint32_t diff = ttf_ptr - prev;
        for (uint32_t i0 = 0; i0 < diff; i0 += kBlockThreads) {
          const uint32_t i = i0 + tid;
          uint32_t full = 0;
          if (i < diff) full = ttf[(prev + i) % kTtfModulo];
          const bool is_weak = i < diff && (full & 0x80000000u);
          uint32_t rk[3], tot[3];
          block_rank3(sb.warp_cnt, is_weak, false, false, rk, tot);
          if (is_weak && weak_ptr + rk[0] < kWeakCap) {
            const uint32_t tp = full & 0x0FFFFFFFu;
            uint16_t* w = weak + 3 * (weak_ptr + rk[0]);
            w[0] = tracklets[3 * tp];
            w[1] = tracklets[3 * tp + 1];
            w[2] = tracklets[3 * tp + 2];
          }
          weak_ptr += tot[0];
        }
      }
      if (weak_ptr > kMaxWeakTracks) flags |= kStatusWeakOverflow;
      __syncthreads();
      const uint32_t n_weak = min(weak_ptr, kWeakCap);
      for (uint32_t i0 = 0; i0 < n_weak; i0 += kBlockThreads) {
        const uint32_t i = i0 + tid;
        bool accept = false;
        uint16_t h[3] = {0, 0, 0};
        if (i < n_weak) {
          h[0] = weak[3 * i];
          h[1] = weak[3 * i + 1];
          h[2] = weak[3 * i + 2];
          const bool any_used = test_used(used, h[0]) || test_used(used, h[1]) || test_used(used, h[2]);
          accept = !any_used && weak_chi2(H, h) < kMaxChi2;
        }
        uint32_t rk[3], tot[3];
        block_rank3(sb.warp_cnt, accept, false, false, rk, tot);
        if (accept) {
          const uint32_t slot = n_tracks + rk[0];
          if (slot < kMaxTracks) {
            uint16_t* th = track_hits + slot * kMaxTrackSize;
            th[0] = h[0];
            th[1] = h[1];
            th[2] = h[2];
            track_n[slot] = 3;
          }
        }
        if (n_tracks + tot[0] > kMaxTracks) flags |= kStatusTrackOverflow;
        n_tracks = min(n_tracks + tot[0], kMaxTracks);
      }
      __syncthreads();
      uint32_t sum = 0;
      for (uint32_t t = tid; t < n_tracks; t += kBlockThreads) sum += track_n[t];
      uint32_t total;
      block_scan(sb.warp_cnt, sum, total);
      total_hits_on_tracks = total;
    }
    if (flags) atomicOr(&sb.flags, flags);
    __syncthreads();
    if (tid == 0) {
      P.event_tracks[ev] = runnable ? n_tracks : 0;
      P.event_track_hits[ev] = runnable ? total_hits_on_tracks : 0;
      P.status[ev] = status | sb.flags;
    }
    __syncthreads();
  }
}

}  // namespace velo
