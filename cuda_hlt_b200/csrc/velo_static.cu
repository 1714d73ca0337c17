// velo_search_static: search_by_triplet for callers that cannot allocate device memory.
//
// Some callers own all device memory themselves and give plugins no way to allocate: a host
// framework that reserves the device up front and hands out fixed slices (the stage this
// library replaces runs inside such an arena: one cudaMalloc per stream at start-up, every
// buffer a slice of it), or an embedding runtime whose allocator is not reachable from this
// code. This entry point needs no allocation: its scratch - the per-event rings of tracklets,
// of tracks to follow and of weak tracklets, and the work-queue counter - lives in one
// file-scope __device__ array of fixed size, and the caller passes inputs and outputs.
//
// Limits and sharing: at most kStaticMaxEvents events per call (larger calls are rejected
// with VELO_ERR_CAPACITY); the array (kStaticScratchBytes) stays resident on every device
// that loads the library until the process exits; every call uses the same array, so calls
// whose work overlaps on a device race with each other. The first call on a device looks up
// the array's device address (cudaGetSymbolAddress) and caches it; that first call should
// come before any stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/velo_b200.h"
#include "velo_search.cuh"

namespace velo {
namespace {

constexpr uint32_t kStaticMaxEvents = 512;
constexpr size_t kTrackletBytes = kTrackletRing * 3 * sizeof(uint16_t);  // 12000
constexpr size_t kTtfBytes = kTtfModulo * sizeof(uint32_t);                // 8000
constexpr size_t kWeakBytes = kWeakCap * 3 * sizeof(uint16_t);            // 24576
constexpr size_t kEventScratchBytes = ((kTrackletBytes + kTtfBytes + kWeakBytes + 255) / 256) * 256;
constexpr size_t kStaticHeaderBytes = 256;  // work-queue counter, zeroed by every call
constexpr size_t kStaticScratchBytes = kStaticHeaderBytes + kStaticMaxEvents * kEventScratchBytes;  // ~22.9 MB

// The scratch. In host code this name is only a stand-in for the device symbol: kernels get
// the device address looked up by cudaGetSymbolAddress below.
static __device__ __align__(256) uint8_t velo_static_scratch[kStaticScratchBytes];

struct StaticSearchArgs {
  const float4* xyzp;
  const uint32_t* module_start;
  const uint32_t* module_num;
  const uint32_t* status_in;
  uint32_t n_events;
  uint16_t* track_n;      // [n * kMaxTracks]
  uint16_t* track_hits;   // [n * kMaxTracks * kMaxTrackSize]
  uint32_t* event_tracks; // [n]
  uint32_t* status_out;   // [n]
  uint8_t* scratch;       // device address of velo_static_scratch
};

// Warp per event, events pulled from the counter at the head of the scratch. Same rules and
// lane-ordered appends as the warp-per-event search of the chain (velo_search.cuh).
__global__ void __launch_bounds__(128) search_static_kernel(StaticSearchArgs A)
{
  __shared__ SearchWarpShared s_warp[4];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  SearchWarpShared& sw = s_warp[warp];
  uint32_t* used = sw.used;
  uint32_t* mstart = sw.mstart;
  uint32_t* mnum = sw.mnum;
  SeedSlots& sl = sw.u.seed;
  uint32_t* queue = reinterpret_cast<uint32_t*>(A.scratch);

  for (;;) {
    uint32_t e = 0;
    if (lane == 0) e = atomicAdd(queue, 1u);
    e = __shfl_sync(0xFFFFFFFFu, e, 0);
    if (e >= A.n_events) break;
    const uint32_t base = A.module_start[e * kModules];
    const uint32_t nhits = A.module_start[e * kModules + kModules - 1] + A.module_num[e * kModules + kModules - 1] - base;
    const uint32_t status = A.status_in[e];
    uint32_t flags = 0;
    uint32_t n_tracks = 0, tracklet_ptr = 0, ttf_ptr = 0, weak_ptr = 0;
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (nhits > kEventHitCap) flags |= kStatusHitOverflow;
    if (runnable) {
      for (uint32_t i = lane; i < (nhits + 31) / 32; i += 32) used[i] = 0u;
      for (uint32_t m = lane; m < kModules; m += 32) {
        mstart[m] = A.module_start[e * kModules + m] - base;
        mnum[m] = A.module_num[e * kModules + m];
      }
      __syncwarp();
      const float4* H = A.xyzp + base;
      uint16_t* track_n = A.track_n + static_cast<size_t>(e) * kMaxTracks;
      uint16_t* track_hits = A.track_hits + static_cast<size_t>(e) * kMaxTracks * kMaxTrackSize;
      uint8_t* ev_scratch = A.scratch + kStaticHeaderBytes + static_cast<size_t>(e) * kEventScratchBytes;
      uint16_t* tracklets = reinterpret_cast<uint16_t*>(ev_scratch);
      uint32_t* ttf = reinterpret_cast<uint32_t*>(ev_scratch + kTrackletBytes);
      uint16_t* weak = reinterpret_cast<uint16_t*>(ev_scratch + kTrackletBytes + kTtfBytes);
      uint32_t last_seeded = 0;

      auto seeding = [&](uint32_t first) {
        uint32_t n_h1 = 0;
        const uint32_t tracklets_before = tracklet_ptr;
        for (int side = 2; side <= 3; ++side) {
          const uint32_t m = first - side;
          const uint32_t start = mstart[m], num = mnum[m];
          const uint32_t m0s = mstart[m + 2], m0n = mnum[m + 2], m2s = mstart[m - 2], m2n = mnum[m - 2];
          for (uint32_t r0 = 0; r0 < num; r0 += kSeedChunk) {
            const uint32_t r_end = min(num, r0 + kSeedChunk);
            uint32_t nc = 0;
            for (uint32_t r1 = r0; r1 < r_end; r1 += 32) {
              const uint32_t r = r1 + lane;
              const uint32_t h1 = start + r;
              int f0 = -1, l0 = -1, f2 = -1, l2 = -1;
              bool has = false;
              if (r < r_end && !test_used(used, h1)) {
                const float p = H[h1].w;
                if (m0n > 0) phi_window4(H, m0s, m0n, p, kPhiExtrapolation, f0, l0);
                if (m2n > 0) phi_window4(H, m2s, m2n, p, kPhiExtrapolation, f2, l2);
                has = f0 != -1 && f2 != -1;
              }
              uint32_t cnt;
              const uint32_t rank = ballot_rank(has, cnt);
              if (has) {
                const uint32_t k = nc + rank;
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
            n_h1 += nc;
            __syncwarp();
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
            for (uint32_t p0 = 0; p0 < total_pairs; p0 += 32) {
              const uint32_t p = p0 + lane;
              if (p < total_pairs) {
                uint32_t lo = 0, hi = nc;
                while (hi - lo > 1) {
                  const uint32_t mid = (lo + hi) >> 1;
                  if (sl.pair_start[mid] <= p) lo = mid; else hi = mid;
                }
                const uint32_t k = lo;
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
                      best = min(best, (static_cast<unsigned long long>(sb) << 32) | idx);
                      last = max(last, (static_cast<unsigned long long>(~sb) << 32) | idx);
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
          }
        }
        if (n_h1 > kMaxHitsPerModule) flags |= kStatusH1Overflow;
        const uint32_t seeded = tracklet_ptr - tracklets_before;
        if (seeded + last_seeded > kTrackletRing) flags |= kStatusTtfOverflow;
        last_seeded = seeded;
      };

      auto forwarding = [&](uint32_t first, uint32_t prev_ttf, uint32_t diff) {
        const uint32_t mo = first - 4, me = first - 5;
        const uint32_t mos = mstart[mo], mon = mnum[mo], mes = mstart[me], men = mnum[me];
        const float moz = c_module_z[mo], mez = c_module_z[me];
        for (uint32_t i0 = 0; i0 < diff; i0 += 32) {
          const uint32_t i = i0 + lane;
          int action = 0;
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
          accept = !any_used && weak_chi2(H, h) < kMaxChi2;
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
    }
    uint32_t f = flags;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) f |= __shfl_xor_sync(0xFFFFFFFFu, f, o);
    if (lane == 0) {
      A.event_tracks[e] = runnable ? n_tracks : 0;
      A.status_out[e] = status | f;
    }
    __syncwarp();
  }
}

std::mutex g_symbol_mutex;
void* g_symbol_address[64] = {};

}  // namespace
}  // namespace velo

extern "C" int velo_search_static(const float* hit_xyzp, const uint32_t* module_hit_start,
                                  const uint32_t* module_hit_num, const uint32_t* status_in, uint32_t n_events,
                                  uint16_t* track_n, uint16_t* track_hits, uint32_t* event_tracks,
                                  uint32_t* status_out, void* stream)
{
  using namespace velo;
  if (n_events == 0) return 0;
  if (!hit_xyzp || !module_hit_start || !module_hit_num || !status_in || !track_n || !track_hits || !event_tracks ||
      !status_out)
    return VELO_ERR_INVALID;
  if (n_events > kStaticMaxEvents) {
    std::fprintf(stderr, "velo_search_static: %u events exceed the %u-event static scratch; split the batch\n",
                 n_events, kStaticMaxEvents);
    return VELO_ERR_CAPACITY;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return VELO_ERR_CUDA;
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_symbol_mutex);
    if (!g_symbol_address[dev]) {
      // set-up, once per device, with that device current
      const cudaError_t e = cudaGetSymbolAddress(&g_symbol_address[dev], velo_static_scratch);
      if (e != cudaSuccess) {
        std::fprintf(stderr, "velo_search_static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        g_symbol_address[dev] = nullptr;
        return VELO_ERR_CUDA;
      }
    }
    scratch = g_symbol_address[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the work-queue counter starts at zero; the rings are written before they are read
  if (cudaMemsetAsync(scratch, 0, kStaticHeaderBytes, s) != cudaSuccess) return VELO_ERR_CUDA;
  StaticSearchArgs A{reinterpret_cast<const float4*>(hit_xyzp), module_hit_start, module_hit_num, status_in,
                     n_events, track_n, track_hits, event_tracks, status_out, static_cast<uint8_t*>(scratch)};
  const uint32_t blocks = (n_events + 3) / 4;
  search_static_kernel<<<blocks, 128, 0, s>>>(A);
  return cudaGetLastError() == cudaSuccess ? 0 : VELO_ERR_CUDA;
}
