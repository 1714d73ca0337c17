// Kernel 1 of the chain: SuperPixel decode, masked clustering, phi and per-module sort.
//
// One block per event (persistent; events are pulled from a device queue), one pass over
// the event's SP words:
//   * isolated SPs give their one or two clusters from the pattern table at once;
//   * a non-isolated SP finds its neighbours by binary search in its bank (banks are
//     address-sorted in LHCb raw data; unsorted banks fall back to the reference's linear
//     scan, with the same result) and pushes its candidate pixels to a shared list, which
//     the block then flood-fills with every thread busy;
//   * clusters go to their module's slice of a staging area sized by the module's SP count
//     (at most two clusters per SP), one shared atomic per cluster;
//   * one warp per module sorts the slice on the key (phi, LHCb id) - in registers with
//     warp shuffles up to 128 clusters, in shared memory up to 512 - and writes it to the
//     compact phi-sorted layout.
// The result equals the reference's estimate -> prefix sum -> masked clustering ->
// calculate_phi_and_sort sequence, whose order within a module depends on the order of its
// atomics only for exactly equal phi.
#pragma once
#include "velo_kernels.cuh"

namespace velo {

constexpr uint32_t kSortCap = 512;  // clusters per module sorted in shared memory

// SPs around one SP: the non-isolated ones of the 4x3-SP flood window
// (MaskedVeloClustering.cu:221-272) and, over every SP of the bank, the five neighbours the
// candidate search reads (EstimateInputSize.cu:124-153).
struct SpWindow {
  uint32_t px[3];
  uint32_t top, top_right, right, right_bottom, bottom;
};

__device__ __forceinline__ void window_add(SpWindow& w, uint32_t o, int32_t r, int32_t c)
{
  const int32_t orow = sp_row(o), ocol = sp_col(o);
  const uint32_t osp = sp_mask(o);
  if (!sp_isolated(o) && orow >= r - 2 && orow <= r + 1 && ocol >= c - 1 && ocol <= c + 1) {
    const int32_t rr = orow - (r - 2), rc = ocol - (c - 1);
    const uint32_t v = (osp & 0x0Fu) << (4 * rr) | (osp & 0xF0u) << (12 + 4 * rr);
    // constant register indices: a runtime index would put the window in local memory
    w.px[0] |= rc == 0 ? v : 0u;
    w.px[1] |= rc == 1 ? v : 0u;
    w.px[2] |= rc == 2 ? v : 0u;
  }
  if (ocol == c) {
    if (orow == r + 1) w.top |= osp;
    if (orow == r - 1) w.bottom |= osp;
  } else if (ocol == c + 1) {
    if (orow == r + 1) w.top_right |= osp;
    if (orow == r) w.right |= osp;
    if (orow == r - 1) w.right_bottom |= osp;
  }
}

__device__ __forceinline__ uint32_t bank_lower_bound(const uint32_t* bank, uint32_t count, uint32_t addr)
{
  uint32_t lo = 0, hi = count;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (sp_addr(__ldg(bank + mid)) < addr) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ SpWindow gather_window(const uint32_t* bank, uint32_t count, bool sorted, int32_t r,
                                                  int32_t c)
{
  SpWindow w{{0u, 0u, 0u}, 0u, 0u, 0u, 0u, 0u};
  if (sorted) {
    // the three columns are adjacent in address order (column << 6 | row): one search and
    // one scan over [(c - 1, r - 2), (c + 1, r + 1)]; the rows outside [r - 2, r + 1] that
    // the scan also meets are rejected by window_add
    const uint32_t a_lo = (static_cast<uint32_t>(max(c - 1, 0)) << 6) | static_cast<uint32_t>(max(r - 2, 0));
    const uint32_t a_hi = (static_cast<uint32_t>(min(c + 1, 511)) << 6) | static_cast<uint32_t>(min(r + 1, 63));
    for (uint32_t i = bank_lower_bound(bank, count, a_lo); i < count; ++i) {
      const uint32_t o = __ldg(bank + i);
      if (sp_addr(o) > a_hi) break;
      window_add(w, o, r, c);
    }
  } else {
    for (uint32_t i = 0; i < count; ++i) window_add(w, __ldg(bank + i), r, c);
  }
  return w;
}

// Candidate-pixel code of a non-isolated SP from its neighbours (EstimateInputSize.cu:118-183).
__device__ __forceinline__ uint32_t window_candidate_code(uint32_t sp, const SpWindow& w)
{
  uint32_t pixels = (sp & 0x0Fu) | ((sp & 0xF0u) << 2);
  pixels |= ((w.top & 0x01u) | ((w.top & 0x10u) << 2)) << 4;
  pixels |= (w.top_right & 0x01u) << 16;
  pixels |= (w.right & 0x0Fu) << 12;
  pixels |= (w.right_bottom & 0x08u) << 8;
  pixels |= (w.bottom & 0x80u) >> 2;
  const uint32_t inside = pixels & 0x3CFu;
  const uint32_t mask = (inside << 1) | (inside << 5) | (inside << 6) | (inside << 7);
  const uint32_t open = mask & (~pixels);
  const uint32_t cand = (open >> 1) & (open >> 5) & (open >> 6) & (open >> 7) & pixels;
  return (cand & 0x03u) | ((cand & 0xC0u) >> 4) | ((cand & 0x0Cu) << 2) | ((cand & 0x0300u) >> 2);
}

// Flood fill seeded by pixel k of the SP at (sp_r, sp_c) over the window pixels
// (MaskedVeloClustering.cu:274-398). True when the cluster is stored.
__device__ __forceinline__ bool flood_window(uint32_t px0, uint32_t px1, uint32_t px2, int32_t sp_r, int32_t sp_c,
                                             uint32_t k, int32_t& xs, int32_t& ys, int32_t& n)
{
  const int32_t row_lower_limit = (sp_r - 2) * 4, col_lower_limit = (sp_c - 1) * 2;
  const uint32_t row = sp_r * 4 + (k % 4);
  const uint32_t col = sp_c * 2 + (k >= 4);
  const uint32_t seed = (0x01u << (row - row_lower_limit)) << (16 * (col % 2));
  uint32_t cl0 = 0, cl1 = seed, cl2 = 0;
  uint32_t w0 = 0, w1 = seed, w2 = 0;
  px1 &= ~cl1;
#pragma unroll 1
  for (uint32_t it = 0; it < kMaxClusteringIterations; ++it) {
    const uint32_t m0 = flood_mask(w0) | flood_right_to_left(w1);
    const uint32_t m1 = flood_mask(w1) | flood_right_to_left(w2) | flood_left_to_right(w0);
    const uint32_t m2 = flood_mask(w2) | flood_left_to_right(w1);
    w0 = px0 & m0;
    w1 = px1 & m1;
    w2 = px2 & m2;
    if ((w0 | w1 | w2) == 0u) break;
    cl0 |= w0;
    cl1 |= w1;
    cl2 |= w2;
    px0 &= ~cl0;
    px1 &= ~cl1;
    px2 &= ~cl2;
  }
  if (cl2) return false;  // a pixel in the SP column to the right owns this cluster
  n = __popc(cl0) + __popc(cl1);
  if (n >= 3) {
    const uint32_t c0 = found_cluster_mask(cl0) & ~cl0;
    const uint32_t c1 = (found_cluster_mask(cl1) | flood_left_to_right(cl0)) & ~cl1;
    const uint32_t c2 = flood_left_to_right(cl1);
    const uint32_t cand0 = precedence_candidates(c0, c1) & cl0;
    const uint32_t cand1 = (precedence_candidates(c1, c2) & cl1) ^ seed;
    if (cand0 | cand1) {
      const int32_t neg = ~(-static_cast<int32_t>(seed));
      const bool under = seed < 4096u;
      uint32_t smaller_row = under * (0xFFF & neg) | (!under) * (0xFFF & (neg >> 16));
      smaller_row |= smaller_row << 16;
      const uint32_t current = smaller_row | under * 0xFFFF0000u;
      if (((cand0 & smaller_row) | (cand1 & current)) != 0u) return false;
    }
  }
  xs = __popc(cl0 & 0x0000FFFFu) * col_lower_limit + __popc(cl0 & 0xFFFF0000u) * (col_lower_limit + 1) +
       __popc(cl1 & 0x0000FFFFu) * (col_lower_limit + 2) + __popc(cl1 & 0xFFFF0000u) * (col_lower_limit + 3);
  const uint32_t t0 = (cl0 & 0x000F000Fu) | ((cl1 & 0x000F000Fu) << 4);
  const uint32_t t1 = ((cl0 & 0x00F000F0u) >> 4) | (cl1 & 0x00F000F0u);
  const uint32_t t2 = ((cl0 & 0x0F000F00u) >> 8) | ((cl1 & 0x0F000F00u) >> 4);
  const uint32_t t3 = ((cl0 & 0xF000F000u) >> 12) | ((cl1 & 0xF000F000u) >> 8);
  int32_t y = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const uint32_t m = 0x11111111u << r;
    y += __popc(t0 & m) * (row_lower_limit + r) + __popc(t1 & m) * (row_lower_limit + 4 + r) +
         __popc(t2 & m) * (row_lower_limit + 8 + r) + __popc(t3 & m) * (row_lower_limit + 12 + r);
  }
  ys = y;
  return true;
}

constexpr uint32_t kCandCap = 4096;    // candidate pixels listed per event (more: flooded inline)
constexpr uint32_t kBankMapCap = 16384; // SPs per event with a bank map (more: binary search)
constexpr uint32_t kNonIsoCap = 2048;   // non-isolated SPs listed per event (more: full rescan)
constexpr uint32_t kRegSortMax = 128;  // modules up to this size are sorted in registers

struct DecodeShared {
  uint32_t bank_start[kSensors];  // word index (from the event start) of the first SP word
  uint32_t bank_count[kSensors];
  uint32_t bank_sensor[kSensors];
  uint32_t sp_prefix[kSensors + 1];  // exclusive scan of bank_count
  uint32_t unsorted[(kSensors + 31) / 32];
  uint32_t mod_count[kModules];  // clusters per module
  uint32_t mod_start[kModules];  // exclusive scan of mod_count: compact layout
  uint32_t event;
  uint32_t n_events;             // events of the run
  uint32_t skipped;              // 1: position left empty (beyond the selection); 2: bad list entry
  uint64_t ev_off, ev_bytes;     // the event's raw bytes: offset in the batch and size
  uint32_t flags;
  uint32_t n_candidates;
  uint32_t n_list;
  uint32_t n_noniso;  // non-isolated SPs met by the first pass
};

__device__ __forceinline__ uint32_t bank_of(const DecodeShared& sh, uint32_t f)
{
  uint32_t lo = 0, hi = kSensors;  // last b with sp_prefix[b] <= f
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (sh.sp_prefix[mid] <= f) lo = mid; else hi = mid;
  }
  return lo;
}

struct DecodeEvent {
  const uint32_t* ev;       // raw event words
  uint32_t stage_base;      // first staging slot of the event
  float4* stage;
  uint32_t* stage_id;
  const uint8_t* bank_map;  // bank of each flat SP index (shared memory), or null
};

__device__ __forceinline__ uint32_t bank_of_sp(const DecodeShared& sh, const DecodeEvent& d, uint32_t f)
{
  return d.bank_map ? d.bank_map[f] : bank_of(sh, f);
}

// Bits 26-27 of an LHCb VP id are always zero (sensor < 208 ends at bit 25): the staging
// record carries the cluster's pixel count there, at most 3.
constexpr uint32_t kSizeShift = 26;
constexpr uint32_t kSizeMask = 3u << kSizeShift;

// Appends one cluster of `pixels` pixels to module m's staging slice: slots
// [2 * SPs before m, ...).
__device__ __forceinline__ void stage_cluster(DecodeShared& sh, const DecodeEvent& d, uint32_t m,
                                              const ClusterPoint& p, uint32_t pixels)
{
  const uint32_t slot = atomicAdd(&sh.mod_count[m], 1u);
  const uint32_t o = d.stage_base + 2 * sh.sp_prefix[4 * m] + slot;
  const float phi = (m & 1) ? phi_odd_side(p.x, p.y) : phi_even_side(p.x, p.y);
  d.stage[o] = make_float4(p.x, p.y, p.z, phi);
  d.stage_id[o] = p.id | (min(pixels, 3u) << kSizeShift);
}

// Flood fill of candidate pixel k of flat SP f and staging of the cluster
// (MaskedVeloClustering.cu:175-461).
__device__ __forceinline__ void flood_candidate(DecodeShared& sh, const DecodeEvent& d, const GeometryView& g,
                                                uint32_t f, uint32_t k)
{
  const uint32_t b = bank_of_sp(sh, d, f);
  const uint32_t s = f - sh.sp_prefix[b];
  const uint32_t* bank = d.ev + sh.bank_start[b];
  const uint32_t count = sh.bank_count[b];
  const bool sorted = !((sh.unsorted[b >> 5] >> (b & 31)) & 1u);
  // The reference packs the SP index into a u8 when it decodes candidates
  // (MaskedVeloClustering.cu:179), so above 255 SPs the flood runs on SP s & 0xFF.
  const uint32_t word2 = __ldg(bank + (s & 0xFFu));
  const int32_t r2 = sp_row(word2), c2 = sp_col(word2);
  const SpWindow w = gather_window(bank, count, sorted, r2, c2);
  int32_t xs, ys, np;
  if (!flood_window(w.px[0], w.px[1], w.px[2], r2, c2, k, xs, ys, np)) return;
  const uint32_t cx = xs / np;
  const uint32_t cy = ys / np;
  const float fx = xs / static_cast<float>(np) - cx;
  const float fy = ys / static_cast<float>(np) - cy;
  stage_cluster(sh, d, b >> 2, place_cluster(g, sh.bank_sensor[b], cx, cy, fx, fy, cx / kChipColumns),
                static_cast<uint32_t>(np));
}

// Sort key of a staged cluster: phi (orderable bits), LHCb id within the module (20 bits:
// sensor in module, chip, column, row), staging slot (12 bits).
__device__ __forceinline__ unsigned long long cluster_key(const float4* src, const uint32_t* src_id, uint32_t i)
{
  return (static_cast<unsigned long long>(orderable(src[i].w)) << 32) |
         (static_cast<unsigned long long>(src_id[i] & 0xFFFFFu) << 12) | i;
}

// Compare-exchange of elements a (lower index) and b in bitonic order `up`: one 64-bit
// comparison and a conditional swap (keys are distinct: the slot is part of the key).
__device__ __forceinline__ void bitonic_cx(unsigned long long& a, unsigned long long& b, bool up)
{
  const bool swap = (b < a) == up;
  const unsigned long long t = a;
  a = swap ? b : a;
  b = swap ? t : b;
}

// Bitonic sort of 32 * PER keys held PER per lane, element lane * PER + j in key[j]
// (the input may sit in any slots: only the sorted order is read back this way). The
// exchanges between elements less than PER apart stay inside a lane, the others take one
// shuffle per key; loops unrolled, so every register index is a compile-time constant and
// the keys stay in registers.
template<uint32_t PER>
__device__ __forceinline__ void warp_register_sort(unsigned long long (&key)[4])
{
  const uint32_t lane = lane_id();
#pragma unroll
  for (uint32_t k = 2; k <= 32 * PER; k <<= 1) {
#pragma unroll
    for (uint32_t d = k >> 1; d > 0; d >>= 1) {
      if (d >= PER) {
        const uint32_t ld = d / PER;  // partner lane distance
        const bool lower = (lane & ld) == 0;
#pragma unroll
        for (uint32_t j = 0; j < PER; ++j) {
          const unsigned long long p = __shfl_xor_sync(0xFFFFFFFFu, key[j], ld);
          const bool up = ((lane * PER + j) & k) == 0;
          // keep the smaller of the pair (lower lane of an ascending pair, or upper lane of a
          // descending one) or the larger
          key[j] = ((p < key[j]) == (lower == up)) ? p : key[j];
        }
      } else if (d == 2) {  // PER == 4: registers j and j + 2
        bitonic_cx(key[0], key[2], ((lane * PER + 0) & k) == 0);
        bitonic_cx(key[1], key[3], ((lane * PER + 1) & k) == 0);
      } else {  // d == 1: registers j and j + 1
        bitonic_cx(key[0], key[1], ((lane * PER + 0) & k) == 0);
        if (PER == 4) bitonic_cx(key[2], key[3], ((lane * PER + 2) & k) == 0);
      }
    }
  }
}

// Bitonic sort of `size` keys (power of two) in shared memory by one warp.
__device__ __forceinline__ void warp_smem_sort(unsigned long long* key, uint32_t size)
{
  const uint32_t lane = lane_id();
  for (uint32_t k = 2; k <= size; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < size; i += 32) {
        const uint32_t ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = key[i], b = key[ixj];
          if ((a > b) == ((i & k) == 0)) {
            key[i] = b;
            key[ixj] = a;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Shared-memory capacity for the event's phi in the windows pass (the union below, free once
// the modules are sorted); larger events search their windows in the cluster records.
constexpr uint32_t kPhiStageCap = (kCandCap * 4 + kBankMapCap + kNonIsoCap * 2) / 4;

// Phi windows of the h1 of one module, after the event's modules are sorted
// (fill_candidates, FillCandidates.cu:8-70, VeloTools.cuh:6-42): for each hit h1 of module m
// (2..49) the hits within kPhiExtrapolation of phi(h1) in module m + 2 (h0) and m - 2 (h2),
// as event-relative u16 pairs {first | last << 16} (0xFFFF: none). `sphi` holds the event's
// phi in hit order (null: read the cluster records). In the pruned mode also the scorer's
// inputs: keep bits (3: seeding candidate, verdict to come; 2: no seed) and, for each
// candidate the gates admit, an 8-byte record (event hit base, h1 | m << 16) appended to the
// candidate list (queue slot 7). One warp per module; every lane takes part in each 32-hit
// round (ballots).
template<bool kPruned>
__device__ __forceinline__ void module_windows(const ChainPointers& P, const float* sphi, const float4* H, uint2* Wn,
                                               uint8_t* K, uint32_t base, uint32_t m, const uint32_t* mstart,
                                               const uint32_t* mcount, bool score)
{
  const uint32_t lane = lane_id();
  const uint32_t s1 = mstart[m], n1 = mcount[m];
  const uint32_t s0 = mstart[m + 2], n0 = mcount[m + 2], s2 = mstart[m - 2], n2 = mcount[m - 2];
  for (uint32_t r0 = 0; r0 < n1; r0 += 32) {
    const uint32_t r = r0 + lane;
    const bool valid = r < n1;
    const uint32_t h = s1 + r;
    int f0 = -1, l0 = -1, f2 = -1, l2 = -1;
    if (valid) {
      if (sphi) {
        const float p = sphi[h];
        if (n0 > 0) phi_window(sphi, s0, n0, p, kPhiExtrapolation, f0, l0);
        if (n2 > 0) phi_window(sphi, s2, n2, p, kPhiExtrapolation, f2, l2);
      } else {
        const float p = H[h].w;
        if (n0 > 0) phi_window4(H, s0, n0, p, kPhiExtrapolation, f0, l0);
        if (n2 > 0) phi_window4(H, s2, n2, p, kPhiExtrapolation, f2, l2);
      }
      Wn[h] = make_uint2((static_cast<uint32_t>(f0) & 0xFFFFu) | (static_cast<uint32_t>(l0) << 16),
                         (static_cast<uint32_t>(f2) & 0xFFFFu) | (static_cast<uint32_t>(l2) << 16));
    }
    if (kPruned) {
      const bool cand = valid && f0 != -1 && f2 != -1;
      if (valid) K[h] = cand ? 3u : 2u;  // candidates: verdict from score_candidates
      // seeds whose pair loop is cheaper than their scoring stay kept, unscored
      const bool append = cand && score && static_cast<uint32_t>((l0 - f0) * (l2 - f2)) >= P.mlp.min_pairs;
      const uint32_t bal = __ballot_sync(0xFFFFFFFFu, append);
      uint32_t row0 = 0;
      if (lane == 0 && bal) row0 = atomicAdd(P.queue + 7, static_cast<uint32_t>(__popc(bal)));
      row0 = __shfl_sync(0xFFFFFFFFu, row0, 0);
      if (append) P.cand_rec[row0 + __popc(bal & ((1u << lane) - 1u))] = make_uint2(base, h | (m << 16));
    }
  }
}

// 40 warps per SM (5 blocks of 8): 48 registers, no spills. kPruned: the windows pass also
// prepares the learned scorer's candidate list.
template<int W, bool kPruned>
__global__ void __launch_bounds__(W * 32, 40 / W) decode_cluster_sort_kernel(ChainPointers P)
{
  __shared__ DecodeShared sh;
  // the candidate list and the per-warp sort buffers are never live together
  __shared__ union {
    struct {
      uint32_t cand[kCandCap];
      uint8_t bank_map[kBankMapCap];  // flat SP index -> bank, saves a binary search per SP
      uint16_t noniso[kNonIsoCap];    // flat SP indices of the non-isolated SPs
    } lists;
    unsigned long long key[W][kSortCap];
  } su;
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  const GeometryView g = geometry_view(P.k.geometry);

  for (;;) {
    if (threadIdx.x == 0) {
      // the event of this pass and its raw bytes, for the whole block
      const uint32_t e = atomicAdd(P.queue + 0, 1u);
      const RunParams& R = *P.run;
      sh.event = e;
      sh.n_events = R.n_events;
      if (e < R.n_events) {
        uint32_t src = e;  // raw event of this position
        uint32_t skipped = 0;
        if (P.event_list) {  // the global event cut of this chain
          if (e < *P.n_selected) src = P.event_list[e];
          else skipped = 1;
        } else if (R.event_list) {  // a selection made by the caller
          src = R.event_list[e];
          if (src >= R.n_raw) skipped = 2;
        }
        sh.skipped = skipped;
        sh.ev_off = skipped ? 0 : raw_offset(R, src);
        sh.ev_bytes = skipped ? 0 : raw_offset(R, src + 1) - sh.ev_off;
      }
      sh.flags = 0;
      sh.n_candidates = 0;
      sh.n_list = 0;
      sh.n_noniso = 0;
    }
    if (threadIdx.x < (kSensors + 31) / 32) sh.unsorted[threadIdx.x] = 0;
    if (threadIdx.x < kModules) sh.mod_count[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t e = sh.event;
    if (e >= sh.n_events) break;
    const uint32_t skipped = sh.skipped;
    const uint64_t off = sh.ev_off;
    const uint64_t bytes = sh.ev_bytes;
    const uint32_t* ev = reinterpret_cast<const uint32_t*>(P.run->raw + off);
    const uint64_t words = bytes / 4;
    const uint32_t header = 2 + kSensors;  // number_of_raw_banks + raw_bank_offset[209]
    // ---- validate the raw event and index its banks ----
    // a batch may start anywhere in the caller's buffer: check the address itself
    const bool bad_header = (reinterpret_cast<uintptr_t>(ev) & 3) || words < header + 1 ||
                            off / 4 + words > P.hit_capacity || __ldg(ev) != kSensors;
    if (!bad_header) {
      const uint64_t payload_bytes = (words - header) * 4;
      for (uint32_t b = threadIdx.x; b < kSensors; b += blockDim.x) {
        const uint32_t o = __ldg(ev + 1 + b), o1 = __ldg(ev + 2 + b);
        bool ok = !(o & 3) && o1 >= o + 8 && o1 <= payload_bytes;
        uint32_t sensor = 0, count = 0;
        if (ok) {
          sensor = __ldg(ev + header + o / 4);
          count = __ldg(ev + header + o / 4 + 1);
          ok = sensor == b && 8ull + 4ull * count <= static_cast<uint64_t>(o1 - o);
        }
        if (!ok) {
          atomicOr(&sh.flags, kStatusBadRawEvent);
          count = 0;
        }
        sh.bank_start[b] = header + o / 4 + 2;
        sh.bank_count[b] = count;
        sh.bank_sensor[b] = sensor;
        if (count > 256) atomicOr(&sh.flags, kStatusBigSpIndex);
      }
    } else if (threadIdx.x == 0) {
      atomicOr(&sh.flags, skipped == 1 ? kStatusNotSelected : kStatusBadRawEvent);
    }
    __syncthreads();
    const bool event_ok = !(sh.flags & (kStatusBadRawEvent | kStatusNotSelected));
    if (!event_ok)
      for (uint32_t b = threadIdx.x; b <= kSensors; b += blockDim.x) sh.sp_prefix[b] = 0;
    // ---- bank prefix (warp 0) ----
    if (event_ok) {
      if (warp == 0) {
        uint32_t carry = 0;
        for (uint32_t b0 = 0; b0 < kSensors; b0 += 32) {
          const uint32_t b = b0 + lane;
          const uint32_t v = b < kSensors ? sh.bank_count[b] : 0;
          uint32_t incl = v;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= static_cast<uint32_t>(o)) incl += t;
          }
          if (b < kSensors) sh.sp_prefix[b] = carry + incl - v;
          carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
        }
        if (lane == 0) sh.sp_prefix[kSensors] = carry;
      }
    }
    __syncthreads();
    const uint32_t total_sp = sh.sp_prefix[kSensors];
    const uint32_t base = static_cast<uint32_t>(off / 4);
    const bool use_map = event_ok && total_sp <= kBankMapCap;  // counts are valid only then
    const DecodeEvent d{ev, 2 * base, P.stage.xyzp, P.stage.id, use_map ? su.lists.bank_map : nullptr};
    // ---- pass 1, one pass over the flat SP index: bank of every SP (map), sortedness of each
    // bank, and the clusters of the isolated SPs from the pattern table (they need neither);
    // the non-isolated SPs are listed for pass 2. Every thread's loads are independent, so
    // the first touches of the raw event overlap instead of queueing bank by bank ----
    const bool can_list = total_sp <= 0x10000u;  // list entries are 16-bit
    if (event_ok) {
      for (uint32_t f = threadIdx.x; f < total_sp; f += blockDim.x) {
        const uint32_t b = bank_of(sh, f);
        if (use_map) su.lists.bank_map[f] = static_cast<uint8_t>(b);
        const uint32_t s = f - sh.sp_prefix[b];
        const uint32_t* bank = ev + sh.bank_start[b];
        const uint32_t word = __ldg(bank + s);
        if (s > 0 && sp_addr(word) < sp_addr(__ldg(bank + s - 1))) atomicOr(&sh.unsorted[b >> 5], 1u << (b & 31));
        if (sp_isolated(word)) {
          // pattern table (MaskedVeloClustering.cu:105-167)
          const uint32_t sp = sp_mask(word);
          const int32_t sp_r = sp_row(word), sp_c = sp_col(word);
          const uint32_t idx = __ldg(P.k.sp_patterns + sp);
          const uint32_t chip = sp_c / (kChipColumns / 2);
          const uint32_t sensor = sh.bank_sensor[b];
          for (int c = 0; c < 2; ++c) {
            if (c == 1 && !(idx & 8)) break;
            const uint32_t row = c ? (idx >> 4) & 3u : idx & 0x03u;
            const uint32_t col = c ? (idx >> 6) & 1u : (idx >> 2) & 1u;
            const uint32_t cx = sp_c * 2 + col;
            const uint32_t cy = sp_r * 4 + row;
            const float fx = __ldg(P.k.sp_fx + sp * 2 + c);
            const float fy = __ldg(P.k.sp_fy + sp * 2 + c);
            stage_cluster(sh, d, b >> 2, place_cluster(g, sensor, cx, cy, fx, fy, chip),
                          (__ldg(P.k.sp_sizes + sp) >> (4 * c)) & 0xFu);
          }
        } else if (can_list) {
          const uint32_t q = atomicAdd(&sh.n_noniso, 1u);
          if (q < kNonIsoCap) su.lists.noniso[q] = static_cast<uint16_t>(f);
        }
      }
    }
    __syncthreads();
    // ---- pass 2: candidate search of the non-isolated SPs (from the list, or every SP when
    // the list overflowed) ----
    uint32_t my_cands = 0;
    const bool listed = can_list && sh.n_noniso <= kNonIsoCap;
    const uint32_t n_scan = listed ? sh.n_noniso : total_sp;
    for (uint32_t i = threadIdx.x; i < n_scan; i += blockDim.x) {
      const uint32_t f = listed ? su.lists.noniso[i] : i;
      const uint32_t b = bank_of_sp(sh, d, f);
      const uint32_t s = f - sh.sp_prefix[b];
      const uint32_t* bank = ev + sh.bank_start[b];
      const uint32_t word = __ldg(bank + s);
      if (sp_isolated(word)) continue;  // emitted in pass 1
      const uint32_t sp = sp_mask(word);
      const int32_t sp_r = sp_row(word), sp_c = sp_col(word);
      const bool sorted = !((sh.unsorted[b >> 5] >> (b & 31)) & 1u);
      const uint32_t code = window_candidate_code(sp, gather_window(bank, sh.bank_count[b], sorted, sp_r, sp_c));
      for (int half = 0; half < 2; ++half) {
        const uint32_t nib = half ? code >> 4 : code & 0xFu;
        if (!nib) continue;
        ++my_cands;
        const uint32_t k = candidate_k(nib) + 2 * half;
        const uint32_t slot = atomicAdd(&sh.n_list, 1u);
        if (slot < kCandCap) su.lists.cand[slot] = (f << 4) | k;
        else flood_candidate(sh, d, g, f, k);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) my_cands += __shfl_xor_sync(0xFFFFFFFFu, my_cands, o);
    if (lane == 0 && my_cands) atomicAdd(&sh.n_candidates, my_cands);
    __syncthreads();
    // ---- pass 3: flood fill of the listed candidates ----
    const uint32_t n_list = min(sh.n_list, kCandCap);
    for (uint32_t i = threadIdx.x; i < n_list; i += blockDim.x) {
      const uint32_t c = su.lists.cand[i];
      flood_candidate(sh, d, g, c >> 4, c & 0xFu);
    }
    __syncthreads();
    // ---- compact layout: exclusive scan of the module counts ----
    if (warp == 0) {
      const uint32_t a = lane < kModules ? sh.mod_count[lane] : 0;
      const uint32_t a2 = lane + 32 < kModules ? sh.mod_count[lane + 32] : 0;
      uint32_t ia = a, ib = a2;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t va = __shfl_up_sync(0xFFFFFFFFu, ia, o), vb = __shfl_up_sync(0xFFFFFFFFu, ib, o);
        if (lane >= static_cast<uint32_t>(o)) {
          ia += va;
          ib += vb;
        }
      }
      const uint32_t first_half = __shfl_sync(0xFFFFFFFFu, ia, 31);
      if (lane < kModules) sh.mod_start[lane] = ia - a;
      if (lane + 32 < kModules) sh.mod_start[lane + 32] = first_half + ib - a2;
      const uint32_t total = first_half + __shfl_sync(0xFFFFFFFFu, ib, 31);
      if (lane == 0) {
        uint32_t fl = 0;
        // the event's hit region is its raw word range: one hit per raw word
        if (total > words) fl |= kStatusHitOverflow;
        if (sh.n_candidates > kMaxCandidatesEvent) fl |= kStatusCandidateOverflow;
        if (fl) atomicOr(&sh.flags, fl);
      }
    }
    __syncthreads();
    const bool write = event_ok && !(sh.flags & kStatusHitOverflow);
    // ---- per-module sort on (phi, LHCb id) into the compact layout ----
    for (uint32_t m = warp; m < kModules; m += W) {
      const uint32_t n = write ? sh.mod_count[m] : 0;
      const uint32_t p0 = base + sh.mod_start[m];
      const float4* src = d.stage + d.stage_base + 2 * sh.sp_prefix[4 * m];
      const uint32_t* src_id = d.stage_id + d.stage_base + 2 * sh.sp_prefix[4 * m];
      float4* dst = P.hits.xyzp + p0;
      uint32_t* dst_id = P.hits.id + p0;
      uint8_t* dst_size = P.hit_size + p0;
      if (n > kMaxHitsPerModule && lane == 0) atomicOr(&sh.flags, kStatusModuleOverflow);
      if (n <= kRegSortMax) {
        const uint32_t per = n > 64 ? 4 : n > 32 ? 2 : 1;
        unsigned long long key[4];
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) {  // coalesced loads; slots j >= per hold padding only
          const uint32_t i = j * 32 + lane;
          key[j] = i < n ? cluster_key(src, src_id, i) : ~0ull;
        }
        if (per == 4) warp_register_sort<4>(key);
        else if (per == 2) warp_register_sort<2>(key);
        else if (n > 1) warp_register_sort<1>(key);
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) {
          const uint32_t i = lane * per + j;  // rank of key[j]
          if (j < per && i < n) {
            const uint32_t from = static_cast<uint32_t>(key[j] & 0xFFFu);
            const uint32_t id = src_id[from];
            dst[i] = src[from];
            dst_id[i] = id & ~kSizeMask;
            dst_size[i] = static_cast<uint8_t>(id >> kSizeShift) & 3u;
          }
        }
      } else if (n <= kSortCap) {
        unsigned long long* key = su.key[warp];
        uint32_t size = 256;
        while (size < n) size <<= 1;
        for (uint32_t i = lane; i < size; i += 32) key[i] = i < n ? cluster_key(src, src_id, i) : ~0ull;
        __syncwarp();
        warp_smem_sort(key, size);
        for (uint32_t i = lane; i < n; i += 32) {
          const uint32_t from = static_cast<uint32_t>(key[i] & 0xFFFu);
          const uint32_t id = src_id[from];
          dst[i] = src[from];
          dst_id[i] = id & ~kSizeMask;
          dst_size[i] = static_cast<uint8_t>(id >> kSizeShift) & 3u;
        }
        __syncwarp();
      } else {
        // beyond the reference's 500-cluster module buffer (flagged above): kept unsorted
        for (uint32_t i = lane; i < n; i += 32) {
          dst[i] = src[i];
          dst_id[i] = src_id[i] & ~kSizeMask;
          dst_size[i] = static_cast<uint8_t>(src_id[i] >> kSizeShift) & 3u;
        }
      }
      if (lane == 0) {
        P.module_start[e * kModules + m] = p0;
        P.module_num[e * kModules + m] = n;
      }
    }
    __syncthreads();
    // ---- phi windows of every h1 (fill_candidates), while the event is in L2: the sorted phi
    // are read back into the shared memory the lists and sort buffers no longer need ----
    {
      const uint32_t nh = write ? sh.mod_start[kModules - 1] + sh.mod_count[kModules - 1] : 0;
      if (nh > 0 && nh <= kEventHitCap) {  // the events the search runs
        const float4* H = P.hits.xyzp + base;
        float* sphi = nh <= kPhiStageCap ? reinterpret_cast<float*>(&su) : nullptr;
        if (sphi)
          for (uint32_t i = threadIdx.x; i < nh; i += blockDim.x) sphi[i] = H[i].w;
        __syncthreads();
        bool score = false;
        uint8_t* K = nullptr;
        if (kPruned) {
          K = P.keep + base;
          const bool fallback = nh > P.mlp.max_hits;  // above the trained occupancy: plain search
          if (fallback && threadIdx.x == 0) sh.flags |= kStatusMlpFallback;
          score = !fallback && nh >= P.mlp.min_hits;
          if (score) {
            // modules 0, 1, 50, 51 hold no h1: extension candidates only
            for (uint32_t h = threadIdx.x; h < sh.mod_start[2]; h += blockDim.x) K[h] = 2;
            for (uint32_t h = sh.mod_start[50] + threadIdx.x; h < nh; h += blockDim.x) K[h] = 2;
          } else {
            // an event the scorer does not score: every seed kept, its windows as in the
            // plain mode (the branch is uniform over the block)
            for (uint32_t h = threadIdx.x; h < nh; h += blockDim.x) K[h] = 3;
          }
        }
        bool scored = false;
        if constexpr (kPruned) {
          if (score) {
            for (uint32_t m = 2 + warp; m < 50; m += W)
              module_windows<true>(P, sphi, H, P.windows + base, K, base, m, sh.mod_start, sh.mod_count, true);
            scored = true;
          }
        }
        if (!scored)
          for (uint32_t m = 2 + warp; m < 50; m += W)
            module_windows<false>(P, sphi, H, P.windows + base, K, base, m, sh.mod_start, sh.mod_count, false);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t nhits = write ? sh.mod_start[kModules - 1] + sh.mod_count[kModules - 1] : 0;
      P.event_hit_base[e] = base;
      P.event_hits[e] = nhits;
      P.status[e] = sh.flags;
      // route the event to the search mapping chosen for its size
      if (nhits > P.block_threshold) P.block_events[atomicAdd(P.queue + 5, 1u)] = e;
      else P.warp_events[atomicAdd(P.queue + 4, 1u)] = e;
    }
    __syncthreads();
  }
}

}  // namespace velo
