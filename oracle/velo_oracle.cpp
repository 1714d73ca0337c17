// ORACLE — test infrastructure only. CPU restatement of the reference VELO chain
// (Qwicen/cuda_hlt "Allen", cuda/velo), used as the checker of the CUDA chain by tests/,
// by __graft_entry__.smoke() and as the CPU baseline leg of bench.py. Never part of the
// product path.
//
// Each stage follows the reference kernel statement by statement, with the threads of a
// block serialised in lane order:
//   estimate_input_size      cuda/velo/mask_clustering/src/EstimateInputSize.cu:3-255
//   masked_velo_clustering   cuda/velo/mask_clustering/src/MaskedVeloClustering.cu:4-464
//   calculate_phi_and_sort   cuda/velo/calculate_phi_and_sort/src/CalculatePhi.cu:10-104,
//                            SortByPhi.cu:8-34, cuda/velo/common/src/VeloTools.cu:3-10
//   fill_candidates          cuda/velo/search_by_triplet/src/FillCandidates.cu:8-70
//   binary searches          cuda/velo/common/include/VeloTools.cuh:6-42
//   search_by_triplet        cuda/velo/search_by_triplet/src/SearchByTriplet.cu:7-111,
//                            ProcessModules.cu:8-163, TrackSeeding.cu:7-200,
//                            TrackForwarding.cu:12-182, TrackForwarding.cuh:28-59
//   weak_tracks_adder        cuda/velo/search_by_triplet/src/WeakTracksAdder.cu:9-115
//   consolidate_velo_tracks  cuda/velo/consolidate_tracks/src/ConsolidateVelo.cu:6-170
//   velo_kalman_fit          cuda/velo/simplified_kalman_filter/src/VeloKalmanFilter.cu:6-73,
//                            include/VeloKalmanFilter.cuh:27-93
// with the constants of cuda/velo/common/include/VeloDefinitions.cuh:7-77 and
// stream/sequence/src/Constants.cu:27-53.
//
// Arithmetic is IEEE fp32 in the reference's operation order, compiled without FMA
// contraction; the reference runs on the GPU with --use_fast_math (approximate division,
// device atan2f), so float fields agree to a few ulp, not bit for bit. Bit-exact parity is
// pinned by running the reference's own kernels (oracle/_ref). An FP64 twin of the two
// track fits gives the residuals of the fp32 states.
//
// Cluster layout: compact per event (module order, no estimate gaps); within a module the
// order is the reference's stable phi sort. Hit indices are event-relative.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t NM = 52, NS = 208;
constexpr uint32_t MAX_CAND = 3000, MAX_TRACKS = 1200, TTF_MOD = 2000, MAX_WEAK = 500, MAX_MOD_HITS = 500;
constexpr float PHI_EXTRAP = 0.062f, FWD_PHI_TOL = 0.052f, MAX_SLOPE = 0.4f, TOL = 0.6f;
constexpr float MAX_SCATTER_SEED = 0.004f, MAX_SCATTER_FWD = 0.004f, PARAM_W = 3966.94f,
                PARAM_W_INV = 0.000252083f, MAX_CHI2 = 20.0f;
constexpr float PIXEL_SIZE = 0.055f;
constexpr float PI_F = 3.141592654f;
const uint8_t CAND_KS[9] = {0, 0, 1, 4, 4, 5, 5, 5, 5};
const float MODULE_Z[NM] = {
  -287.5f, -275.f, -262.5f, -250.f, -237.5f, -225.f, -212.5f, -200.f, -137.5f, -125.f, -62.5f, -50.f, -37.5f,
  -25.f,   -12.5f, 0.f,     12.5f,  25.f,    37.5f,  50.f,    62.5f,  75.f,    87.5f,  100.f,  112.5f, 125.f,
  137.5f,  150.f,  162.5f,  175.f,  187.5f,  200.f,  212.5f,  225.f,  237.5f,  250.f,  262.5f, 275.f,  312.5f,
  325.f,   387.5f, 400.f,   487.5f, 500.f,   587.5f, 600.f,   637.5f, 650.f,   687.5f, 700.f,  737.5f, 750.f};

enum : uint32_t {
  F_BAD_RAW = 1u << 0,
  F_MODULE_OVF = 1u << 1,
  F_HIT_OVF = 1u << 2,
  F_CAND_OVF = 1u << 3,
  F_TRACK_OVF = 1u << 4,
  F_TTF_OVF = 1u << 5,
  F_WEAK_OVF = 1u << 6,
  F_H1_OVF = 1u << 7,
  F_BIG_SP = 1u << 8,
  F_SEED_TIE = 1u << 16,         // equal scatter between two seeding candidates of one h1
  F_EMPTY_MODULE_READ = 1u << 17 // forwarding into an empty module (reference reads outside it)
};

struct Luts {
  uint8_t pat[256];
  float fx[512], fy[512];
};

// Same table as x86/velo/clustering/src/ClusteringCommon.cpp:3-101 (8-way flood fill).
void build_luts(Luts& L)
{
  const int dx[] = {-1, 0, 1, -1, 0, 1, -1, 1};
  const int dy[] = {-1, -1, -1, 1, 1, 1, 0, 0};
  for (unsigned sp = 0; sp < 256; ++sp) {
    L.pat[sp] = 0;
    L.fx[2 * sp] = L.fx[2 * sp + 1] = L.fy[2 * sp] = L.fy[2 * sp + 1] = 0.f;
    unsigned char buf[8], idx[8], n_idx = 0;
    for (unsigned s = 0; s < 8; ++s) {
      buf[s] = sp & (1u << s);
      if (buf[s]) idx[n_idx++] = s;
    }
    unsigned char clu = 0;
    for (unsigned ip = 0; ip < n_idx; ++ip) {
      unsigned char i0 = idx[ip];
      if (!buf[i0]) continue;
      unsigned char stack[8], sptr = 0;
      stack[sptr++] = i0;
      buf[i0] = 0;
      unsigned char x = 0, y = 0, n = 0;
      while (sptr) {
        const unsigned char id = stack[--sptr];
        const int row = id % 4, col = id / 4;
        x += col;
        y += row;
        ++n;
        for (int k = 0; k < 8; ++k) {
          const int nc = col + dx[k], nr = row + dy[k];
          if (nc < 0 || nc > 1 || nr < 0 || nr > 3) continue;
          const unsigned char ni = (nc << 2) | nr;
          if (!buf[ni]) continue;
          stack[sptr++] = ni;
          buf[ni] = 0;
        }
      }
      const uint32_t cx = x / n, cy = y / n;
      L.pat[sp] |= ((cx << 2) | cy) << 4 * clu;
      L.pat[sp] |= clu << 3;
      L.fx[2 * sp + clu] = x / static_cast<float>(n) - cx;
      L.fy[2 * sp + clu] = y / static_cast<float>(n) - cy;
      ++clu;
    }
  }
}

struct Geo {
  const float* local_x;
  const float* x_pitch;
  const float* ltg;
};

struct Hit {
  float x, y, z, phi;
  uint32_t id;
};

struct TrackHits {
  uint16_t n;
  uint16_t h[26];
};

struct State {
  float x, y, tx, ty, c00, c20, c22, c11, c31, c33, chi2, z;
  bool backward;
};
struct State64 {
  double x, y, tx, ty, c00, c20, c22, c11, c31, c33, chi2, z;
  bool backward;
};

struct EventOut {
  uint32_t flags = 0;
  uint32_t module_num[NM] = {};
  std::vector<Hit> hits;  // compact, module order, phi-sorted within module
  uint32_t module_start[NM + 1] = {};
  std::vector<TrackHits> tracks;
  std::vector<State> lsq, kal;
  std::vector<State64> lsq64, kal64;
  uint32_t n_candidates = 0, n_weak = 0, n_tracklets = 0;
};

uint32_t channel_id(uint32_t sensor, uint32_t chip, uint32_t col, uint32_t row)
{
  return (sensor << 18) | (chip << 16) | (col << 8) | row;
}
uint32_t lhcb_id(uint32_t cid) { return (8u << 28) + cid; }

// ---- masks of MaskedVeloClustering.cu:4-46 ----
uint32_t current_mask(uint32_t p)
{
  return ((p & 0xFFFF7FFFu) << 1) | ((p & 0xFFFEFFFFu) >> 1) | ((p & 0xFFFEFFFEu) << 15) | ((p & 0x7FFF7FFFu) >> 15) |
         (p >> 16) | (p >> 17) | (p << 16) | (p << 17);
}
uint32_t mask_ltr(uint32_t p) { return ((p & 0x7FFF0000u) >> 15) | (p >> 16) | (p >> 17); }
uint32_t mask_rtl(uint32_t p) { return ((p & 0x0000FFFEu) << 15) | (p << 16) | (p << 17); }
uint32_t cluster_current_mask(uint32_t p)
{
  return ((p & 0xFFFF7FFFu) << 1) | ((p & 0xFFFEFFFEu) << 15) | (p << 16) | (p << 17);
}
uint32_t cand_mask_right(uint32_t p, uint32_t rp)
{
  return ((p & 0xFFFEFFFFu) >> 1) & (((p & 0x7FFF7FFFu) >> 15) | (rp << 17)) & ((p >> 16) | (rp << 16)) &
         ((p >> 17) | ((rp & 0x0000FFFEu) << 15));
}

struct RawView {
  uint32_t nb;
  const uint32_t* offs;
  const uint8_t* payload;
  uint32_t sensor(uint32_t b) const { return reinterpret_cast<const uint32_t*>(payload + offs[b])[0]; }
  uint32_t count(uint32_t b) const { return reinterpret_cast<const uint32_t*>(payload + offs[b])[1]; }
  const uint32_t* words(uint32_t b) const { return reinterpret_cast<const uint32_t*>(payload + offs[b]) + 2; }
};

bool validate(const uint8_t* ev, uint64_t bytes)
{
  if (bytes < 4) return false;
  uint32_t nb;
  std::memcpy(&nb, ev, 4);
  if (nb != NS || bytes < 4ull * (nb + 2)) return false;
  const uint32_t* offs = reinterpret_cast<const uint32_t*>(ev + 4);
  const uint64_t payload = bytes - 4ull * (nb + 2);
  for (uint32_t b = 0; b < nb; ++b) {
    const uint64_t o = offs[b], e = offs[b + 1];
    if ((o & 3) || e < o + 8 || e > payload) return false;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(ev + 4ull * (nb + 2) + o);
    if (w[0] != b || 8ull + 4ull * w[1] > e - o) return false;
  }
  return true;
}

// atan2 conventions of cuda/velo/common/src/VeloTools.cu:3-10
float phi_odd(float x, float y) { return std::atan2(y, x); }
float phi_even(float x, float y)
{
  const float phi = std::atan2(y, x);
  const bool neg = phi < 0.f;
  return phi + neg * 2 * PI_F;
}

// cuda/velo/common/include/VeloTools.cuh:6-24
int bsearch_first(const float* a, uint32_t size, float value, float margin)
{
  bool found = false;
  int l = 0, r = static_cast<int>(size) - 1;
  while (l < r) {
    const int m = (l + r) / 2;
    const float e = a[m];
    found |= std::fabs(value - e) < margin;
    if (value - margin > e) l = m + 1; else r = m;
  }
  found |= std::fabs(value - a[l]) < margin;
  return found ? l : -1;
}
// cuda/velo/common/include/VeloTools.cuh:26-42
int bsearch_second(const float* a, uint32_t size, float value, float margin)
{
  int l = 0, r = static_cast<int>(size) - 1;
  while (l < r) {
    const int m = (l + r) / 2;
    if (value + margin > a[m]) l = m + 1; else r = m;
  }
  const bool last_compatible = std::fabs(value - a[l]) < margin;
  return last_compatible ? l + 1 : l;
}

// ============================================================================
// Clustering: estimate_input_size + masked_velo_clustering for one event.
// Fills per-module cluster lists in slot order (the order the atomics hand out slots
// when threads are serialised).
// ============================================================================
void cluster_event(const RawView& ev, const Geo& g, const Luts& L, std::vector<Hit> (&mod)[NM], uint32_t& flags,
                   uint32_t& n_cand_out)
{
  // ---- estimate_input_size: candidates (EstimateInputSize.cu:40-253) ----
  std::vector<uint32_t> cands;
  uint32_t est[NM] = {};
  for (uint32_t b = 0; b < ev.nb; ++b) {
    const uint32_t sensor = ev.sensor(b), cnt = ev.count(b);
    const uint32_t* w = ev.words(b);
    if (cnt > 256) flags |= F_BIG_SP;
    for (uint32_t s = 0; s < cnt; ++s) {
      const uint32_t word = w[s];
      const uint32_t iso = word & 0x80000000u;
      const uint32_t addr = (word & 0x007FFF00u) >> 8;
      const uint8_t sp = word & 0xFFu;
      if (iso) {
        const bool p0 = (sp & 0x88) && !(sp & 0x44) && (sp & 0x33);
        const bool p1 = (sp & 0xCC) && !(sp & 0x22) && (sp & 0x11);
        est[(sensor >> 2) % NM] += 1 + (p0 | p1);
      } else {
        uint32_t pixels = (sp & 0x0F) | ((sp & 0xF0) << 2);
        const uint32_t row = addr & 0x3Fu, col = addr >> 6;
        for (uint32_t k = 0; k < cnt; ++k) {
          const uint32_t ow = w[k];
          // The reference tests the isolation bit of the current word here
          // (EstimateInputSize.cu:126), so every word of the bank is scanned.
          const uint32_t other_iso = word & 0x80000000u;
          if (other_iso) continue;
          const uint32_t oaddr = (ow & 0x007FFF00u) >> 8;
          const uint32_t orow = oaddr & 0x3Fu, ocol = oaddr >> 6;
          const uint8_t osp = ow & 0xFFu;
          const bool top = orow == row + 1 && ocol == col;
          const bool top_right = orow == row + 1 && ocol == col + 1;
          const bool right = orow == row && ocol == col + 1;
          const bool right_bottom = orow == row - 1 && ocol == col + 1;
          const bool bottom = orow == row - 1 && ocol == col;
          if (top || top_right || right || right_bottom || bottom) {
            pixels |= top * (((osp & 0x01) | ((osp & 0x10) << 2)) << 4);
            pixels |= top_right * ((osp & 0x01) << 16);
            pixels |= right * ((osp & 0x0F) << 12);
            pixels |= right_bottom * ((osp & 0x08) << 8);
            pixels |= bottom * ((osp & 0x80) >> 2);
          }
        }
        const uint32_t inside = pixels & 0x3CF;
        const uint32_t mask = (inside << 1) | (inside << 5) | (inside << 6) | (inside << 7);
        const uint32_t wc = mask & (~pixels);
        const uint32_t ct = (wc >> 1) & (wc >> 5) & (wc >> 6) & (wc >> 7);
        const uint32_t c = ct & pixels;
        const uint8_t c8 = (c & 0x03) | ((c & 0xC0) >> 4) | ((c & 0x0C) << 2) | ((c & 0x0300) >> 2);
        uint32_t found = 0;
        if (c8 & 0xF) {
          const uint8_t k = CAND_KS[c8 & 0xF];
          cands.push_back((s << 11) | (b << 3) | k);
          ++found;
        }
        if (c8 & 0xF0) {
          const uint8_t k = CAND_KS[c8 >> 4] + 2;
          cands.push_back((s << 11) | (b << 3) | k);
          ++found;
        }
        est[(sensor >> 2) % NM] += found;
      }
    }
  }
  n_cand_out = static_cast<uint32_t>(cands.size());
  if (cands.size() > MAX_CAND) flags |= F_CAND_OVF;

  auto store = [&](uint32_t module, const float* ltg, float local_x, float local_y, uint32_t cid) {
    Hit h;
    h.x = ltg[0] * local_x + ltg[1] * local_y + ltg[9];
    h.y = ltg[3] * local_x + ltg[4] * local_y + ltg[10];
    h.z = ltg[6] * local_x + ltg[7] * local_y + ltg[11];
    h.phi = 0.f;
    h.id = lhcb_id(cid);
    mod[module].push_back(h);
  };

  // ---- masked_velo_clustering phase 1: isolated SPs (MaskedVeloClustering.cu:88-170) ----
  for (uint32_t b = 0; b < ev.nb; ++b) {
    const uint32_t module = b >> 2;
    const uint32_t sensor = ev.sensor(b), cnt = ev.count(b);
    const uint32_t* w = ev.words(b);
    const float* ltg = g.ltg + 16 * sensor;
    for (uint32_t s = 0; s < cnt; ++s) {
      const uint32_t word = w[s];
      if (!(word & 0x80000000u)) continue;
      const uint32_t addr = (word & 0x007FFF00u) >> 8;
      const int32_t sp_row = addr & 0x3Fu, sp_col = addr >> 6;
      const uint8_t sp = word & 0xFFu;
      const uint32_t idx = L.pat[sp];
      const uint32_t chip = sp_col / (256 / 2);
      for (int second = 0; second < 2; ++second) {
        if (second && !(idx & 8)) break;
        const uint32_t row = second ? (idx >> 4) & 3 : idx & 0x03u;
        const uint32_t col = second ? (idx >> 6) & 1 : (idx >> 2) & 1;
        const uint32_t cx = sp_col * 2 + col, cy = sp_row * 4 + row;
        const uint32_t cid = channel_id(sensor, chip, cx % 256, cy);
        const float fx = L.fx[sp * 2 + second], fy = L.fy[sp * 2 + second];
        const float local_x = g.local_x[cx] + fx * g.x_pitch[cx];
        const float local_y = (cy + 0.5 + fy) * PIXEL_SIZE;
        store(module, ltg, local_x, local_y, cid);
      }
    }
  }

  // ---- phase 2: candidates (MaskedVeloClustering.cu:175-462) ----
  for (uint32_t candidate : cands) {
    const uint8_t sp_index = candidate >> 11;  // u8: wraps for banks above 255 SPs
    const uint8_t bank = (candidate >> 3) & 0xFF;
    const uint32_t module = bank >> 2;
    const uint8_t k = candidate & 0x7;
    const uint32_t sensor = ev.sensor(bank), cnt = ev.count(bank);
    const uint32_t* w = ev.words(bank);
    const float* ltg = g.ltg + 16 * sensor;
    const uint32_t word = w[sp_index];
    const uint32_t addr = (word & 0x007FFF00u) >> 8;
    const int32_t sp_row = addr & 0x3Fu, sp_col = addr >> 6;
    uint32_t pa[3] = {0, 0, 0};
    const int32_t rlo = sp_row - 2, rhi = sp_row + 1, clo = sp_col - 1, chi = sp_col + 1;
    const int32_t row_lower_limit = rlo * 4, col_lower_limit = clo * 2;
    for (uint32_t j = 0; j < cnt; ++j) {
      const uint32_t ow = w[j];
      if (ow & 0x80000000u) continue;
      const uint32_t oaddr = (ow & 0x007FFF00u) >> 8;
      const int32_t orow = oaddr & 0x3Fu, ocol = oaddr >> 6;
      const uint8_t osp = ow & 0xFFu;
      if (orow >= rlo && orow <= rhi && ocol >= clo && ocol <= chi) {
        const int rr = orow - rlo, rc = ocol - clo;
        pa[rc] |= (osp & 0x0F) << (4 * rr) | (osp & 0xF0) << (12 + 4 * rr);
      }
    }
    const uint32_t row = sp_row * 4 + (k % 4);
    const uint32_t col = sp_col * 2 + (k >= 4);
    uint32_t cl[3] = {0, (uint32_t)((0x01 << (row - row_lower_limit)) << (16 * (col % 2))), 0};
    uint32_t wc[3] = {0, cl[1], 0};
    pa[1] &= ~cl[1];
    for (uint32_t it = 0; it < 12; ++it) {
      uint32_t pm[3];
      pm[0] = current_mask(wc[0]) | mask_rtl(wc[1]);
      pm[1] = current_mask(wc[1]) | mask_rtl(wc[2]) | mask_ltr(wc[0]);
      pm[2] = current_mask(wc[2]) | mask_ltr(wc[1]);
      wc[0] = pa[0] & pm[0];
      wc[1] = pa[1] & pm[1];
      wc[2] = pa[2] & pm[2];
      if (!wc[0] && !wc[1] && !wc[2]) break;
      cl[0] |= wc[0];
      cl[1] |= wc[1];
      cl[2] |= wc[2];
      pa[0] &= ~cl[0];
      pa[1] &= ~cl[1];
      pa[2] &= ~cl[2];
    }
    if (cl[2]) continue;
    const int n = __builtin_popcount(cl[0]) + __builtin_popcount(cl[1]);
    bool do_store = true;
    if (n >= 3) {
      uint32_t pm[3];
      pm[0] = cluster_current_mask(cl[0]);
      pm[1] = cluster_current_mask(cl[1]) | mask_ltr(cl[0]);
      pm[2] = mask_ltr(cl[1]);
      wc[0] = pm[0] & (~cl[0]);
      wc[1] = pm[1] & (~cl[1]);
      wc[2] = pm[2];
      uint32_t cnd[2];
      cnd[0] = cand_mask_right(wc[0], wc[1]) & cl[0];
      cnd[1] = cand_mask_right(wc[1], wc[2]) & cl[1];
      const uint32_t working_candidate = (0x01 << (row - row_lower_limit)) << (16 * (col % 2));
      cnd[1] ^= working_candidate;
      if (cnd[0] || cnd[1]) {
        const int32_t neg = ~(-static_cast<int32_t>(working_candidate));
        const bool under = working_candidate < 4096;
        uint32_t srm = under * (0xFFF & neg) | (!under) * (0xFFF & (neg >> 16));
        srm |= srm << 16;
        const uint32_t cpm = srm | under * 0xFFFF0000u;
        do_store = ((cnd[0] & srm) | (cnd[1] & cpm)) == 0;
      }
    }
    if (!do_store) continue;
    const int x = __builtin_popcount(cl[0] & 0x0000FFFF) * col_lower_limit +
                  __builtin_popcount(cl[0] & 0xFFFF0000) * (col_lower_limit + 1) +
                  __builtin_popcount(cl[1] & 0x0000FFFF) * (col_lower_limit + 2) +
                  __builtin_popcount(cl[1] & 0xFFFF0000) * (col_lower_limit + 3);
    const uint32_t tr[4] = {(cl[0] & 0x000F000F) | ((cl[1] & 0x000F000F) << 4),
                            ((cl[0] & 0x00F000F0) >> 4) | (cl[1] & 0x00F000F0),
                            ((cl[0] & 0x0F000F00) >> 8) | ((cl[1] & 0x0F000F00) >> 4),
                            ((cl[0] & 0xF000F000) >> 12) | ((cl[1] & 0xF000F000) >> 8)};
    int y = 0;
    for (int q = 0; q < 4; ++q)
      for (int r4 = 0; r4 < 4; ++r4)
        y += __builtin_popcount(tr[q] & (0x11111111u << r4)) * (row_lower_limit + 4 * q + r4);
    const uint32_t cx = x / n, cy = y / n;
    const float fx = x / static_cast<float>(n) - cx;
    const float fy = y / static_cast<float>(n) - cy;
    const uint32_t chip = cx / 256;
    const uint32_t cid = channel_id(sensor, chip, cx % 256, cy);
    const float local_x = g.local_x[cx] + fx * g.x_pitch[cx];
    const float local_y = (cy + 0.5 + fy) * PIXEL_SIZE;
    store(module, ltg, local_x, local_y, cid);
  }
}

// ============================================================================
// Track fits.
// ============================================================================
template<class F, class S>
S lsq_fit(const std::vector<Hit>& hits, const TrackHits& t)
{
  // ConsolidateVelo.cu:6-114 (means_square_fit); F = float or double
  S st{};
  F s0 = 0, sx = 0, sz = 0, sxz = 0, sz2 = 0, u0 = 0, uy = 0, uz = 0, uyz = 0, uz2 = 0;
  for (int h = 0; h < t.n; ++h) {
    const Hit& hit = hits[t.h[h]];
    const F x = hit.x, y = hit.y, z = hit.z;
    const F w = static_cast<F>(PARAM_W);
    const F wxx = w * x, wxz = w * z;
    s0 += w;
    sx += wxx;
    sz += wxz;
    sxz += wxx * z;
    sz2 += wxz * z;
    const F wyy = w * y, wyz = w * z;
    u0 += w;
    uy += wyy;
    uz += wyz;
    uyz += wyy * z;
    uz2 += wyz * z;
  }
  const F dens = F(1) / (sz2 * s0 - sz * sz);
  st.tx = (sxz * s0 - sx * sz) * dens;
  st.x = (sx * sz2 - sxz * sz) * dens;
  const F denu = F(1) / (uz2 * u0 - uz * uz);
  st.ty = (uyz * u0 - uy * uz) * denu;
  st.y = (uy * uz2 - uyz * uz) * denu;
  st.z = -(st.x * st.tx + st.y * st.ty) / (st.tx * st.tx + st.ty * st.ty);
  st.backward = st.z > static_cast<F>(hits[t.h[0]].z);
  const F m00 = s0, m11 = u0;
  const F m20 = sz - st.z * s0, m31 = uz - st.z * u0;
  const F m22 = sz2 - 2 * st.z * sz + st.z * st.z * s0;
  const F m33 = uz2 - 2 * st.z * uz + st.z * st.z * u0;
  const F den20 = F(1) / (m22 * m00 - m20 * m20);
  const F den31 = F(1) / (m33 * m11 - m31 * m31);
  st.c00 = m22 * den20;
  st.c20 = -m20 * den20;
  st.c22 = m00 * den20;
  st.c11 = m33 * den31;
  st.c31 = -m31 * den31;
  st.c33 = m11 * den31;
  F ch = 0;
  int ndof = -4;
  for (int h = 0; h < t.n; ++h) {
    const Hit& hit = hits[t.h[h]];
    const F z = hit.z;
    const F x = st.x + st.tx * z;
    const F y = st.y + st.ty * z;
    const F dx = x - F(hit.x), dy = y - F(hit.y);
    ch += dx * dx * F(PARAM_W) + dy * dy * F(PARAM_W);
    ndof += 2;
  }
  st.chi2 = ch / ndof;
  st.x = st.x + st.tx * st.z;
  st.y = st.y + st.ty * st.z;
  return st;
}

template<class F>
F kf_step(F z, F zhit, F xhit, F whit, F& x, F& tx, F& cxx, F& cxt, F& ctt)
{
  // VeloKalmanFilter.cu:6-41
  const F dz = zhit - z;
  const F predx = x + dz * tx;
  const F dz_t_ctt = dz * ctt;
  const F predcxt = cxt + dz_t_ctt;
  const F dx_t_cxt = dz * cxt;
  const F predcxx = cxx + 2 * dx_t_cxt + dz * dz_t_ctt;
  const F predctt = ctt;
  const F R = F(1) / ((F(1) / whit) + predcxx);
  const F Kx = predcxx * R;
  const F KTx = predcxt * R;
  const F r = xhit - predx;
  x = predx + Kx * r;
  tx = tx + KTx * r;
  cxx = (1 - Kx) * predcxx;
  cxt = (1 - Kx) * predcxt;
  ctt = predctt - KTx * predcxt;
  return r * r * R;
}

template<class F, class S>
S kalman_fit(const std::vector<Hit>& hits, const TrackHits& t, const S& beam)
{
  // VeloKalmanFilter.cuh:27-93, simplified_fit<true>
  const uint32_t n = t.n;
  auto H = [&](int i) -> const Hit& { return hits[t.h[i]]; };
  const bool backward = beam.z > static_cast<decltype(beam.z)>(H(0).z);
  const int direction = backward ? 1 : -1;
  const F noise = static_cast<F>(1e-8 + 7e-6 * (beam.tx * beam.tx + beam.ty * beam.ty));
  int first = 0, last = static_cast<int>(n) - 1, d = 1;
  if ((H(last).z - H(first).z) * direction < 0) {
    std::swap(first, last);
    d = -1;
  }
  S st{};
  st.x = H(first).x;
  st.y = H(first).y;
  st.z = H(first).z;
  st.tx = beam.tx;
  st.ty = beam.ty;
  st.c00 = static_cast<F>(PARAM_W_INV);
  st.c11 = static_cast<F>(PARAM_W_INV);
  st.c20 = 0;
  st.c31 = 0;
  st.c22 = 1;
  st.c33 = 1;
  st.chi2 = 0;
  for (int i = first + d; i != last + d; i += d) {
    const F hx = H(i).x, hy = H(i).y, hz = H(i).z;
    st.c22 += noise;
    st.c33 += noise;
    st.chi2 += kf_step<F>(st.z, hz, hx, F(PARAM_W), st.x, st.tx, st.c00, st.c20, st.c22);
    st.chi2 += kf_step<F>(st.z, hz, hy, F(PARAM_W), st.y, st.ty, st.c11, st.c31, st.c33);
    st.z = hz;
  }
  st.c22 += noise;
  st.c33 += noise;
  st.backward = backward;  // the reference leaves this field unset
  return st;
}

float weak_chi2(const std::vector<Hit>& hits, const uint16_t h[3])
{
  // WeakTracksAdder.cu:9-86
  float s0 = 0, sx = 0, sz = 0, sxz = 0, sz2 = 0, u0 = 0, uy = 0, uz = 0, uyz = 0, uz2 = 0;
  for (int k = 0; k < 3; ++k) {
    const Hit& hit = hits[h[k]];
    const float w = PARAM_W;
    const float wxx = w * hit.x, wxz = w * hit.z;
    s0 += w;
    sx += wxx;
    sz += wxz;
    sxz += wxx * hit.z;
    sz2 += wxz * hit.z;
    const float wyy = w * hit.y, wyz = w * hit.z;
    u0 += w;
    uy += wyy;
    uz += wyz;
    uyz += wyy * hit.z;
    uz2 += wyz * hit.z;
  }
  const float dens = 1.0f / (sz2 * s0 - sz * sz);
  const float tx = (sxz * s0 - sx * sz) * dens;
  const float x0 = (sx * sz2 - sxz * sz) * dens;
  const float denu = 1.0f / (uz2 * u0 - uz * uz);
  const float ty = (uyz * u0 - uy * uz) * denu;
  const float y0 = (uy * uz2 - uyz * uz) * denu;
  float ch = 0;
  int ndof = -4;
  for (int k = 0; k < 3; ++k) {
    const Hit& hit = hits[h[k]];
    const float x = x0 + tx * hit.z, y = y0 + ty * hit.z;
    const float dx = x - hit.x, dy = y - hit.y;
    ch += dx * dx * PARAM_W + dy * dy * PARAM_W;
    ndof += 2;
  }
  return ch / ndof;
}

// ============================================================================
// search_by_triplet for one event (one warp of 32 lanes, serialised in lane order).
// ============================================================================
struct ModuleData {
  uint32_t start, num;
  float z;
};

void search_event(EventOut& out)
{
  const auto& hits = out.hits;
  const uint32_t H = static_cast<uint32_t>(hits.size());
  std::vector<float> phis(H + 1, 0.f);
  for (uint32_t i = 0; i < H; ++i) phis[i] = hits[i].phi;
  // fill_candidates (FillCandidates.cu:8-70): windows for h1 in modules 2..49
  std::vector<int> h0c(2 * H, -1), h2c(2 * H, -1);
  for (uint32_t m = 2; m < 50; ++m) {
    const uint32_t m0s = out.module_start[m + 2], m2s = out.module_start[m - 2];
    const uint32_t m0n = out.module_num[m + 2], m2n = out.module_num[m - 2];
    for (uint32_t r = 0; r < out.module_num[m]; ++r) {
      const uint32_t h1 = out.module_start[m] + r;
      const float p = phis[h1];
      int f0 = -1, l0 = -1;
      if (m0n > 0) {
        f0 = bsearch_first(&phis[m0s], m0n, p, PHI_EXTRAP);
        if (f0 != -1) {
          l0 = bsearch_second(&phis[m0s + f0], m0n - f0, p, PHI_EXTRAP);
          f0 += m0s;
          l0 = l0 == 0 ? f0 + 1 : f0 + l0;
        }
      }
      h0c[2 * h1] = f0;
      h0c[2 * h1 + 1] = l0;
      int f2 = -1, l2 = -1;
      if (m2n > 0) {
        f2 = bsearch_first(&phis[m2s], m2n, p, PHI_EXTRAP);
        if (f2 != -1) {
          l2 = bsearch_second(&phis[m2s + f2], m2n - f2, p, PHI_EXTRAP);
          f2 += m2s;
          l2 = l2 == 0 ? f2 + 1 : f2 + l2;
        }
      }
      h2c[2 * h1] = f2;
      h2c[2 * h1 + 1] = l2;
    }
  }

  std::vector<uint8_t> used(H, 0);
  std::vector<TrackHits>& tracks = out.tracks;
  tracks.clear();
  std::vector<TrackHits> track_slots(MAX_TRACKS + 64);
  uint32_t n_tracks = 0;
  std::vector<uint16_t> tracklets(3 * TTF_MOD);
  std::vector<uint32_t> ttf(TTF_MOD);
  std::vector<uint16_t> weak;  // unbounded here; the reference holds MAX_WEAK per event
  uint32_t weak_ptr = 0, tracklet_ptr = 0, ttf_ptr = 0;
  ModuleData md[6];
  auto load = [&](uint32_t first) {
    for (int i = 0; i < 6; ++i) {
      const uint32_t m = first - i;
      md[i] = {out.module_start[m], out.module_num[m], MODULE_Z[m]};
    }
  };
  std::vector<uint16_t> h1_list;

  auto seeding = [&]() {
    // TrackSeeding.cu:24-49
    h1_list.clear();
    for (int side = 2; side <= 3; ++side)
      for (uint32_t r = 0; r < md[side].num; ++r) {
        const uint32_t h1 = md[side].start + r;
        if (!used[h1] && h0c[2 * h1] != -1 && h2c[2 * h1] != -1) h1_list.push_back(static_cast<uint16_t>(h1));
      }
    if (h1_list.size() > MAX_MOD_HITS) out.flags |= F_H1_OVF;
    const uint32_t nh1 = static_cast<uint32_t>(h1_list.size());
    const uint32_t last_it = (nh1 + 15) / 16;
    const uint32_t n_last = ((nh1 - 1) % 16) + 1;
    for (uint32_t i = 0; i < last_it; ++i) {
      const bool is_last = i == last_it - 1;
      const uint32_t bdx = is_last ? n_last : 16;
      float best_fit[32];
      uint16_t best_h0[32], best_h2[32], h1_idx[32];
      for (uint32_t t = 0; t < 32; ++t) {
        const uint32_t tx = t % bdx, ty = t / bdx;
        const bool numerous = tx < ((32 - 1) % bdx) + 1;
        const uint32_t bdy = numerous ? (32 + bdx - 1) / bdx : (32 - 1) / bdx;
        best_fit[t] = FLT_MAX;
        best_h0[t] = best_h2[t] = h1_idx[t] = 0;
        const uint32_t rel = i * 16 + tx;
        if (rel >= nh1) continue;
        const uint32_t h1i = h1_list[rel];
        h1_idx[t] = static_cast<uint16_t>(h1i);
        const Hit& h1 = hits[h1i];
        const int h0f = h0c[2 * h1i], h0l = h0c[2 * h1i + 1], h2f = h2c[2 * h1i], h2l = h2c[2 * h1i + 1];
        const int h0n = h0l - h0f;
        for (int j = 0; j < (h0n + static_cast<int>(bdy) - 1) / static_cast<int>(bdy); ++j) {
          const int h0r = j * bdy + ty;
          if (h0r >= h0n) continue;
          const int h0i = h0f + h0r;
          if (used[h0i]) continue;
          const Hit& h0 = hits[h0i];
          for (int h2i = h2f; h2i < h2l; ++h2i) {
            if (used[h2i]) continue;
            const Hit& h2 = hits[h2i];
            const float dmax = MAX_SLOPE * (h0.z - h1.z);
            const float sd2 = 1.f / ((h2.z - h1.z) * (h2.z - h1.z));
            const float z2_tz = (h2.z - h0.z) / (h1.z - h0.z);
            const float x = h0.x + (h1.x - h0.x) * z2_tz;
            const float y = h0.y + (h1.y - h0.y) * z2_tz;
            const float dx = x - h2.x, dy = y - h2.y;
            const float sn = (dx * dx) + (dy * dy);
            const float scatter = sn * sd2;
            const bool pass = std::fabs(h1.x - h0.x) < dmax && std::fabs(h1.y - h0.y) < dmax &&
                              std::fabs(dx) < TOL && std::fabs(dy) < TOL && scatter < MAX_SCATTER_SEED;
            if (pass && scatter == best_fit[t]) out.flags |= F_SEED_TIE;
            if (pass && scatter < best_fit[t]) {
              best_fit[t] = scatter;
              best_h0[t] = static_cast<uint16_t>(h0i);
              best_h2[t] = static_cast<uint16_t>(h2i);
            }
          }
        }
      }
      // argmin over the thread column (TrackSeeding.cu:175-195), winners in lane order
      for (uint32_t t = 0; t < 32; ++t) {
        const uint32_t tx = t % bdx;
        const bool numerous = tx < ((32 - 1) % bdx) + 1;
        const uint32_t bdy = numerous ? (32 + bdx - 1) / bdx : (32 - 1) / bdx;
        int winner = -1;
        float bf = FLT_MAX;
        for (uint32_t yy = 0; yy < bdy; ++yy) {
          const uint32_t a = yy * bdx + tx;
          if (best_fit[a] < FLT_MAX && best_fit[a] == bf && static_cast<int>(t) == static_cast<int>(tx))
            out.flags |= F_SEED_TIE;
          if (best_fit[a] < bf) {
            winner = a;
            bf = best_fit[a];
          }
        }
        if (static_cast<int>(t) == winner) {
          const uint32_t tp = tracklet_ptr++ % TTF_MOD;
          tracklets[3 * tp] = best_h0[t];
          tracklets[3 * tp + 1] = h1_idx[t];
          tracklets[3 * tp + 2] = best_h2[t];
          ttf[ttf_ptr++ % TTF_MOD] = 0x80000000u | tp;
        }
      }
    }
  };

  auto fwd_candidates = [&](const ModuleData& m, float tx, float ty, const Hit& h0, bool odd, int& first, int& last) {
    // TrackForwarding.cuh:28-59
    const float dz = m.z - h0.z;
    const float predx = tx * dz, predy = ty * dz;
    const float xp = h0.x + predx, yp = h0.y + predy;
    const float phi = odd ? phi_odd(xp, yp) : phi_even(xp, yp);
    first = -1;
    last = -1;
    if (m.num == 0) {
      out.flags |= F_EMPTY_MODULE_READ;
      return;
    }
    first = bsearch_first(&phis[m.start], m.num, phi, FWD_PHI_TOL);
    if (first != -1) {
      last = bsearch_second(&phis[m.start + first], m.num - first, phi, FWD_PHI_TOL);
      first += m.start;
      last = last == 0 ? first + 1 : first + last;
    }
  };

  auto forwarding = [&](uint32_t prev_ttf, uint32_t diff) {
    // TrackForwarding.cu:41-181
    for (uint32_t e = 0; e < diff; ++e) {
      const uint32_t full = ttf[(prev_ttf + e) % TTF_MOD];
      const bool flag = (full & 0x80000000u) == 0x80000000u;
      const uint32_t skipped = (full & 0x70000000u) >> 28;
      uint32_t trackno = full & 0x0FFFFFFFu;
      TrackHits t;
      if (flag) {
        t.n = 3;
        t.h[0] = tracklets[3 * trackno];
        t.h[1] = tracklets[3 * trackno + 1];
        t.h[2] = tracklets[3 * trackno + 2];
      } else {
        t = track_slots[trackno];
      }
      const Hit& h0 = hits[t.h[t.n - 2]];
      const Hit& h1 = hits[t.h[t.n - 1]];
      const float td = 1.0f / (h1.z - h0.z);
      const float tx = (h1.x - h0.x) * td, ty = (h1.y - h0.y) * td;
      float best = FLT_MAX;
      uint16_t best_h2 = 0;
      int of, ol, ef, el;
      fwd_candidates(md[4], tx, ty, h0, true, of, ol);
      fwd_candidates(md[5], tx, ty, h0, false, ef, el);
      const int no = ol - of, ne = el - ef;
      for (int j = 0; j < no + ne; ++j) {
        const int h2i = j < no ? of + j : ef + j - no;
        const Hit& h2 = hits[h2i];
        const float dz = h2.z - h0.z;
        const float predx = tx * dz, predy = ty * dz;
        const float sd2 = 1.f / ((h2.z - h1.z) * (h2.z - h1.z));
        const float xp = h0.x + predx;
        const float dx = std::fabs(xp - h2.x);
        const float yp = h0.y + predy;
        const float dy = std::fabs(yp - h2.y);
        const float scatter = ((dx * dx) + (dy * dy)) * sd2;
        const bool cond = dx < TOL && dy < TOL && scatter < MAX_SCATTER_FWD;
        const float fit = cond ? scatter : FLT_MAX;
        if (fit < best) {
          best = fit;
          best_h2 = static_cast<uint16_t>(h2i);
        }
      }
      if (best != FLT_MAX) {
        used[best_h2] = 1;
        t.h[t.n++] = best_h2;
        if (t.n <= 4) {
          used[t.h[0]] = used[t.h[1]] = used[t.h[2]] = 1;
          trackno = n_tracks++;
          if (trackno >= MAX_TRACKS) out.flags |= F_TRACK_OVF;
          if (trackno >= track_slots.size()) track_slots.resize(trackno + 64);
        }
        track_slots[trackno] = t;
        ttf[ttf_ptr++ % TTF_MOD] = trackno;
      } else if (skipped < 1) {
        ttf[ttf_ptr++ % TTF_MOD] = ((skipped + 1) << 28) | (full & 0x8FFFFFFFu);
      } else if (t.n == 3) {
        weak.push_back(t.h[0]);
        weak.push_back(t.h[1]);
        weak.push_back(t.h[2]);
        ++weak_ptr;
      }
    }
  };

  // ProcessModules.cu:37-162
  uint32_t first_module = 51;
  load(first_module);
  seeding();
  uint32_t last_seeded = tracklet_ptr;
  uint32_t last_ttf = 0;
  first_module -= 2;
  while (first_module >= 4) {
    load(first_module);
    const uint32_t prev = last_ttf;
    last_ttf = ttf_ptr;
    if (last_ttf - prev > TTF_MOD) out.flags |= F_TTF_OVF;
    forwarding(prev, last_ttf - prev);
    if (ttf_ptr - prev > TTF_MOD) out.flags |= F_TTF_OVF;
    const uint32_t tracklets_before = tracklet_ptr;
    seeding();
    // tracklets of the previous and this seeding are still referenced by the ring
    if (tracklet_ptr - tracklets_before + last_seeded > TTF_MOD) out.flags |= F_TTF_OVF;
    last_seeded = tracklet_ptr - tracklets_before;
    first_module -= 2;
  }
  {
    const uint32_t prev = last_ttf;
    last_ttf = ttf_ptr;
    for (uint32_t e = 0; e < last_ttf - prev; ++e) {
      const uint32_t full = ttf[(prev + e) % TTF_MOD];
      if (full & 0x80000000u) {
        const uint32_t trackno = full & 0x0FFFFFFFu;
        weak.push_back(tracklets[3 * trackno]);
        weak.push_back(tracklets[3 * trackno + 1]);
        weak.push_back(tracklets[3 * trackno + 2]);
        ++weak_ptr;
      }
    }
  }
  if (weak_ptr > MAX_WEAK) out.flags |= F_WEAK_OVF;
  out.n_weak = weak_ptr;
  out.n_tracklets = tracklet_ptr;
  // weak_tracks_adder (WeakTracksAdder.cu:88-115)
  for (uint32_t w = 0; w < weak_ptr; ++w) {
    const uint16_t* h = &weak[3 * w];
    const bool any_used = used[h[0]] || used[h[1]] || used[h[2]];
    const float chi2 = weak_chi2(hits, h);
    if (!any_used && chi2 < MAX_CHI2) {
      const uint32_t trackno = n_tracks++;
      if (trackno >= MAX_TRACKS) out.flags |= F_TRACK_OVF;
      if (trackno >= track_slots.size()) track_slots.resize(trackno + 64);
      TrackHits t;
      t.n = 3;
      t.h[0] = h[0];
      t.h[1] = h[1];
      t.h[2] = h[2];
      track_slots[trackno] = t;
    }
  }
  tracks.assign(track_slots.begin(), track_slots.begin() + n_tracks);
}

void run_event(const uint8_t* ev_bytes, uint64_t bytes, const Geo& g, const Luts& L, int stages, EventOut& out)
{
  out = EventOut();
  if (!validate(ev_bytes, bytes)) {
    out.flags |= F_BAD_RAW;
    return;
  }
  RawView ev;
  std::memcpy(&ev.nb, ev_bytes, 4);
  ev.offs = reinterpret_cast<const uint32_t*>(ev_bytes + 4);
  ev.payload = ev_bytes + 4ull * (ev.nb + 2);
  std::vector<Hit> mod[NM];
  cluster_event(ev, g, L, mod, out.flags, out.n_candidates);
  // calculate_phi_and_sort: per-module stable sort on phi (CalculatePhi.cu:21-65)
  uint32_t start = 0;
  for (uint32_t m = 0; m < NM; ++m) {
    auto& v = mod[m];
    const bool odd = m & 1;
    for (auto& h : v) h.phi = odd ? phi_odd(h.x, h.y) : phi_even(h.x, h.y);
    std::vector<Hit> sorted(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
      uint32_t pos = 0;
      for (size_t j = 0; j < v.size(); ++j) pos += v[i].phi > v[j].phi || (v[i].phi == v[j].phi && i > j);
      sorted[pos] = v[i];
    }
    out.module_start[m] = start;
    out.module_num[m] = static_cast<uint32_t>(v.size());
    if (v.size() > MAX_MOD_HITS) out.flags |= F_MODULE_OVF;
    start += static_cast<uint32_t>(v.size());
    out.hits.insert(out.hits.end(), sorted.begin(), sorted.end());
  }
  out.module_start[NM] = start;
  if (start > 32767) out.flags |= F_HIT_OVF;  // short candidate windows of the reference
  if (stages < 2) return;
  search_event(out);
  // consolidate_velo_tracks + velo_kalman_fit
  for (const auto& t : out.tracks) {
    const State s = lsq_fit<float, State>(out.hits, t);
    const State64 s64 = lsq_fit<double, State64>(out.hits, t);
    out.lsq.push_back(s);
    out.lsq64.push_back(s64);
    out.kal.push_back(kalman_fit<float, State>(out.hits, t, s));
    out.kal64.push_back(kalman_fit<double, State64>(out.hits, t, s64));
  }
}

}  // namespace

// ============================================================================
// C ABI for tests and the CPU baseline.
// ============================================================================
struct OracleResult {
  std::vector<EventOut> events;
};

extern "C" {

// stages: 1 = clustering + phi sort only, 2 = full chain.
int oracle_run(const void* raw, const uint64_t* offsets, uint32_t n_events, const void* geometry, int n_threads,
               int stages, OracleResult** out)
{
  if (!raw || !offsets || !geometry || !out) return -1;
  auto* r = new OracleResult();
  r->events.resize(n_events);
  const float* f = static_cast<const float*>(geometry);
  const Geo g{f, f + 768, f + 1536};
  Luts L;
  build_luts(L);
  if (n_threads <= 0) n_threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  std::atomic<uint32_t> next{0};
  auto work = [&]() {
    for (;;) {
      const uint32_t i = next.fetch_add(1);
      if (i >= n_events) break;
      const uint8_t* ev = static_cast<const uint8_t*>(raw) + offsets[i];
      run_event(ev, offsets[i + 1] - offsets[i], g, L, stages, r->events[i]);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  *out = r;
  return 0;
}

void oracle_destroy(OracleResult* r) { delete r; }

void oracle_sizes(const OracleResult* r, uint64_t* n_hits, uint64_t* n_tracks, uint64_t* n_track_hits)
{
  uint64_t h = 0, t = 0, th = 0;
  for (const auto& e : r->events) {
    h += e.hits.size();
    t += e.tracks.size();
    for (const auto& tr : e.tracks) th += tr.n;
  }
  *n_hits = h;
  *n_tracks = t;
  *n_track_hits = th;
}

// Clusters: event_hit_offsets[N+1], module_num[N*52], hits SoA (x, y, z, phi, id) in the
// compact per-event order; flags[N]; extras[N*3] = (candidates, weak tracklets, tracklets).
void oracle_copy_clusters(const OracleResult* r, uint64_t* event_hit_offsets, uint32_t* module_num, float* x,
                          float* y, float* z, float* phi, uint32_t* id, uint32_t* flags, uint32_t* extras)
{
  uint64_t o = 0;
  for (size_t e = 0; e < r->events.size(); ++e) {
    const auto& ev = r->events[e];
    event_hit_offsets[e] = o;
    for (uint32_t m = 0; m < NM; ++m) module_num[e * NM + m] = ev.module_num[m];
    for (const auto& h : ev.hits) {
      x[o] = h.x;
      y[o] = h.y;
      z[o] = h.z;
      phi[o] = h.phi;
      id[o] = h.id;
      ++o;
    }
    flags[e] = ev.flags;
    if (extras) {
      extras[3 * e] = ev.n_candidates;
      extras[3 * e + 1] = ev.n_weak;
      extras[3 * e + 2] = ev.n_tracklets;
    }
  }
  event_hit_offsets[r->events.size()] = o;
}

// Tracks: event_track_offsets[N+1], track_hit_offsets[T+1], hit_index[H] (event-relative
// compact index), hit_id[H]; states SoA of 13 floats per track (x,y,tx,ty,c00,c20,c22,c11,
// c31,c33,chi2,z,backward) for the fp32 LSQ and Kalman fits and their fp64 twins.
void oracle_copy_tracks(const OracleResult* r, uint64_t* event_track_offsets, uint64_t* track_hit_offsets,
                        uint32_t* hit_index, uint32_t* hit_id, float* lsq, float* kal, double* lsq64, double* kal64)
{
  uint64_t t = 0, h = 0;
  for (size_t e = 0; e < r->events.size(); ++e) {
    const auto& ev = r->events[e];
    event_track_offsets[e] = t;
    for (size_t k = 0; k < ev.tracks.size(); ++k) {
      const auto& tr = ev.tracks[k];
      track_hit_offsets[t] = h;
      for (int i = 0; i < tr.n; ++i) {
        hit_index[h] = tr.h[i];
        hit_id[h] = ev.hits[tr.h[i]].id;
        ++h;
      }
      auto put = [&](float* dst, const State& s) {
        const float v[13] = {s.x, s.y, s.tx, s.ty, s.c00, s.c20, s.c22, s.c11, s.c31, s.c33, s.chi2, s.z,
                             s.backward ? 1.f : 0.f};
        std::memcpy(dst + 13 * t, v, sizeof v);
      };
      auto put64 = [&](double* dst, const State64& s) {
        const double v[13] = {s.x, s.y, s.tx, s.ty, s.c00, s.c20, s.c22, s.c11, s.c31, s.c33, s.chi2, s.z,
                              s.backward ? 1.0 : 0.0};
        std::memcpy(dst + 13 * t, v, sizeof v);
      };
      if (lsq) put(lsq, ev.lsq[k]);
      if (kal) put(kal, ev.kal[k]);
      if (lsq64) put64(lsq64, ev.lsq64[k]);
      if (kal64) put64(kal64, ev.kal64[k]);
      ++t;
    }
  }
  event_track_offsets[r->events.size()] = t;
  track_hit_offsets[t] = h;
}

void oracle_sp_luts(uint8_t* pat, float* fx, float* fy)
{
  Luts L;
  build_luts(L);
  std::memcpy(pat, L.pat, 256);
  std::memcpy(fx, L.fx, sizeof L.fx);
  std::memcpy(fy, L.fy, sizeof L.fy);
}
}
