// Host-side support of the VELO chain: SuperPixel lookup tables, raw-event validation,
// the seeded synthetic event generator (raw banks + MC truth) and the MC-truth track
// checker. Plain C++ (no CUDA): it is loaded by the Python mirror, by bench.py and by
// the C-ABI library at context creation.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <thread>
#include <vector>

#include "velo_format.hpp"
#include "../../include/velo_b200.h"

using namespace velo;

// ============================================================================
// SuperPixel pattern tables.
//
// For every 8-bit SP mask: the (at most two) 8-connected pixel groups, their centroid
// pixel, size and fractional centroid. Same contents as the table the reference builds
// with a flood fill (x86/velo/clustering/src/ClusteringCommon.cpp:3-101): groups are
// numbered in order of their lowest set bit, pattern byte = centroid (col<<2|row) of
// group 0 in bits 0..2, two-group flag in bit 3, group 1 centroid in bits 4..6.
// Here the groups come from bit-parallel dilation of the 2x4 mask.
// ============================================================================
static uint32_t sp_neighbours(uint32_t m)
{
  // pixel bit = col*4 + row, rows 0..3 in a column
  const uint32_t c0 = m & 0x0Fu, c1 = (m >> 4) & 0x0Fu;
  auto vert = [](uint32_t c) { return (c | (c << 1) | (c >> 1)) & 0x0Fu; };
  const uint32_t n0 = vert(c0) | vert(c1);  // column 0 touched by either column (incl. diagonals)
  const uint32_t n1 = vert(c1) | vert(c0);
  return (n0 | (n1 << 4)) & 0xFFu;
}

extern "C" void velo_build_sp_luts(uint8_t* patterns, uint8_t* sizes, float* fx, float* fy)
{
  for (uint32_t sp = 0; sp < 256; ++sp) {
    patterns[sp] = 0;
    sizes[sp] = 0;
    fx[2 * sp] = fx[2 * sp + 1] = 0.f;
    fy[2 * sp] = fy[2 * sp + 1] = 0.f;
    uint32_t remaining = sp;
    uint32_t group = 0;
    while (remaining) {
      uint32_t g = remaining & (~remaining + 1u);  // lowest pixel seeds the group
      for (;;) {
        const uint32_t grown = sp_neighbours(g) & remaining;
        if ((grown | g) == g) break;
        g |= grown;
      }
      remaining &= ~g;
      uint32_t n = 0, sx = 0, sy = 0;
      for (uint32_t b = 0; b < 8; ++b)
        if (g & (1u << b)) {
          ++n;
          sx += b >> 2;
          sy += b & 3u;
        }
      const uint32_t cx = sx / n, cy = sy / n;
      sizes[sp] |= static_cast<uint8_t>(n << (4 * group));
      patterns[sp] |= static_cast<uint8_t>(((cx << 2) | cy) << (4 * group));
      patterns[sp] |= static_cast<uint8_t>(group << 3);
      fx[2 * sp + group] = sx / static_cast<float>(n) - cx;
      fy[2 * sp + group] = sy / static_cast<float>(n) - cy;
      ++group;
    }
  }
}

// ============================================================================
// Raw-event validation. Returns 0 when the event is well formed: 208 banks, offsets
// non-decreasing and inside the event, bank i carries sensor i, sp_count fits the bank.
// ============================================================================
extern "C" int velo_validate_raw_event(const void* event, uint64_t event_bytes)
{
  const uint8_t* p = static_cast<const uint8_t*>(event);
  if (event_bytes < 4) return VELO_ERR_BAD_RAW;
  uint32_t nb;
  std::memcpy(&nb, p, 4);
  if (nb != kSensors) return VELO_ERR_BAD_RAW;
  const uint64_t header = 4ull * (1 + nb + 1);
  if (event_bytes < header) return VELO_ERR_BAD_RAW;
  const uint32_t* offs = reinterpret_cast<const uint32_t*>(p + 4);
  const uint64_t payload = event_bytes - header;
  for (uint32_t b = 0; b < nb; ++b) {
    const uint64_t o = offs[b], e = offs[b + 1];
    if ((o & 3) || e < o + 8 || e > payload) return VELO_ERR_BAD_RAW;
    uint32_t sensor, count;
    std::memcpy(&sensor, p + header + o, 4);
    std::memcpy(&count, p + header + o + 4, 4);
    if (sensor != b) return VELO_ERR_BAD_RAW;
    if (8ull + 4ull * count > e - o) return VELO_ERR_BAD_RAW;
  }
  return 0;
}

// ============================================================================
// Synthetic event generator.
// ============================================================================
namespace {

struct Rng {  // xoshiro256**, seeded by splitmix64 of (seed, stream)
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x)
  {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  Rng(uint64_t seed, uint64_t stream)
  {
    uint64_t x = seed * 0xD1B54A32D192ED03ull ^ (stream + 0x632BE59BD9B4E019ull);
    for (auto& v : s) v = splitmix(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next()
  {
    const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  double gauss()
  {
    double u1 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * uniform());
  }
  uint32_t poisson(double lambda)
  {
    if (lambda <= 0) return 0;
    if (lambda > 60) {  // normal approximation for very large means
      const double v = lambda + std::sqrt(lambda) * gauss();
      return v < 0 ? 0u : static_cast<uint32_t>(v + 0.5);
    }
    const double L = std::exp(-lambda);
    uint32_t k = 0;
    double p = uniform();
    while (p > L) {
      ++k;
      p *= uniform();
    }
    return k;
  }
};

struct Geometry {
  const float* local_x;
  const float* x_pitch;
  const float* ltg;
  float lo[kSensorColumns], hi[kSensorColumns];
  double box[kSensors][4];  // global x/y bounding box of each sensor (xmin, xmax, ymin, ymax)
  double z[kSensors];
  explicit Geometry(const void* blob)
  {
    GeometryView v = geometry_view(blob);
    local_x = v.local_x;
    x_pitch = v.x_pitch;
    ltg = v.ltg;
    for (uint32_t c = 0; c < kSensorColumns; ++c) {
      lo[c] = local_x[c] - 0.5f * x_pitch[c];
      hi[c] = local_x[c] + 0.5f * x_pitch[c];
    }
    const double w = hi[kSensorColumns - 1] + 0.01, h = kRows * kPixelSize + 0.01;
    for (uint32_t s = 0; s < kSensors; ++s) {
      const float* L = ltg + 16 * s;
      double b[4] = {1e9, -1e9, 1e9, -1e9};
      for (double u : {-0.01, w})
        for (double v2 : {-0.01, h}) {
          const double gx = L[0] * u + L[1] * v2 + L[9], gy = L[3] * u + L[4] * v2 + L[10];
          b[0] = std::min(b[0], gx);
          b[1] = std::max(b[1], gx);
          b[2] = std::min(b[2], gy);
          b[3] = std::max(b[3], gy);
        }
      for (int k = 0; k < 4; ++k) box[s][k] = b[k];
      z[s] = L[11];
    }
  }
  // Column whose pixel contains lx (nearest centre when lx falls in an edge gap); -1 outside.
  int column(double lx) const
  {
    if (lx < lo[0] || lx >= hi[kSensorColumns - 1]) return -1;
    int a = 0, b = kSensorColumns - 1;
    while (a < b) {  // first column with hi > lx
      const int m = (a + b) / 2;
      if (hi[m] > lx) b = m; else a = m + 1;
    }
    if (a > 0 && lx < lo[a] && (lo[a] - lx) > (lx - hi[a - 1])) return a - 1;
    return a;
  }
};

struct McParticle {
  uint32_t key;
  int32_t pid;
  float p, pt, eta, phi;
  uint8_t is_long, has_velo;
  uint32_t n_pv;
  std::vector<uint32_t> hits;
};

struct GenEvent {
  std::vector<uint32_t> raw;  // u32 words of the raw event
  std::vector<uint8_t> mc;    // MC_info tracks blob
  uint32_t n_clusters_truth = 0;
};

void serialize_mc(const std::vector<McParticle>& mcps, std::vector<uint8_t>& out)
{
  // Layout of checker/tracking/src/MCEvent.cpp:16-92 (VELO part; UT and SciFi empty).
  auto put32 = [&](uint32_t v) {
    const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
    out.insert(out.end(), b, b + 4);
  };
  auto putf = [&](float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    put32(u);
  };
  put32(static_cast<uint32_t>(mcps.size()));
  for (const auto& m : mcps) {
    put32(m.key);
    put32(static_cast<uint32_t>(m.pid));
    putf(m.p);
    putf(m.pt);
    putf(m.eta);
    putf(m.phi);
    const uint8_t flags[8] = {m.is_long, 0, m.has_velo, 0, 0, 0, 0, 0};
    out.insert(out.end(), flags, flags + 8);
    put32(m.n_pv);
    put32(static_cast<uint32_t>(m.hits.size()));
    for (uint32_t h : m.hits) put32(h);
    put32(0);  // UT hits
    put32(0);  // SciFi hits
  }
}

void generate_event(const VeloGenConfig& cfg, const Geometry& g, uint64_t index, GenEvent& ev)
{
  Rng rng(cfg.seed, index);
  const double nu = cfg.nu_min == cfg.nu_max ? cfg.nu_min : rng.uniform(cfg.nu_min, cfg.nu_max);
  const bool noisy = cfg.noisy_event_fraction > 0 && rng.uniform() < cfg.noisy_event_fraction;
  const double noise_mean = cfg.noise_per_asic_per_nu * nu * (noisy ? cfg.noisy_factor : 1.0);
  const uint32_t n_pv = rng.poisson(nu * cfg.visible_fraction);

  std::vector<uint32_t> pixels;  // key = sensor<<20 | col<<8 | row
  pixels.reserve(4096);
  std::vector<McParticle> mcps;

  for (uint32_t v = 0; v < n_pv; ++v) {
    const double x0 = cfg.pv_sigma_xy * rng.gauss(), y0 = cfg.pv_sigma_xy * rng.gauss();
    const double z0 = cfg.pv_sigma_z * rng.gauss();
    const uint32_t n_tracks = rng.poisson(cfg.tracks_per_pv);
    for (uint32_t t = 0; t < n_tracks; ++t) {
      const bool backward = rng.uniform() < cfg.backward_fraction;
      const double eta = backward ? rng.uniform(-4.0, -2.0) : rng.uniform(2.0, 5.0);
      const double phi = rng.uniform(0.0, 2.0 * M_PI);
      const double pt = -600.0 * std::log(1.0 - rng.uniform() + 1e-12) + 50.0;  // MeV
      const double theta = 2.0 * std::atan(std::exp(-eta));
      const double tan_t = std::tan(theta);
      const double tx = tan_t * std::cos(phi), ty = tan_t * std::sin(phi);
      const double dir = backward ? -1.0 : 1.0;

      McParticle mcp;
      mcp.key = static_cast<uint32_t>(mcps.size());
      mcp.pid = (rng.next() & 1) ? 211 : -211;
      mcp.pt = static_cast<float>(pt);
      mcp.p = static_cast<float>(pt * std::cosh(eta));
      mcp.eta = static_cast<float>(eta);
      mcp.phi = static_cast<float>(phi);
      mcp.n_pv = n_pv;
      uint64_t modules_hit = 0;

      uint8_t crossed[kSensors];
      for (uint32_t s = 0; s < kSensors; ++s) {
        const double dzs = g.z[s] - z0;
        const double gx = x0 + tx * dzs, gy = y0 + ty * dzs;
        crossed[s] = (dzs * dir > 0) & (gx >= g.box[s][0]) & (gx <= g.box[s][1]) & (gy >= g.box[s][2]) &
                     (gy <= g.box[s][3]);
      }
      for (uint32_t s = 0; s < kSensors; ++s) {
        if (!crossed[s]) continue;
        const float* L = g.ltg + 16 * s;
        const double zs = L[11];
        const double gx = x0 + tx * (zs - z0), gy = y0 + ty * (zs - z0);
        const double dx = gx - L[9], dy = gy - L[10];
        const double lx = L[0] * dx + L[3] * dy;
        const double ly = L[1] * dx + L[4] * dy;
        if (ly < 0 || ly >= kRows * kPixelSize) continue;
        const int col = g.column(lx);
        if (col < 0) continue;
        if (rng.uniform() >= cfg.hit_efficiency) continue;
        const int row = static_cast<int>(ly / kPixelSize);
        // Deposit 1-3 adjacent pixels, spread towards the nearer pixel edge.
        const double fxp = (lx - g.lo[col]) / g.x_pitch[col] - 0.5;
        const double fyp = ly / kPixelSize - row - 0.5;
        const int sc = fxp >= 0 ? 1 : -1, sr = fyp >= 0 ? 1 : -1;
        int cols[3] = {col, col, col}, rows[3] = {row, row, row};
        const double u = rng.uniform();
        int n = u < cfg.p_one_pixel ? 1 : (u < cfg.p_one_pixel + cfg.p_two_pixels ? 2 : 3);
        if (n >= 2) {
          if (std::fabs(fxp) > std::fabs(fyp)) cols[1] = col + sc; else rows[1] = row + sr;
        }
        if (n == 3) {
          if (cols[1] != col) rows[2] = row + sr; else cols[2] = col + sc;
        }
        uint32_t sx = 0, sy = 0, m = 0;
        for (int k = 0; k < n; ++k) {
          if (cols[k] < 0 || cols[k] >= static_cast<int>(kSensorColumns) || rows[k] < 0 ||
              rows[k] >= static_cast<int>(kRows))
            continue;
          pixels.push_back((s << 20) | (static_cast<uint32_t>(cols[k]) << 8) | static_cast<uint32_t>(rows[k]));
          sx += cols[k];
          sy += rows[k];
          ++m;
        }
        const uint32_t cx = sx / m, cy = sy / m;
        mcp.hits.push_back(lhcb_id(channel_id(s, cx / kChipColumns, cx % kChipColumns, cy)));
        modules_hit |= 1ull << (s >> 2);
      }
      const int n_modules = __builtin_popcountll(modules_hit);
      mcp.has_velo = n_modules >= 3;
      mcp.is_long = mcp.has_velo && eta > 2.0 && eta < 5.0;
      ev.n_clusters_truth += static_cast<uint32_t>(mcp.hits.size());
      if (!mcp.hits.empty()) mcps.push_back(std::move(mcp));
    }
  }
  // Noise pixels, uniformly over every ASIC.
  for (uint32_t s = 0; s < kSensors; ++s)
    for (uint32_t chip = 0; chip < kChipsPerSensor; ++chip) {
      const uint32_t k = rng.poisson(noise_mean);
      for (uint32_t i = 0; i < k; ++i) {
        const uint32_t c = chip * kChipColumns + static_cast<uint32_t>(rng.next() % kChipColumns);
        const uint32_t r = static_cast<uint32_t>(rng.next() % kRows);
        pixels.push_back((s << 20) | (c << 8) | r);
      }
    }
  for (auto& m : mcps) m.n_pv = n_pv;

  // Encode SuperPixels per sensor: address-sorted words, isolation from the 8 neighbours.
  ev.raw.clear();
  ev.raw.push_back(kSensors);
  const size_t offs_at = ev.raw.size();
  ev.raw.resize(offs_at + kSensors + 1, 0);
  const size_t payload_at = ev.raw.size();
  std::sort(pixels.begin(), pixels.end());
  pixels.erase(std::unique(pixels.begin(), pixels.end()), pixels.end());
  std::vector<std::pair<uint32_t, uint32_t>> sps, merged;  // (addr, mask)
  std::vector<uint64_t> occupancy(384, 0);
  size_t p = 0;
  for (uint32_t s = 0; s < kSensors; ++s) {
    sps.clear();
    for (; p < pixels.size() && (pixels[p] >> 20) == s; ++p) {
      const uint32_t c = (pixels[p] >> 8) & 0xFFF, r = pixels[p] & 0xFF;
      const uint32_t addr = ((c >> 1) << 6) | (r >> 2);
      const uint32_t bit = 1u << (((c & 1u) << 2) | (r & 3u));
      sps.emplace_back(addr, bit);
    }
    std::sort(sps.begin(), sps.end());
    merged.clear();
    for (auto& e : sps) {
      if (!merged.empty() && merged.back().first == e.first) merged.back().second |= e.second;
      else merged.push_back(e);
    }
    ev.raw[offs_at + s] = static_cast<uint32_t>((ev.raw.size() - payload_at) * 4);
    ev.raw.push_back(s);
    ev.raw.push_back(static_cast<uint32_t>(merged.size()));
    // occupancy of SP columns: one 64-bit row mask per SP column (384 columns)
    for (auto& e : merged) occupancy[e.first >> 6] |= 1ull << (e.first & 0x3F);
    for (auto& e : merged) {
      const int32_t c = e.first >> 6, r = e.first & 0x3F;
      const uint64_t rows3 = (r > 0 ? 7ull << (r - 1) : 3ull) & ~0ull;  // rows r-1..r+1
      const uint64_t self = 1ull << r;
      uint64_t near = (occupancy[c] & rows3 & ~self);
      if (c > 0) near |= occupancy[c - 1] & rows3;
      if (c < 383) near |= occupancy[c + 1] & rows3;
      ev.raw.push_back(make_sp_word(c, r, e.second, near == 0));
    }
    for (auto& e : merged) occupancy[e.first >> 6] = 0;
  }
  ev.raw[offs_at + kSensors] = static_cast<uint32_t>((ev.raw.size() - payload_at) * 4);
  ev.mc.clear();
  serialize_mc(mcps, ev.mc);
}

}  // namespace

struct VeloGenBatch {
  std::vector<GenEvent> events;
  uint64_t raw_bytes = 0, mc_bytes = 0;
};

extern "C" void velo_gen_default_config(VeloGenConfig* cfg)
{
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->seed = 0;
  cfg->nu_min = cfg->nu_max = 7.6f;
  cfg->visible_fraction = 0.7f;
  cfg->tracks_per_pv = 20.f;
  cfg->backward_fraction = 0.1f;
  cfg->pv_sigma_xy = 0.03f;
  cfg->pv_sigma_z = 50.f;
  cfg->hit_efficiency = 0.96f;
  cfg->p_one_pixel = 0.45f;
  cfg->p_two_pixels = 0.40f;
  cfg->noise_per_asic_per_nu = 0.316f;
  cfg->noisy_event_fraction = 0.f;
  cfg->noisy_factor = 1.f;
}

extern "C" int velo_gen_create(const VeloGenConfig* cfg, const void* geometry, uint64_t first_event,
                               uint32_t n_events, int n_threads, VeloGenBatch** out)
{
  if (!cfg || !geometry || !out) return VELO_ERR_INVALID;
  auto* b = new VeloGenBatch();
  b->events.resize(n_events);
  Geometry g(geometry);
  if (n_threads <= 0) n_threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  n_threads = std::min<int>(n_threads, std::max<uint32_t>(1, n_events));
  std::atomic<uint32_t> next{0};
  auto work = [&]() {
    for (;;) {
      const uint32_t i = next.fetch_add(16);
      if (i >= n_events) break;
      for (uint32_t k = i; k < std::min(n_events, i + 16); ++k) generate_event(*cfg, g, first_event + k, b->events[k]);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  for (auto& e : b->events) {
    b->raw_bytes += 4ull * e.raw.size();
    b->mc_bytes += e.mc.size();
  }
  *out = b;
  return 0;
}

extern "C" uint64_t velo_gen_raw_bytes(const VeloGenBatch* b) { return b ? b->raw_bytes : 0; }
extern "C" uint64_t velo_gen_mc_bytes(const VeloGenBatch* b) { return b ? b->mc_bytes : 0; }

// raw: raw_bytes; offsets: n_events+1 byte offsets (u64 so batches above 4 GiB are described).
extern "C" int velo_gen_copy(const VeloGenBatch* b, void* raw, uint64_t* raw_offsets, void* mc,
                             uint64_t* mc_offsets, uint32_t* truth_clusters)
{
  if (!b) return VELO_ERR_INVALID;
  uint64_t r = 0, m = 0;
  for (size_t i = 0; i < b->events.size(); ++i) {
    const auto& e = b->events[i];
    if (raw_offsets) raw_offsets[i] = r;
    if (mc_offsets) mc_offsets[i] = m;
    if (raw) std::memcpy(static_cast<uint8_t*>(raw) + r, e.raw.data(), 4 * e.raw.size());
    if (mc) std::memcpy(static_cast<uint8_t*>(mc) + m, e.mc.data(), e.mc.size());
    if (truth_clusters) truth_clusters[i] = e.n_clusters_truth;
    r += 4 * e.raw.size();
    m += e.mc.size();
  }
  if (raw_offsets) raw_offsets[b->events.size()] = r;
  if (mc_offsets) mc_offsets[b->events.size()] = m;
  return 0;
}

extern "C" void velo_gen_destroy(VeloGenBatch* b) { delete b; }

// ============================================================================
// MC-truth checker: association of track LHCb ids to MC particles and the VELO
// efficiency/ghost/clone bookkeeping of checker/tracking/src/TrackChecker.cpp:349-405,
// checker/tracking/include/MCAssociator.h:166-182 (weight = hits on best MCP / matched
// hits, ghost below 0.7), for the categories "Not electron long eta25"
// (CategoriesTrackChecker.cpp:120) and "Not electron Velo" (:215).
// ============================================================================
namespace {
struct ParsedMcp {
  uint32_t key;
  int32_t pid;
  float p, pt, eta;
  bool is_long, has_velo;
  uint32_t n_hits;
};
}  // namespace

extern "C" int velo_check_tracks(const void* mc_blob, const uint64_t* mc_offsets, uint32_t n_events,
                                 const uint32_t* event_track_offsets, const uint32_t* track_hit_offsets,
                                 const uint32_t* hit_ids, VeloCheckResult* res)
{
  if (!mc_blob || !mc_offsets || !event_track_offsets || !track_hit_offsets || !hit_ids || !res) return VELO_ERR_INVALID;
  std::memset(res, 0, sizeof(*res));
  const uint8_t* base = static_cast<const uint8_t*>(mc_blob);
  double ghost_per_event_acc = 0;
  for (uint32_t e = 0; e < n_events; ++e) {
    const uint8_t* p = base + mc_offsets[e];
    const uint8_t* end = base + mc_offsets[e + 1];
    auto get32 = [&](uint32_t& v) {
      if (p + 4 > end) return false;
      std::memcpy(&v, p, 4);
      p += 4;
      return true;
    };
    uint32_t n_mcp = 0;
    if (!get32(n_mcp)) return VELO_ERR_BAD_MC;
    std::vector<ParsedMcp> mcps;
    std::vector<std::pair<uint32_t, uint32_t>> id_map;  // (lhcb id, mcp index)
    for (uint32_t i = 0; i < n_mcp; ++i) {
      ParsedMcp m{};
      uint32_t u;
      if (!get32(m.key)) return VELO_ERR_BAD_MC;
      if (!get32(u)) return VELO_ERR_BAD_MC;
      m.pid = static_cast<int32_t>(u);
      float f[4];
      for (float& x : f) {
        if (!get32(u)) return VELO_ERR_BAD_MC;
        std::memcpy(&x, &u, 4);
      }
      m.p = f[0];
      m.pt = f[1];
      m.eta = f[2];
      if (p + 8 > end) return VELO_ERR_BAD_MC;
      m.is_long = p[0] != 0;
      m.has_velo = p[2] != 0;
      p += 8;
      uint32_t npv, nv, nut, nft;
      if (!get32(npv) || !get32(nv)) return VELO_ERR_BAD_MC;
      std::vector<uint32_t> hits(nv);
      for (auto& h : hits)
        if (!get32(h)) return VELO_ERR_BAD_MC;
      if (!get32(nut)) return VELO_ERR_BAD_MC;
      p += 4ull * nut;
      if (!get32(nft)) return VELO_ERR_BAD_MC;
      p += 4ull * nft;
      if (p > end) return VELO_ERR_BAD_MC;
      if (nv == 0) continue;  // only MCPs with VELO hits enter the VELO checker
      m.n_hits = nv;
      for (uint32_t h : hits) id_map.emplace_back(h, static_cast<uint32_t>(mcps.size()));
      mcps.push_back(m);
    }
    // The association map is built and sorted as the reference's MCAssociator builds it
    // (checker/tracking/src/MCAssociator.cpp:13-29): entries appended particle by particle in
    // file order, sorted on the id alone with std::sort, looked up with lower_bound. An id
    // that several particles share (real data has some) counts for the particle whose entry
    // that sort leaves first; comparing the index too would pick another particle for some
    // of them and change the weight of those tracks.
    std::sort(id_map.begin(), id_map.end(),
              [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
                return a.first < b.first;
              });
    auto is_electron = [](const ParsedMcp& m) { return std::abs(m.pid) == 11; };
    auto cat_long = [&](const ParsedMcp& m) { return m.is_long && !is_electron(m) && m.eta > 2.f && m.eta < 5.f; };
    auto cat_velo = [&](const ParsedMcp& m) { return m.has_velo && !is_electron(m); };
    for (const auto& m : mcps) {
      res->long_reconstructible += cat_long(m);
      res->velo_reconstructible += cat_velo(m);
    }
    std::vector<uint8_t> seen_long(mcps.size(), 0), seen_velo(mcps.size(), 0);
    const uint32_t t0 = event_track_offsets[e], t1 = event_track_offsets[e + 1];
    uint32_t ghosts = 0;
    for (uint32_t t = t0; t < t1; ++t) {
      std::map<uint32_t, uint32_t> counts;
      uint32_t matched = 0;
      for (uint32_t h = track_hit_offsets[t]; h < track_hit_offsets[t + 1]; ++h) {
        auto it = std::lower_bound(id_map.begin(), id_map.end(), hit_ids[h],
                                   [](const std::pair<uint32_t, uint32_t>& a, uint32_t id) { return a.first < id; });
        if (it == id_map.end() || it->first != hit_ids[h]) continue;
        ++matched;
        ++counts[it->second];
      }
      uint32_t best = 0, best_n = 0;
      for (auto& kv : counts)
        if (kv.second > best_n) {
          best = kv.first;
          best_n = kv.second;
        }
      const float w = matched ? float(best_n) / float(matched) : 0.f;
      if (!matched || w < 0.7f) {
        ++ghosts;
        continue;
      }
      const ParsedMcp& m = mcps[best];
      if (cat_long(m)) {
        if (seen_long[best]) ++res->long_clones; else { seen_long[best] = 1; ++res->long_found; }
      }
      if (cat_velo(m)) {
        if (seen_velo[best]) ++res->velo_clones; else { seen_velo[best] = 1; ++res->velo_found; }
      }
    }
    res->tracks += t1 - t0;
    res->ghosts += ghosts;
    if (t1 > t0) ghost_per_event_acc += double(ghosts) / double(t1 - t0);
    ++res->events;
  }
  res->long_efficiency = res->long_reconstructible ? double(res->long_found) / res->long_reconstructible : 0.0;
  res->velo_efficiency = res->velo_reconstructible ? double(res->velo_found) / res->velo_reconstructible : 0.0;
  res->ghost_rate = res->tracks ? double(res->ghosts) / res->tracks : 0.0;
  res->ghost_rate_per_event = res->events ? ghost_per_event_acc / res->events : 0.0;
  return 0;
}
