// Shared constants and data-format definitions of the VELO chain (host and device).
//
// Values and layouts are the ones the LHCb Allen VELO stage defines, so that raw
// input and consolidated output are interchangeable with it:
//   detector constants          cuda/velo/common/include/VeloDefinitions.cuh:7-77
//   clustering constants        cuda/velo/common/include/ClusteringDefinitions.cuh:9-50
//   raw event / bank layout     cuda/velo/common/src/ClusteringDefinitions.cu:3-21, cuda/velo/readme.md
//   geometry layout             cuda/velo/common/src/ClusteringDefinitions.cu:23-53
//   channel id / LHCb id        cuda/velo/common/src/ClusteringDefinitions.cu:55-61
//   module z table              stream/sequence/src/Constants.cu:27-31
//   consolidated output layout  cuda/event_model/velo/include/VeloConsolidated.cuh:12-144,
//                               cuda/event_model/common/include/ConsolidatedTypes.cuh:11-66
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define VELO_HD __host__ __device__ __forceinline__
#else
#define VELO_HD inline
#endif

namespace velo {

// ---- detector ---------------------------------------------------------------
constexpr uint32_t kModules = 52;
constexpr uint32_t kSensorsPerModule = 4;
constexpr uint32_t kSensors = kModules * kSensorsPerModule;  // 208 raw banks per event
constexpr uint32_t kChipsPerSensor = 3;
constexpr uint32_t kRows = 256;
constexpr uint32_t kChipColumns = 256;
constexpr uint32_t kSensorColumns = kChipColumns * kChipsPerSensor;  // 768
constexpr float kPixelSize = 0.055f;
constexpr uint32_t kGeometryBytes = 4u * (2u * kSensorColumns + 16u * kSensors);  // 19456

// ---- capacities of the reference stage (kept as the plain-path limits) --------
constexpr uint32_t kMaxHitsPerModule = 500;     // shared phi buffer of the reference sort
constexpr uint32_t kMaxHitsPerEvent = 9500;     // u16 hit indices
constexpr uint32_t kMaxTracks = 1200;           // per event
constexpr uint32_t kMaxTrackSize = 26;
constexpr uint32_t kMaxCandidatesEvent = 3000;  // clustering candidates per event
constexpr uint32_t kTtfModulo = 2000;           // tracks-to-follow / tracklet ring size
constexpr uint32_t kMaxWeakTracks = 500;

// ---- tracking tunables (VeloDefinitions.cuh:36-76) ----------------------------
constexpr uint32_t kMaxConcurrentH1 = 16;
constexpr float kPhiExtrapolation = 0.062f;
constexpr float kForwardPhiTolerance = 0.052f;
constexpr float kMaxSlope = 0.4f;
constexpr float kTolerance = 0.6f;
constexpr float kMaxScatterSeeding = 0.004f;
constexpr float kMaxScatterForwarding = 0.004f;
constexpr uint32_t kMaxSkippedModules = 1;
constexpr float kParamW = 3966.94f;
constexpr float kParamWInverted = 0.000252083f;
constexpr float kMaxChi2 = 20.0f;

// ---- clustering masks (ClusteringDefinitions.cuh:14-21) ----------------------
constexpr uint32_t kMaskBottom = 0xFFFEFFFFu;
constexpr uint32_t kMaskTop = 0xFFFF7FFFu;
constexpr uint32_t kMaskTopLeft = 0x7FFF7FFFu;
constexpr uint32_t kMaskBottomRight = 0xFFFEFFFEu;
constexpr uint32_t kMaskLtrTopRight = 0x7FFF0000u;
constexpr uint32_t kMaskRtlBottomLeft = 0x0000FFFEu;
constexpr uint32_t kMaxClusteringIterations = 12;

// Candidate pixel index (0..8 one-hot nibble) -> k, Constants.cu:36
constexpr uint8_t kCandidateKs[9] = {0, 0, 1, 4, 4, 5, 5, 5, 5};

// Module z positions used by tracking (Constants.cu:27-31).
#define VELO_MODULE_Z_VALUES                                                                                      \
  -287.5f, -275.f, -262.5f, -250.f, -237.5f, -225.f, -212.5f, -200.f, -137.5f, -125.f, -62.5f, -50.f, -37.5f,    \
    -25.f, -12.5f, 0.f, 12.5f, 25.f, 37.5f, 50.f, 62.5f, 75.f, 87.5f, 100.f, 112.5f, 125.f, 137.5f, 150.f,        \
    162.5f, 175.f, 187.5f, 200.f, 212.5f, 225.f, 237.5f, 250.f, 262.5f, 275.f, 312.5f, 325.f, 387.5f, 400.f,      \
    487.5f, 500.f, 587.5f, 600.f, 637.5f, 650.f, 687.5f, 700.f, 737.5f, 750.f
constexpr float kModuleZ[kModules] = {VELO_MODULE_Z_VALUES};

// ---- raw event ----------------------------------------------------------------
// u32 number_of_raw_banks, u32 raw_bank_offset[n+1] (byte offsets into the payload),
// then per bank: u32 sensor_index, u32 sp_count, u32 sp_word[sp_count].
// SP word: bit31 = no neighbouring SP, bits 8..22 = SP address (row = addr & 0x3F,
// col = addr >> 6), bits 0..7 = 2x4 pixel mask (0x01..0x08 column 0 rows 0..3,
// 0x10..0x80 column 1 rows 0..3).
VELO_HD uint32_t sp_isolated(uint32_t w) { return w & 0x80000000u; }
VELO_HD uint32_t sp_addr(uint32_t w) { return (w & 0x007FFF00u) >> 8; }
VELO_HD uint32_t sp_row(uint32_t w) { return sp_addr(w) & 0x3Fu; }
VELO_HD uint32_t sp_col(uint32_t w) { return sp_addr(w) >> 6; }
VELO_HD uint32_t sp_mask(uint32_t w) { return w & 0xFFu; }
VELO_HD uint32_t make_sp_word(uint32_t col, uint32_t row, uint32_t mask, bool isolated)
{
  return (isolated ? 0x80000000u : 0u) | (((col << 6) | row) << 8) | (mask & 0xFFu);
}

// channel id = sensor<<18 | chip<<16 | col<<8 | row ; LHCb id = VP(8)<<28 + cid
VELO_HD uint32_t channel_id(uint32_t sensor, uint32_t chip, uint32_t col, uint32_t row)
{
  return (sensor << 18) | (chip << 16) | (col << 8) | row;
}
VELO_HD uint32_t lhcb_id(uint32_t cid) { return (8u << 28) + cid; }
VELO_HD uint32_t lhcb_id_sensor(uint32_t id) { return (id >> 18) & 0x3FFu; }
VELO_HD uint32_t lhcb_id_module(uint32_t id) { return lhcb_id_sensor(id) >> 2; }

// ---- geometry blob ------------------------------------------------------------
// float local_x[768], float x_pitch[768], float ltg[208][16] (3x3 rotation row-major in
// [0..8], translation in [9..11]).
struct GeometryView {
  const float* local_x;
  const float* x_pitch;
  const float* ltg;
};
VELO_HD GeometryView geometry_view(const void* blob)
{
  const float* f = static_cast<const float*>(blob);
  return GeometryView{f, f + kSensorColumns, f + 2 * kSensorColumns};
}

// ---- per-event status flags (velo_run outputs) ----------------------------
enum StatusFlags : uint32_t {
  kStatusOk = 0,
  kStatusBadRawEvent = 1u << 0,       // malformed banks; event skipped (no clusters)
  kStatusModuleOverflow = 1u << 1,    // > kMaxHitsPerModule clusters in a module
  kStatusHitOverflow = 1u << 2,       // > kMaxHitsPerEvent clusters in the event
  kStatusCandidateOverflow = 1u << 3, // > kMaxCandidatesEvent clustering candidates
  kStatusTrackOverflow = 1u << 4,     // > kMaxTracks tracks (extra tracks dropped)
  kStatusTtfOverflow = 1u << 5,       // > kTtfModulo live tracks-to-follow / tracklets
  kStatusWeakOverflow = 1u << 6,      // > kMaxWeakTracks weak tracklets (reference would spill)
  kStatusH1Overflow = 1u << 7,        // > kMaxHitsPerModule seeding h1 hits in one step
  kStatusBigSpIndex = 1u << 8,        // a bank holds > 256 SPs (reference u8 sp_index wraps)
  kStatusMlpFallback = 1u << 9,       // learned pruning skipped: occupancy outside trained range
  kStatusNotSelected = 1u << 14,      // position beyond the events the global event cut selected
};

}  // namespace velo
