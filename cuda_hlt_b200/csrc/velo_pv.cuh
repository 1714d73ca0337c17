// Stage after the chain (optional, velo_set_pv): the beamline primary-vertex finder of
// cuda/PV/beamlinePV (pv_beamline_extrapolate, pv_beamline_histo, pv_beamline_peak,
// pv_beamline_multi_fitter: DefaultSequence.h:20-23) on the Kalman beamline states, as one
// kernel with one 128-thread block per event:
//   1. every track is extrapolated to its point of closest approach to the beamline
//      (pv_beamline_extrapolate.cu:3-30, the PVTrack constructor of
//      TrackBeamLineVertexFinder.cuh:9-31) into a scratch array;
//   2. the z histogram (2400 bins of 0.25 mm) lives in shared memory only: each warp owns a
//      quarter of the bins and adds every track's contributions to them, tracks in order, a
//      track's bins over the lanes. The reference adds with float atomics into global memory
//      (pv_beamline_histo.cu:14-76), so its bins carry an arbitrary summation order; these
//      are reproducible. Each bin receives the same per-track contributions,
//      G(bin) - G(bin - 1) of the polynomial Gaussian integral G;
//   3. warp 0 finds the peaks (pv_beamline_peak.cu:3-147) on the shared histogram: the
//      proto-clusters from ballots over the bins, their extrema walked a lane each;
//   4. a warp per seed fits its vertex (pv_beamline_multi_fitter.cu:6-183), the tracks over
//      the lanes (the reference: a thread per seed), the sums reduced across the warp in a
//      fixed order; vertices stored in seed order (the reference appends them with an atomic).
// The float expressions keep the reference's order, so they round as its kernels do under
// the same compiler flags, except the order of the sums over bins and tracks. Kept as in the reference: a vertex counts every track of its
// event in n_tracks (the track weights of the fit are not kept), so the 5-track cut applies
// to the event's track count. Beyond the reference's fixed arrays (32 peaks per event, 32
// extrema per proto-cluster, 200 cluster edges and clusters, 50 subclusters), where it writes
// past them, this stage keeps the first ones and flags VELO_STATUS_PV_OVERFLOW.
#pragma once
#include "velo_kernels.cuh"

namespace velo {

// BeamlinePVConstants.cuh:3-25, PV_Definitions.cuh:8-17
constexpr int kPvBins = 2400;
constexpr float kPvZmin = -300.f;
constexpr float kPvZmax = 300.f;
constexpr float kPvDz = 0.25f;
constexpr float kPvMaxTrackZ0Err = 1.5f;
constexpr float kPvMinDensity = 1.0f;
constexpr float kPvMinDipDensity = 2.0f;
constexpr float kPvMinTracksInSeed = 2.5f;
constexpr float kPvMaxVertexRho2 = 0.09f;
constexpr unsigned kPvMaxFitIter = 2;
constexpr float kPvMaxDeltaChi2 = 9.f;
constexpr float kPvMinWeight = 0.3f;
constexpr int kPvOrderPolynomial = 2;
constexpr unsigned kPvMinTracksPerVertex = 5;
constexpr uint32_t kPvMaxVertices = 32;
constexpr uint32_t kPvMaxClusters = 200;
constexpr uint32_t kPvMaxSubclusters = 50;
constexpr uint32_t kPvMaxEdges = 200;
constexpr uint32_t kPvThreads = 128;
constexpr uint32_t kPvWarps = kPvThreads / 32;
constexpr uint32_t kStatusPvOverflow = 1u << 13;

// A track at its point of closest approach to the beamline (PVTrack).
struct PvTrack {
  float z, x, y, tx, ty, w00, w11;
};

// Vertex record of the output, PV::Vertex's layout (PV_Definitions.cuh:64-109).
struct PvVertex {
  float x, y, z;
  float chi2;
  int32_t ndof;  // left unset by the reference; 0 here
  uint32_t n_tracks;
  float cov00, cov10, cov11, cov20, cov21, cov22;
  int32_t n_tracks_unused;  // nTracks, never set by the reference
};
static_assert(sizeof(PvVertex) == 52, "PV::Vertex layout");

struct PvPointers {
  const char* kalman;  // Kalman beamline states, States SoA of T tracks
  PvTrack* tracks;     // [T] scratch
  PvVertex* vertices;  // [N * 32]
  uint32_t* n_vertices;
  float* zpeaks;  // [N * 32]
  uint32_t* n_peaks;
};

// gauss_integral of pv_beamline_histo.cu:3-12 (polynomial of order 2)
__device__ __forceinline__ float pv_gauss_integral(float x)
{
  const float a = sqrtf(float(2 * kPvOrderPolynomial + 3));
  const float xi = x / a;
  const float eta = 1.f - xi * xi;
  return 0.5f + xi * (0.5f + eta * (0.25f + eta * 0.1875f));
}

// Contribution of a track to bin i of its window [minbin, maxbin]: the difference of the
// integral at the bin's upper edge and at the previous bin's (0 before the first bin; the
// last bin receives the rest up to 1).
__device__ __forceinline__ float pv_bin_contribution(const PvTrack& t, float zerr, int minbin, int maxbin, int i)
{
  auto g = [&](int b) { return pv_gauss_integral((kPvZmin + (b + 1) * kPvDz - t.z) / zerr); };
  const float below = i > minbin ? g(i - 1) : 0.f;
  return (i < maxbin ? g(i) : 1.f) - below;
}

struct PvExtremum {
  uint16_t index;
  float value, integral;
};

constexpr uint32_t kPvMaxToggles = 512;  // changes between empty and filled bins kept

constexpr int kPvBinsPerWarp = kPvBins / kPvWarps;

struct PvSmem {
  float histo[kPvBins];
  float zpeaks[kPvMaxVertices];
  uint32_t n_peaks, flags;
  uint16_t tog[kPvMaxToggles];
  uint16_t proto[kPvMaxEdges / 2][2];
  uint16_t izmax[kPvMaxClusters];
  PvVertex vtx[kPvMaxVertices];
  uint32_t vkeep[kPvMaxVertices];
};

__global__ void __launch_bounds__(kPvThreads) pv_beamline_kernel(ChainPointers P, PvPointers V)
{
  __shared__ PvSmem s;
  const uint32_t e = blockIdx.x;
  const uint32_t N = P.run->n_events;
  if (e >= N) return;
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  const uint32_t T = P.atomics[2 * N];
  const uint32_t nt = P.atomics[e];
  const uint32_t t0 = P.atomics[N + e];
  const float* K = reinterpret_cast<const float*>(V.kalman);
  PvTrack* tracks = V.tracks + t0;

  // ---- 1. extrapolation to the beamline (x, y) = (0, 0) ----
  for (uint32_t i = threadIdx.x; i < nt; i += kPvThreads) {
    const uint32_t k = t0 + i;
    const float x = K[k], y = K[T + k], tx = K[2 * T + k], ty = K[3 * T + k];
    const float c00 = K[4 * T + k], c20 = K[5 * T + k], c22 = K[6 * T + k];
    const float c11 = K[7 * T + k], c31 = K[8 * T + k], c33 = K[9 * T + k], z = K[11 * T + k];
    const float dz = (tx * (0.f - x) + ty * (0.f - y)) / (tx * tx + ty * ty);
    PvTrack t;
    t.z = float(z + dz);
    t.x = float(x + dz * tx);
    t.y = float(y + dz * ty);
    t.tx = tx;
    t.ty = ty;
    float a00 = c00, a11 = c11;
    const float dz2 = dz * dz;
    a00 += dz2 * c22 + 2.f * dz * c20;
    a11 += dz2 * c33 + 2.f * dz * c31;
    t.w00 = 1.f / a00;
    t.w11 = 1.f / a11;
    tracks[i] = t;
  }
  for (uint32_t b = threadIdx.x; b < kPvBins; b += kPvThreads) s.histo[b] = 0.f;
  if (threadIdx.x == 0) {
    s.n_peaks = 0;
    s.flags = 0;
  }
  __syncthreads();

  // ---- 2. z histogram: warp w fills bins [w * 600, (w + 1) * 600) from every track, in order ----
  {
    float* h = s.histo;
    const int own_lo = static_cast<int>(warp) * kPvBinsPerWarp, own_hi = own_lo + kPvBinsPerWarp - 1;
    for (uint32_t i = 0; i < nt; ++i) {
      const PvTrack t = tracks[i];
      if (!(kPvZmin < t.z && t.z < kPvZmax)) continue;
      const float zbin = (t.z - kPvZmin) / kPvDz;
      const float zweight = t.tx * t.tx * t.w00 + t.ty * t.ty * t.w11;
      const float zerr = 1.f / sqrtf(zweight);
      if (!(zerr < kPvMaxTrackZ0Err)) continue;
      const float a = sqrtf(float(2 * kPvOrderPolynomial + 3));
      const float halfwindow = a * zerr / kPvDz;
      const int minbin = max(int(zbin - halfwindow), 1);
      const int maxbin = min(int(zbin + halfwindow), kPvBins - 2);
      const int first = max(minbin, own_lo), last = min(maxbin, own_hi);
      for (int b = first + static_cast<int>(lane); b <= last; b += 32)
        h[b] += pv_bin_contribution(t, zerr, minbin, maxbin, b);
      __syncwarp();
    }
  }
  __syncthreads();

  // ---- 3. peaks (warp 0) ----
  // (a) The reference scans the bins once (pv_beamline_peak.cu:18-41): at every change
  // between empty and filled bins (starting from "empty" before bin 1) it opens a
  // proto-cluster, and at the next change it keeps it if the histogram integral since the
  // opening bin exceeds minTracksInSeed, otherwise drops it. The changes come here from
  // ballots over the bins; each proto-cluster's integral is summed in bin order by one lane.
  // (b) Per kept proto-cluster one lane walks its extrema and splits it into subclusters
  // (:43-119); (c) the cluster means (:128-137), in bin order.
  const float* zh = s.histo;
  if (warp == 0) {
    uint32_t flags = 0;
    const float inv_max_err = 1.f / (10.f * kPvMaxTrackZ0Err);
    const float threshold = kPvDz * inv_max_err;
    uint32_t n_tog = 0;
    for (uint32_t c = 0; c < (kPvBins + 31) / 32; ++c) {
      const int i = static_cast<int>(c * 32 + lane);
      bool tog = false;
      if (i >= 1 && i < kPvBins) {
        const bool empty = zh[i] < threshold;
        const bool prev = i == 1 ? true : zh[i - 1] < threshold;
        tog = empty != prev;
      }
      const uint32_t bal = __ballot_sync(0xFFFFFFFFu, tog);
      if (tog) {
        const uint32_t k = n_tog + __popc(bal & ((1u << lane) - 1u));
        if (k < kPvMaxToggles) s.tog[k] = static_cast<uint16_t>(i);
      }
      n_tog += __popc(bal);
    }
    __syncwarp();  // the toggles written by other lanes are read below
    if (n_tog > kPvMaxToggles) flags |= kStatusPvOverflow;
    const uint32_t n_open = min(n_tog, kPvMaxToggles) / 2;  // toggles alternate: open, close
    uint32_t n_proto = 0;
    for (uint32_t m0 = 0; m0 < n_open; m0 += 32) {
      const uint32_t m = m0 + lane;
      bool keep = false;
      if (m < n_open) {
        float integral = 0;
        for (uint32_t j = s.tog[2 * m] + 1u; j <= s.tog[2 * m + 1]; ++j) integral += zh[j];
        keep = integral > kPvMinTracksInSeed;
      }
      const uint32_t bal = __ballot_sync(0xFFFFFFFFu, keep);
      if (keep) {
        const uint32_t k = n_proto + __popc(bal & ((1u << lane) - 1u));
        if (k < kPvMaxEdges / 2) {
          s.proto[k][0] = s.tog[2 * m];
          s.proto[k][1] = s.tog[2 * m + 1];
        }
      }
      n_proto += __popc(bal);
    }
    __syncwarp();
    if (n_proto > kPvMaxEdges / 2) flags |= kStatusPvOverflow;
    n_proto = min(n_proto, kPvMaxEdges / 2);
    const float mindip = kPvMinDipDensity * kPvDz;
    const float minpeak = kPvMinDensity * kPvDz;
    uint32_t n_clusters = 0;
    for (uint32_t p0 = 0; p0 < n_proto; p0 += 32) {
      const uint32_t pc = p0 + lane;
      uint16_t izm[kPvMaxSubclusters];
      uint32_t nz = 0;
      if (pc < n_proto) {
        const uint16_t ibegin = s.proto[pc][0], iend = s.proto[pc][1];
        PvExtremum ex[kPvMaxVertices];
        int n_ex = 0;
        auto push = [&](uint16_t idx, float value, float integ) {
          if (n_ex < static_cast<int>(kPvMaxVertices)) ex[n_ex] = PvExtremum{idx, value, integ};
          else flags |= kStatusPvOverflow;
          ++n_ex;
        };
        bool rising = true;
        float integral = zh[ibegin];
        push(ibegin, zh[ibegin], integral);
        for (uint16_t i = ibegin; i < iend; ++i) {
          const float value = zh[i];
          const bool stillrising = zh[i + 1] > value;
          if (rising && !stillrising && value >= minpeak) {
            const int n = min(n_ex, static_cast<int>(kPvMaxVertices));
            if (n >= 2) {
              const float dv1 = ex[n - 2].value - ex[n - 1].value;
              const float dv2 = value - ex[n - 1].value;
              if (dv1 > mindip && dv2 > mindip) {
                push(i, value, integral + 0.5f * value);
              } else if (dv1 > dv2) {
                n_ex = max(n_ex - 1, 0);
              } else {
                n_ex = max(n_ex - 2, 0);
                push(i, value, integral + 0.5f * value);
              }
            } else {
              push(i, value, integral + 0.5f * value);
            }
          } else if (rising != stillrising) {
            push(i, value, integral + 0.5f * value);
          }
          rising = stillrising;
          integral += value;
        }
        push(iend, zh[iend], integral);
        const int n = min(n_ex, static_cast<int>(kPvMaxVertices));
        if (n > 3) {
          for (int i = 1; i < n / 2 + 1; ++i) {
            if (2 * i < n && ex[2 * i].integral - ex[2 * i - 2].integral > kPvMinTracksInSeed) {
              if (nz < kPvMaxSubclusters) izm[nz++] = ex[2 * i - 1].index;
              else flags |= kStatusPvOverflow;
            }
          }
        }
        if (nz == 0 && n > 1 && ex[1].value >= minpeak) izm[nz++] = ex[1].index;
      }
      // clusters in proto-cluster order
      uint32_t incl = nz;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= static_cast<uint32_t>(o)) incl += t;
      }
      for (uint32_t j = 0; j < nz; ++j) {
        const uint32_t k = n_clusters + incl - nz + j;
        if (k < kPvMaxClusters) s.izmax[k] = izm[j];
      }
      n_clusters += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    __syncwarp();
    if (n_clusters > kPvMaxClusters) flags |= kStatusPvOverflow;
    n_clusters = min(n_clusters, kPvMaxClusters);
    if (n_clusters > kPvMaxVertices) flags |= kStatusPvOverflow;
    const uint32_t n_peaks = min(n_clusters, kPvMaxVertices);
    if (lane < n_peaks) {
      const uint16_t izmax = s.izmax[lane];
      const float* b = zh + izmax;
      const float d1 = *b - *(b - 1);
      const float d2 = *b - *(b + 1);
      const float idz = d1 + d2 > 0 ? 0.5f * (d1 - d2) / (d1 + d2) : 0.0f;
      s.zpeaks[lane] = kPvZmin + kPvDz * (izmax + idz + 0.5f);
    }
    flags = __reduce_or_sync(0xFFFFFFFFu, flags);
    if (lane == 0) {
      s.n_peaks = n_peaks;
      s.flags = flags;
    }
  }
  __syncthreads();
  if (threadIdx.x < kPvMaxVertices)  // slots past the peaks hold 0
    V.zpeaks[e * kPvMaxVertices + threadIdx.x] = threadIdx.x < s.n_peaks ? s.zpeaks[threadIdx.x] : 0.f;
  if (threadIdx.x == 0) {
    V.n_peaks[e] = s.n_peaks;
    if (s.flags) P.status[e] |= s.flags;
  }

  // ---- 4. multi-vertex fit (pv_beamline_multi_fitter.cu:34-181): a warp per seed, the
  // tracks over the lanes, sums reduced across the warp in a fixed order ----
  const uint32_t n_seeds = s.n_peaks;
  for (uint32_t seed = warp; seed < n_seeds; seed += kPvWarps) {
    bool converged = false;
    float vtxcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float vx = 0.f, vy = 0.f;
    float vz = s.zpeaks[seed];
    const float max_dz_converged = 0.001f;
    float chi2tot = 0.f;
    for (uint32_t iter = 0; iter < kPvMaxFitIter && !converged; ++iter) {
      float a00 = 0.f, a11 = 0.f, a20 = 0.f, a21 = 0.f, a22 = 0.f;
      float gx = 0.f, gy = 0.f, gz = 0.f, c2 = 0.f;
      uint32_t nselected = 0;
      const float chi2_cut = 0.1f + 0.01f * kPvMaxFitIter / (iter + 1);
      const float denom0 = expf(-chi2_cut * 0.5f);
      for (uint32_t i = lane; i < nt; i += 32) {
        const PvTrack t = tracks[i];
        if (kPvZmin > t.z || t.z > kPvZmax) continue;
        const float dz = vz - t.z;
        const float rx = vx - (t.x + t.tx * dz);
        const float ry = vy - (t.y + t.ty * dz);
        const float chi2 = rx * rx * t.w00 + ry * ry * t.w11;
        if (chi2 < kPvMaxDeltaChi2) {
          ++nselected;
          float weight = expf(-chi2 * 0.5f);
          float denom = denom0;
          for (uint32_t o = 0; o < n_seeds; ++o) {
            const float odz = s.zpeaks[o] - t.z;
            const float ox = 0.f - (t.x + t.tx * odz);
            const float oy = 0.f - (t.y + t.ty * odz);
            const float ochi2 = ox * ox * t.w00 + oy * oy * t.w11;
            denom += expf(-ochi2 * 0.5f);
          }
          weight = weight / denom;
          if (weight < kPvMinWeight) continue;
          const float hx = rx * t.w00;
          const float hy = ry * t.w11;
          const float hz = -t.tx * rx * t.w00 - t.ty * ry * t.w11;
          gx = gx + hx * weight;
          gy = gy + hy * weight;
          gz = gz + hz * weight;
          // HWH of PVTrackInVertex (TrackBeamLineVertexFinder.cuh:57-75)
          const float h20 = -t.tx, h21 = -t.ty;
          a00 += weight * t.w00;
          a11 += weight * t.w11;
          a20 += weight * (h20 * t.w00);
          a21 += weight * (h21 * t.w11);
          a22 += weight * (h20 * h20 * t.w00 + h21 * h21 * t.w11);
          c2 += weight * chi2;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        a00 += __shfl_xor_sync(0xFFFFFFFFu, a00, o);
        a11 += __shfl_xor_sync(0xFFFFFFFFu, a11, o);
        a20 += __shfl_xor_sync(0xFFFFFFFFu, a20, o);
        a21 += __shfl_xor_sync(0xFFFFFFFFu, a21, o);
        a22 += __shfl_xor_sync(0xFFFFFFFFu, a22, o);
        gx += __shfl_xor_sync(0xFFFFFFFFu, gx, o);
        gy += __shfl_xor_sync(0xFFFFFFFFu, gy, o);
        gz += __shfl_xor_sync(0xFFFFFFFFu, gz, o);
        c2 += __shfl_xor_sync(0xFFFFFFFFu, c2, o);
        nselected += __shfl_xor_sync(0xFFFFFFFFu, nselected, o);
      }
      chi2tot = c2;
      if (nselected >= 2) {
        const float det = a00 * (a22 * a11 - a21 * a21) + a20 * (-a11 * a20);
        const float inv_det = 1.f / det;
        vtxcov[0] = (a22 * a11 - a21 * a21) * inv_det;
        vtxcov[1] = -(-a20 * a21) * inv_det;
        vtxcov[2] = (a22 * a00 - a20 * a20) * inv_det;
        vtxcov[3] = (-a20 * a11) * inv_det;
        vtxcov[4] = -(a21 * a00) * inv_det;
        vtxcov[5] = (a11 * a00) * inv_det;
        const float dx = -1.f * (vtxcov[0] * gx + vtxcov[1] * gy + vtxcov[3] * gz);
        const float dy = -1.f * (vtxcov[1] * gx + vtxcov[2] * gy + vtxcov[4] * gz);
        const float dzv = -1.f * (vtxcov[3] * gx + vtxcov[4] * gy + vtxcov[5] * gz);
        chi2tot += dx * gx + dy * gy + dzv * gz;
        vx = vx + dx;
        vy = vy + dy;
        vz = vz + dzv;
        converged = fabsf(dzv) < max_dz_converged;
      } else {
        break;  // the reference's placeholder position is overwritten below
      }
    }
    if (lane == 0) {
      PvVertex v{};
      v.chi2 = chi2tot;
      v.x = vx;
      v.y = vy;
      v.z = vz;
      v.cov00 = vtxcov[0];
      v.cov10 = vtxcov[1];
      v.cov11 = vtxcov[2];
      v.cov20 = vtxcov[3];
      v.cov21 = vtxcov[4];
      v.cov22 = vtxcov[5];
      v.n_tracks = nt;  // every track of the event (the weights of fresh track copies are 1)
      s.vtx[seed] = v;
      s.vkeep[seed] = nt >= kPvMinTracksPerVertex && v.x * v.x + v.y * v.y < kPvMaxVertexRho2;
    }
  }
  __syncthreads();
  // kept vertices in seed order (the reference appends them with an atomic)
  if (warp == 0) {
    const bool keep = lane < n_seeds && s.vkeep[lane];
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, keep);
    const uint32_t stored = __popc(bal);
    if (keep) V.vertices[e * kPvMaxVertices + __popc(bal & ((1u << lane) - 1u))] = s.vtx[lane];
    if (lane >= stored) V.vertices[e * kPvMaxVertices + lane] = PvVertex{};
    if (lane == 0) V.n_vertices[e] = stored;
  }
}

}  // namespace velo
