// Stage after the chain (optional, velo_set_pv): the beamline primary-vertex finder of
// cuda/PV/beamlinePV (pv_beamline_extrapolate, pv_beamline_histo, pv_beamline_peak,
// pv_beamline_multi_fitter: DefaultSequence.h:20-23) on the Kalman beamline states, as one
// kernel with one 128-thread block per event:
//   1. every track is extrapolated to its point of closest approach to the beamline
//      (pv_beamline_extrapolate.cu:3-30, the PVTrack constructor of
//      TrackBeamLineVertexFinder.cuh:9-31) into a scratch array;
//   2. the z histogram (2400 bins of 0.25 mm) lives in shared memory only: each warp adds
//      its share of the tracks, in track order, into a histogram of its own (a track's bins
//      over the lanes), and the four are summed bin by bin in a fixed order. The reference
//      adds with float atomics into global memory (pv_beamline_histo.cu:14-76), so its bins
//      carry an arbitrary summation order; these are reproducible. Each bin receives the same
//      per-track contributions, G(bin) - G(bin - 1) of the polynomial Gaussian integral G;
//   3. one thread finds the peaks (pv_beamline_peak.cu:3-147) on the shared histogram;
//   4. warp 0 fits one vertex per seed, a lane per seed (pv_beamline_multi_fitter.cu:6-183),
//      vertices stored in seed order (the reference appends them with an atomic).
// The float expressions keep the reference's order, so they round as its kernels do under
// the same compiler flags. Kept as in the reference: a vertex counts every track of its
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

struct PvSmem {
  float histo[kPvWarps][kPvBins];  // per-warp histograms; histo[0] holds the sum
  float zpeaks[kPvMaxVertices];
  uint32_t n_peaks, flags;
  uint16_t edges[kPvMaxEdges];
  uint16_t izmax[kPvMaxClusters];
};

__global__ void __launch_bounds__(kPvThreads) pv_beamline_kernel(ChainPointers P, PvPointers V)
{
  __shared__ PvSmem s;
  const uint32_t e = blockIdx.x;
  if (e >= P.n_events) return;
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  const uint32_t N = P.n_events;
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
  for (uint32_t b = threadIdx.x; b < kPvWarps * kPvBins; b += kPvThreads) (&s.histo[0][0])[b] = 0.f;
  if (threadIdx.x == 0) {
    s.n_peaks = 0;
    s.flags = 0;
  }
  __syncthreads();

  // ---- 2. z histogram: warp w adds tracks w, w + 4, ... in order, one bin per lane ----
  {
    float* h = s.histo[warp];
    for (uint32_t i = warp; i < nt; i += kPvWarps) {
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
      for (int b = minbin + static_cast<int>(lane); b <= maxbin; b += 32)
        h[b] += pv_bin_contribution(t, zerr, minbin, maxbin, b);
      __syncwarp();
    }
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < kPvBins; b += kPvThreads) {
    float v = s.histo[0][b];
#pragma unroll
    for (uint32_t w = 1; w < kPvWarps; ++w) v += s.histo[w][b];
    s.histo[0][b] = v;
  }
  __syncthreads();

  // ---- 3. peaks (one thread) ----
  const float* zh = s.histo[0];
  if (threadIdx.x == 0) {
    uint32_t flags = 0;
    uint32_t n_edges = 0, n_clusters = 0;
    {
      const float inv_max_err = 1.f / (10.f * kPvMaxTrackZ0Err);
      const float threshold = kPvDz * inv_max_err;
      bool prevempty = true;
      float integral = zh[0];
      for (uint16_t i = 1; i < kPvBins; ++i) {
        integral += zh[i];
        const bool empty = zh[i] < threshold;
        if (empty != prevempty) {
          if (prevempty || integral > kPvMinTracksInSeed) {
            if (n_edges < kPvMaxEdges) s.edges[n_edges] = i;
            else flags |= kStatusPvOverflow;
            ++n_edges;
          } else {
            --n_edges;
          }
          prevempty = empty;
          integral = 0;
        }
      }
    }
    const uint32_t n_proto = min(n_edges, kPvMaxEdges) / 2;
    const float mindip = kPvMinDipDensity * kPvDz;
    const float minpeak = kPvMinDensity * kPvDz;
    for (uint32_t c = 0; c < n_proto; ++c) {
      const uint16_t ibegin = s.edges[2 * c], iend = s.edges[2 * c + 1];
      PvExtremum ex[kPvMaxVertices];
      int n_ex = 0;
      auto push = [&](uint16_t idx, float value, float integ) {
        if (n_ex < static_cast<int>(kPvMaxVertices)) ex[n_ex] = PvExtremum{idx, value, integ};
        else flags |= kStatusPvOverflow;
        ++n_ex;
      };
      {
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
      }
      const int n = min(n_ex, static_cast<int>(kPvMaxVertices));
      uint32_t n_sub = 0;
      uint16_t sub_izmax[kPvMaxSubclusters];
      if (n > 3) {
        for (int i = 1; i < n / 2 + 1; ++i) {
          if (2 * i < n && ex[2 * i].integral - ex[2 * i - 2].integral > kPvMinTracksInSeed) {
            if (n_sub < kPvMaxSubclusters) sub_izmax[n_sub++] = ex[2 * i - 1].index;
            else flags |= kStatusPvOverflow;
          }
        }
      }
      if (n_sub == 0) {
        if (n > 1 && ex[1].value >= minpeak) {
          if (n_clusters < kPvMaxClusters) s.izmax[n_clusters++] = ex[1].index;
          else flags |= kStatusPvOverflow;
        }
      } else {
        for (uint32_t i = 0; i < n_sub; ++i) {
          if (n_clusters < kPvMaxClusters) s.izmax[n_clusters++] = sub_izmax[i];
          else flags |= kStatusPvOverflow;
        }
      }
    }
    // cluster means (zClusterMean, pv_beamline_peak.cu:128-137)
    uint32_t n_peaks = 0;
    for (uint32_t c = 0; c < n_clusters; ++c) {
      const uint16_t izmax = s.izmax[c];
      const float* b = zh + izmax;
      const float d1 = *b - *(b - 1);
      const float d2 = *b - *(b + 1);
      const float idz = d1 + d2 > 0 ? 0.5f * (d1 - d2) / (d1 + d2) : 0.0f;
      if (n_peaks < kPvMaxVertices) s.zpeaks[n_peaks++] = kPvZmin + kPvDz * (izmax + idz + 0.5f);
      else flags |= kStatusPvOverflow;
    }
    s.n_peaks = n_peaks;
    s.flags = flags;
  }
  __syncthreads();
  if (threadIdx.x < kPvMaxVertices)  // slots past the peaks hold 0
    V.zpeaks[e * kPvMaxVertices + threadIdx.x] = threadIdx.x < s.n_peaks ? s.zpeaks[threadIdx.x] : 0.f;
  if (threadIdx.x == 0) {
    V.n_peaks[e] = s.n_peaks;
    if (s.flags) P.status[e] |= s.flags;
  }

  // ---- 4. multi-vertex fit: warp 0, a lane per seed ----
  if (warp != 0) return;
  const uint32_t n_seeds = s.n_peaks;
  PvVertex vertex{};  // one per lane for all its seeds, as in the reference
  uint32_t stored = 0;
  for (uint32_t seed0 = 0; seed0 < n_seeds; seed0 += 32) {
    const uint32_t seed = seed0 + lane;
    bool keep = false;
    if (seed < n_seeds) {
      bool converged = false;
      float vtxcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float vx = 0.f, vy = 0.f;
      float vz = s.zpeaks[seed];
      const float max_dz_converged = 0.001f;
      float chi2tot = 0.f;
      uint32_t nselected = 0;
      for (uint32_t iter = 0; iter < kPvMaxFitIter && !converged; ++iter) {
        float a00 = 0.f, a11 = 0.f, a20 = 0.f, a21 = 0.f, a22 = 0.f;
        float gx = 0.f, gy = 0.f, gz = 0.f;
        chi2tot = 0.f;
        nselected = 0;
        for (uint32_t i = 0; i < nt; ++i) {
          const PvTrack t = tracks[i];
          if (kPvZmin > t.z || t.z > kPvZmax) continue;
          const float dz = vz - t.z;
          const float rx = vx - (t.x + t.tx * dz);
          const float ry = vy - (t.y + t.ty * dz);
          const float chi2 = rx * rx * t.w00 + ry * ry * t.w11;
          if (chi2 < kPvMaxDeltaChi2) {
            ++nselected;
            const float chi2_cut = 0.1f + 0.01f * kPvMaxFitIter / (iter + 1);
            float weight = expf(-chi2 * 0.5f);
            float denom = expf(-chi2_cut * 0.5f);
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
            chi2tot += weight * chi2;
          }
        }
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
      vertex.chi2 = chi2tot;
      vertex.x = vx;
      vertex.y = vy;
      vertex.z = vz;
      vertex.cov00 = vtxcov[0];
      vertex.cov10 = vtxcov[1];
      vertex.cov11 = vtxcov[2];
      vertex.cov20 = vtxcov[3];
      vertex.cov21 = vtxcov[4];
      vertex.cov22 = vtxcov[5];
      vertex.n_tracks += nt;  // every track of the event (weights of fresh track copies are 1)
      const float rho2 = vertex.x * vertex.x + vertex.y * vertex.y;
      keep = vertex.n_tracks >= kPvMinTracksPerVertex && rho2 < kPvMaxVertexRho2;
    }
    uint32_t n_keep;
    const uint32_t b = __ballot_sync(0xFFFFFFFFu, keep);
    n_keep = __popc(b);
    if (keep) V.vertices[e * kPvMaxVertices + stored + __popc(b & ((1u << lane) - 1u))] = vertex;
    stored += n_keep;
  }
  for (uint32_t k = stored + lane; k < kPvMaxVertices; k += 32) V.vertices[e * kPvMaxVertices + k] = PvVertex{};
  if (lane == 0) V.n_vertices[e] = stored;
}

}  // namespace velo
