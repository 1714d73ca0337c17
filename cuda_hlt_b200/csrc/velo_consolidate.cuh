// Kernels 3 and 4 of the chain: exclusive scans over the events, then consolidation of
// the tracks into the reference's output layout with the beamline least-squares state and
// the simplified Kalman state.
#pragma once
#include "velo_kernels.cuh"

namespace velo {

// Exclusive scans of tracks and track hits per event (single block), in the layout of
// copy_and_prefix_sum_single_block + the track-hit prefix sum (PrefixSumSingleBlock.cu:130-168).
__global__ void __launch_bounds__(1024) event_scan_kernel(ChainPointers P)
{
  __shared__ uint32_t s_warp_t[32], s_warp_h[32];
  const uint32_t N = P.run->n_events;
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

// Consolidation, beamline state and Kalman state of one event per warp. Tracks are
// taken 32 at a time, one per lane: an exclusive warp scan of their hit counts gives
// their slices of the output; the hits of the 32 tracks form one contiguous range of the
// Velo::Consolidated::Hits SoA, which the warp then writes in order (coalesced), each lane
// finding the track of an output position by binary search over the 32 offsets. The same
// loop keeps x, y, z of the range in shared memory (up to kConsolidateStage hits), from
// where the fits run per lane on their track's slice; a larger range (32 tracks averaging
// more than 16 hits) fits from per-lane copies instead.
constexpr uint32_t kConsolidateStage = 512;

template<int WPB>
__global__ void __launch_bounds__(WPB * 32) consolidate_fit_kernel(ChainPointers P)
{
  __shared__ uint32_t s_off[WPB][33];
  __shared__ float s_hit[WPB][3][kConsolidateStage];
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t e = blockIdx.x * WPB + warp;
  const uint32_t N = P.run->n_events;
  if (e >= N) return;
  const uint32_t T = P.atomics[2 * N];
  const uint32_t Htot = P.event_hit_offset[N];
  const uint32_t nt = P.atomics[e];
  const uint32_t t0 = P.atomics[N + e];
  const float4* H = P.hits.xyzp + P.event_hit_base[e];
  const uint32_t* ids = P.hits.id + P.event_hit_base[e];
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
    const uint32_t n_chunk = min(32u, nt - i0);  // tracks of this chunk
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= static_cast<uint32_t>(o)) incl += v;
    }
    const uint32_t chunk_hits = __shfl_sync(0xFFFFFFFFu, incl, 31);
    s_off[warp][lane] = incl - n;
    if (lane == 31) s_off[warp][32] = incl;
    __syncwarp();
    // coalesced write of the chunk's hit range [carry, carry + chunk_hits)
    const bool staged = chunk_hits <= kConsolidateStage;
    // four output positions per lane at a time: their dependent gathers (hit index, then
    // record and id) are in flight together. The track of a position: every track has hits,
    // so the tracks starting inside 32 consecutive positions are marked by one bit each (an
    // OR across the warp of the lanes' own starts) and counted with a popcount.
    const uint32_t my_start = lane < n_chunk ? s_off[warp][lane] : 0xFFFFFFFFu;
    uint32_t started = 0;  // tracks starting before the current group of 32 positions
    for (uint32_t base = 0; base < chunk_hits; base += 4 * 32) {  // warp-uniform
      const uint32_t j0 = base + lane;
      uint32_t hh[4];
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t p0 = base + 32 * u;  // first position of this group
        const uint32_t heads =
          __reduce_or_sync(0xFFFFFFFFu, my_start - p0 < 32u ? 1u << (my_start - p0) : 0u);
        const uint32_t j = p0 + lane;
        const uint32_t t = started + __popc(heads & (0xFFFFFFFFu >> (31 - lane))) - 1;  // track of j
        started += __popc(heads);
        hh[u] = j < chunk_hits ? track_hits[(i0 + t) * kMaxTrackSize + (j - s_off[warp][t])] : 0u;
      }
      float4 p[4];
      uint32_t id[4];
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        if (j0 + 32 * u < chunk_hits) {
          p[u] = H[hh[u]];
          id[u] = ids[hh[u]];
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint32_t j = j0 + 32 * u;
        if (j < chunk_hits) {
          ox[carry + j] = p[u].x;
          oy[carry + j] = p[u].y;
          oz[carry + j] = p[u].z;
          oid[carry + j] = id[u];
          if (staged) {
            s_hit[warp][0][j] = p[u].x;
            s_hit[warp][1][j] = p[u].y;
            s_hit[warp][2][j] = p[u].z;
          }
        }
      }
    }
    __syncwarp();
    if (i < nt) {
      const uint32_t hoff = carry + s_off[warp][lane];
      P.track_hit_number[t0 + i] = hoff;
      FitState beam, kal;
      if (staged) {
        const uint32_t o = s_off[warp][lane];
        beam = beamline_fit(&s_hit[warp][0][o], &s_hit[warp][1][o], &s_hit[warp][2][o], n);
        kal = kalman_fit(&s_hit[warp][0][o], &s_hit[warp][1][o], &s_hit[warp][2][o], n, beam);
      } else {
        float hx[kMaxTrackSize], hy[kMaxTrackSize], hz[kMaxTrackSize];
        for (uint32_t k = 0; k < n; ++k) {
          const float4 p = H[track_hits[i * kMaxTrackSize + k]];
          hx[k] = p.x;
          hy[k] = p.y;
          hz[k] = p.z;
        }
        beam = beamline_fit(hx, hy, hz, n);
        kal = kalman_fit(hx, hy, hz, n, beam);
      }
      store_state(P.states, T, t0 + i, beam);
      store_state(P.kalman_states, T, t0 + i, kal);
    }
    carry += chunk_hits;
    __syncwarp();
  }
}

}  // namespace velo
