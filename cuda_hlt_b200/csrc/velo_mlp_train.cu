// Training of the learned seed/extension scorer on the GPU (include/velo_b200.h,
// velo_mlp_*): sample collection from plain runs of the chain, forward and backward passes
// of 128-sample tiles on the tensor cores (tcgen05, bf16 operands, fp32 accumulators in
// tensor memory), and Adam on fp32 master weights.
//
// No counterpart in the reference. Loss: mean binary cross-entropy of the two logits
// against the labels the plain search gives each seeding candidate h1:
//   label 0  h1 lies on a final track of the plain search ("seed keep"),
//   label 1  h1 is the fourth or a later hit of a final track ("extension keep").
//
// One training tile (128 samples, one per thread):
//   forward   D1 = X W1^T, H1 = relu(D1); D2 = H1 W2^T, H2 = relu(D2); Z = H2 W3^T
//   backward  dZ = (sigmoid(Z) - Y) / (2 B); dH2 = (dZ W3) . [D2 > 0]; dH1 = (dH2 W2) . [D1 > 0]
//   gradients G1 += [X^T; H1^T] [dH1^T; dH2^T]^T  (dW1^T in rows 0..15, cols 0..63;
//                                                  dW2^T in rows 16..95, cols 64..127)
//             G2 += H2^T dZ                        (dW3^T in rows 0..79)
// with the bias of each layer as the weight of a constant-1 input column, so its gradient
// comes out of the same GEMM. The weight-gradient GEMMs contract over the samples: their
// operands are the activations transposed into K-major tiles (K = the 128 samples).
// Per-CTA gradient sums go to a partial buffer that the Adam kernel adds in a fixed order,
// so a training run is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/velo_b200.h"
#include "velo_ctx.hpp"
#include "velo_mlp.cuh"

using namespace velo;

namespace {

constexpr uint32_t kSboT = (kMlpTile / 8) * 128;  // 2048: K-major tiles over the 128 samples
constexpr uint32_t kTrainTmemCols = 256;
constexpr uint32_t kTmemFwd = 0;    // D1, D2, Z, dH2, dH1 in turn (64 columns)
constexpr uint32_t kTmemG1 = 64;    // 128 columns
constexpr uint32_t kTmemG2 = 192;   // 16 columns
constexpr uint32_t kW1 = 0, kW2 = kMlpW1, kW3 = kMlpW1 + kMlpW2;

struct __align__(128) MlpTrainSmem {
  uint8_t w1[kMlpW1 * 2];              // B of layer 1: W1 [64][16]
  uint8_t w2[kMlpW2 * 2];              // B of layer 2: W2 [64][80]
  uint8_t w3[kMlpW3 * 2];              // B of layer 3: W3 [16][80]
  uint8_t w3t[64 * 16 * 2];            // B of dH2 = dZ W3: W3^T [64][16]
  uint8_t w2t[64 * 64 * 2];            // B of dH1 = dH2 W2: W2^T [64][64]
  uint8_t x[kMlpTile * kMlpK1 * 2];    // A: X
  uint8_t h1[kMlpTile * kMlpK2 * 2];   // A: H1 with the ones column
  uint8_t h2[kMlpTile * kMlpK2 * 2];   // A: H2 with the ones column
  uint8_t dz[kMlpTile * 16 * 2];       // A: dZ
  uint8_t dh2[kMlpTile * 64 * 2];      // A: dH2
  uint8_t at[128 * kMlpTile * 2];      // A of G1: [X^T (16 rows); H1^T (80 rows); zeros]
  uint8_t bt[128 * kMlpTile * 2];      // B of G1: [dH1^T (64 rows); dH2^T (64 rows)]
  uint8_t a2t[128 * kMlpTile * 2];     // A of G2: [H2^T (80 rows); zeros]
  uint8_t b2t[16 * kMlpTile * 2];      // B of G2: dZ^T (rows 0, 1; zeros)
  uint64_t mbar;
  uint32_t tmem;
  float norm[32];
  float red[4];
};
constexpr size_t kTrainSmem = sizeof(MlpTrainSmem) + 128;

struct TrainArgs {
  const float* feat;         // [n][12]
  const uint8_t* lab;        // [n] label bits
  const uint32_t* perm;      // sample order
  uint64_t first;            // first position of this step's batch in perm
  uint32_t batch;            // samples of this step
  float inv_count;           // 1 / (2 * batch)
  const __nv_bfloat16* w;    // [kMlpParams]
  const __nv_bfloat16* w2t;  // [64][64]
  const __nv_bfloat16* w3t;  // [64][16]
  const float* norm;         // mean[16], inv_std[16]
  float* partial;            // [gridDim.x][kMlpParams]
  float* loss;               // [gridDim.x] summed cross-entropy of the CTA's samples
  uint32_t* error;
};

__device__ __forceinline__ uint8_t* align128(uint8_t* p)
{
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 127) & ~uintptr_t(127));
}

__device__ __forceinline__ void store_bf16(uint8_t* tile, uint32_t off, float v)
{
  *reinterpret_cast<__nv_bfloat16*>(tile + off) = __float2bfloat16_rn(v);
}

// Stores a row of N values (bf16, N a multiple of 8) into a canonical tile.
template<int N>
__device__ __forceinline__ void store_row(uint8_t* tile, uint32_t row, uint32_t sbo, const float (&v)[N])
{
#pragma unroll
  for (uint32_t kb = 0; kb < N / 8; ++kb) {
    uint4 q;
    q.x = pack_bf16x2(v[8 * kb + 0], v[8 * kb + 1]);
    q.y = pack_bf16x2(v[8 * kb + 2], v[8 * kb + 3]);
    q.z = pack_bf16x2(v[8 * kb + 4], v[8 * kb + 5]);
    q.w = pack_bf16x2(v[8 * kb + 6], v[8 * kb + 7]);
    *reinterpret_cast<uint4*>(tile + canon_off(row, kb, sbo)) = q;
  }
}

__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64])
{
#pragma unroll
  for (int c = 0; c < 4; ++c) tmem_ld16(taddr + 16 * c, *reinterpret_cast<float(*)[16]>(v + 16 * c));
  tmem_ld_wait();
}

__global__ void __launch_bounds__(kMlpTile, 1) mlp_train_kernel(TrainArgs A)
{
  extern __shared__ uint8_t s_dyn[];
  MlpTrainSmem& s = *reinterpret_cast<MlpTrainSmem*>(align128(s_dyn));
  const uint32_t t = threadIdx.x;
  if (t < 32) tmem_alloc(&s.tmem, kTrainTmemCols);
  if (t == 0) mbar_init1(&s.mbar);
  if (t < 32) s.norm[t] = A.norm[t];
  load_canon(s.w1, A.w + kW1, kMlpHidden, kMlpK1);
  load_canon(s.w2, A.w + kW2, kMlpHidden, kMlpK2);
  load_canon(s.w3, A.w + kW3, kMlpOutPad, kMlpK2);
  load_canon(s.w3t, A.w3t, 64, 16);
  load_canon(s.w2t, A.w2t, 64, 64);
  // rows of the transposed operands that no sample writes stay zero
  for (uint32_t c = t; c < 32 * 16; c += kMlpTile) {
    const uint32_t row = c / 16, kb = c % 16;
    *reinterpret_cast<uint4*>(s.at + canon_off(96 + row, kb, kSboT)) = make_uint4(0, 0, 0, 0);
  }
  for (uint32_t c = t; c < 48 * 16; c += kMlpTile) {
    const uint32_t row = c / 16, kb = c % 16;
    *reinterpret_cast<uint4*>(s.a2t + canon_off(80 + row, kb, kSboT)) = make_uint4(0, 0, 0, 0);
  }
  for (uint32_t c = t; c < 16 * 16; c += kMlpTile) {
    const uint32_t row = c / 16, kb = c % 16;
    *reinterpret_cast<uint4*>(s.b2t + canon_off(row, kb, kSboT)) = make_uint4(0, 0, 0, 0);
  }
  umma_stage_barrier();
  const uint32_t lane_addr = s.tmem + ((t & ~31u) << 16);
  uint32_t phase = 0;
  float loss = 0.f;
  bool ok = true;
  uint32_t done = 0;
  const uint32_t tiles = (A.batch + kMlpTile - 1) / kMlpTile;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++done) {
    const uint32_t i = tile * kMlpTile + t;
    const bool valid = i < A.batch;
    float x[16];
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = 0.f;
    if (valid) {
      const uint32_t idx = A.perm[A.first + i];
#pragma unroll
      for (int k = 0; k < 12; ++k) x[k] = (A.feat[static_cast<size_t>(idx) * 12 + k] - s.norm[k]) * s.norm[16 + k];
      const uint8_t l = A.lab[idx];
      y0 = static_cast<float>(l & 1u);
      y1 = static_cast<float>((l >> 1) & 1u);
    }
    x[12] = 1.f;
    store_row<16>(s.x, t, kSbo1, x);
#pragma unroll
    for (uint32_t k = 0; k < 16; ++k) store_bf16(s.at, canon_elem(k, t, kSboT), x[k]);

    // ---- layer 1 ----
    umma_stage_barrier();
    if (t == 0) {
      umma_issue(s.tmem + kTmemFwd, s.x, kSbo1, s.w1, kSbo1, kMlpK1, kMlpHidden, false);
      umma_commit(&s.mbar);
    }
    if (!(ok = umma_wait(&s.mbar, phase))) break;
    uint32_t mask1[2] = {0u, 0u}, mask2[2] = {0u, 0u};
    {
      float v[64];
      tmem_ld64(lane_addr + kTmemFwd, v);
      float h[80];
#pragma unroll
      for (int k = 0; k < 64; ++k) {
        if (v[k] > 0.f) mask1[k >> 5] |= 1u << (k & 31);
        h[k] = fmaxf(v[k], 0.f);
      }
      h[64] = 1.f;
#pragma unroll
      for (int k = 65; k < 80; ++k) h[k] = 0.f;
      store_row<80>(s.h1, t, kSbo2, h);
#pragma unroll
      for (uint32_t k = 0; k < 80; ++k) store_bf16(s.at, canon_elem(16 + k, t, kSboT), h[k]);
    }
    // ---- layer 2 ----
    umma_stage_barrier();
    if (t == 0) {
      umma_issue(s.tmem + kTmemFwd, s.h1, kSbo2, s.w2, kSbo2, kMlpK2, kMlpHidden, false);
      umma_commit(&s.mbar);
    }
    if (!(ok = umma_wait(&s.mbar, phase))) break;
    {
      float v[64];
      tmem_ld64(lane_addr + kTmemFwd, v);
      float h[80];
#pragma unroll
      for (int k = 0; k < 64; ++k) {
        if (v[k] > 0.f) mask2[k >> 5] |= 1u << (k & 31);
        h[k] = fmaxf(v[k], 0.f);
      }
      h[64] = 1.f;
#pragma unroll
      for (int k = 65; k < 80; ++k) h[k] = 0.f;
      store_row<80>(s.h2, t, kSbo2, h);
#pragma unroll
      for (uint32_t k = 0; k < 80; ++k) store_bf16(s.a2t, canon_elem(k, t, kSboT), h[k]);
    }
    // ---- layer 3 ----
    umma_stage_barrier();
    if (t == 0) {
      umma_issue(s.tmem + kTmemFwd, s.h2, kSbo2, s.w3, kSbo2, kMlpK2, kMlpOutPad, false);
      umma_commit(&s.mbar);
    }
    if (!(ok = umma_wait(&s.mbar, phase))) break;
    {
      float z[16];
      tmem_ld16(lane_addr + kTmemFwd, z);
      tmem_ld_wait();
      float d[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) d[k] = 0.f;
      if (valid) {
        const float zz[2] = {z[0], z[1]}, yy[2] = {y0, y1};
#pragma unroll
        for (int o = 0; o < 2; ++o) {
          const float a = fabsf(zz[o]);
          loss += fmaxf(zz[o], 0.f) - zz[o] * yy[o] + log1pf(expf(-a));
          const float sig = 1.f / (1.f + expf(-zz[o]));
          d[o] = (sig - yy[o]) * A.inv_count;
        }
      }
      store_row<16>(s.dz, t, kSbo1, d);
      store_bf16(s.b2t, canon_elem(0, t, kSboT), d[0]);
      store_bf16(s.b2t, canon_elem(1, t, kSboT), d[1]);
    }
    // ---- dH2 = dZ W3, and G2 += H2^T dZ ----
    umma_stage_barrier();
    if (t == 0) {
      umma_issue(s.tmem + kTmemFwd, s.dz, kSbo1, s.w3t, kSbo1, 16, 64, false);
      umma_issue(s.tmem + kTmemG2, s.a2t, kSboT, s.b2t, kSboT, kMlpTile, 16, done > 0);
      umma_commit(&s.mbar);
    }
    if (!(ok = umma_wait(&s.mbar, phase))) break;
    {
      float v[64];
      tmem_ld64(lane_addr + kTmemFwd, v);
#pragma unroll
      for (int k = 0; k < 64; ++k) v[k] = ((mask2[k >> 5] >> (k & 31)) & 1u) ? v[k] : 0.f;
      store_row<64>(s.dh2, t, 1024u, v);
#pragma unroll
      for (uint32_t k = 0; k < 64; ++k) store_bf16(s.bt, canon_elem(64 + k, t, kSboT), v[k]);
    }
    // ---- dH1 = dH2 W2 ----
    umma_stage_barrier();
    if (t == 0) {
      umma_issue(s.tmem + kTmemFwd, s.dh2, 1024u, s.w2t, 1024u, 64, 64, false);
      umma_commit(&s.mbar);
    }
    if (!(ok = umma_wait(&s.mbar, phase))) break;
    {
      float v[64];
      tmem_ld64(lane_addr + kTmemFwd, v);
#pragma unroll
      for (uint32_t k = 0; k < 64; ++k)
        store_bf16(s.bt, canon_elem(k, t, kSboT), ((mask1[k >> 5] >> (k & 31)) & 1u) ? v[k] : 0.f);
    }
    // ---- G1 += [X^T; H1^T] [dH1^T; dH2^T]^T ----
    umma_stage_barrier();
    if (t == 0) {
      umma_issue(s.tmem + kTmemG1, s.at, kSboT, s.bt, kSboT, kMlpTile, 128, done > 0);
      umma_commit(&s.mbar);
    }
    if (!(ok = umma_wait(&s.mbar, phase))) break;
  }
  if (!ok && t == 0) atomicOr(A.error, 1u);
  // ---- per-CTA gradient sums (every slot written exactly once) ----
  float* part = A.partial + static_cast<size_t>(blockIdx.x) * kMlpParams;
  for (uint32_t c0 = 0; c0 < 128; c0 += 16) {
    float g[16];
    tmem_ld16(lane_addr + kTmemG1 + c0, g);
    tmem_ld_wait();
#pragma unroll
    for (uint32_t j = 0; j < 16; ++j) {
      const uint32_t col = c0 + j;
      const float v = (done > 0 && ok) ? g[j] : 0.f;
      if (t < 16 && col < 64) part[kW1 + col * kMlpK1 + t] = v;
      else if (t >= 16 && t < 96 && col >= 64) part[kW2 + (col - 64) * kMlpK2 + (t - 16)] = v;
    }
  }
  {
    float g[16];
    tmem_ld16(lane_addr + kTmemG2, g);
    tmem_ld_wait();
    if (t < 80)
#pragma unroll
      for (uint32_t o = 0; o < 16; ++o) part[kW3 + o * kMlpK2 + t] = (done > 0 && ok) ? g[o] : 0.f;
  }
  // loss of the CTA's samples
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
  if ((t & 31) == 0) s.red[t >> 5] = loss;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (t == 0) A.loss[blockIdx.x] = s.red[0] + s.red[1] + s.red[2] + s.red[3];
  if (t < 32) tmem_dealloc(s.tmem, kTrainTmemCols);
}

// Trainable slots: W1 columns 0..12, W2 columns 0..64, W3 rows 0..1 columns 0..64.
__device__ __forceinline__ bool trainable(uint32_t p)
{
  if (p < kW2) return (p % kMlpK1) <= kMlpFeatures;
  if (p < kW3) return ((p - kW2) % kMlpK2) <= kMlpHidden;
  const uint32_t q = p - kW3;
  return q / kMlpK2 < 2 && (q % kMlpK2) <= kMlpHidden;
}

struct AdamArgs {
  float* master;
  float* m;
  float* v;
  const float* partial;
  uint32_t parts;
  float lr, beta1, beta2, eps, bias1, bias2;  // bias = 1 - beta^step
  int update;
  __nv_bfloat16* w;
  __nv_bfloat16* w2t;
  __nv_bfloat16* w3t;
  float* grad_out;  // optional: summed gradient
  const float* loss;
  float* loss_total;  // += sum of the step's CTA losses
};

// Sums the per-CTA gradients in CTA order, applies one Adam step to the trainable slots
// and publishes the bf16 copies (row-major and the two transposed blocks).
__global__ void mlp_adam_kernel(AdamArgs A)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && A.loss_total) {
    float l = 0.f;
    for (uint32_t c = 0; c < A.parts; ++c) l += A.loss[c];
    *A.loss_total += l;
  }
  if (p >= kMlpParams) return;
  float g = 0.f;
  for (uint32_t c = 0; c < A.parts; ++c) g += A.partial[static_cast<size_t>(c) * kMlpParams + p];
  if (A.grad_out) A.grad_out[p] = g;
  float w = A.master[p];
  if (A.update && trainable(p)) {
    const float m = A.beta1 * A.m[p] + (1.f - A.beta1) * g;
    const float v = A.beta2 * A.v[p] + (1.f - A.beta2) * g * g;
    A.m[p] = m;
    A.v[p] = v;
    w -= A.lr * (m / A.bias1) / (sqrtf(v / A.bias2) + A.eps);
    A.master[p] = w;
  }
  const __nv_bfloat16 b = __float2bfloat16_rn(trainable(p) ? w : 0.f);
  A.w[p] = b;
  if (p >= kW2 && p < kW3) {
    const uint32_t j = (p - kW2) / kMlpK2, i = (p - kW2) % kMlpK2;
    if (i < 64) A.w2t[i * 64 + j] = b;
  } else if (p >= kW3) {
    const uint32_t o = (p - kW3) / kMlpK2, i = (p - kW3) % kMlpK2;
    if (i < 64) A.w3t[i * 16 + o] = b;
  }
}

// Inference over feature rows (the fill kernel's tile code): logits [n][2].
__global__ void __launch_bounds__(kMlpTile) mlp_infer_rows_kernel(MlpDevice mlp, const float* feat, uint32_t n,
                                                                  float* logits, uint32_t* error)
{
  extern __shared__ uint8_t s_dyn[];
  MlpInferSmem& sm = *reinterpret_cast<MlpInferSmem*>(align128(s_dyn));
  mlp_infer_setup(sm, mlp);
  uint32_t phase = 0;
  for (uint32_t tile = blockIdx.x; tile * kMlpTile < n; tile += gridDim.x) {
    const uint32_t i = tile * kMlpTile + threadIdx.x;
    float f[kMlpFeatures];
    for (int k = 0; k < 12; ++k) f[k] = i < n ? feat[static_cast<size_t>(i) * 12 + k] : 0.f;
    mlp_store_features(sm, f, i < n);
    float z0 = 0.f, z1 = 0.f;
    if (!mlp_tile_forward(sm, phase, z0, z1)) {
      if (threadIdx.x == 0) atomicOr(error, 1u);
      break;
    }
    if (i < n) {
      logits[2 * i] = z0;
      logits[2 * i + 1] = z1;
    }
  }
  mlp_infer_teardown(sm);
}

// ---- sample collection ----------------------------------------------------------
__device__ __forceinline__ bool event_runnable(const ChainPointers& P, uint32_t e)
{
  const uint32_t nhits = P.event_hits[e], status = P.status[e];
  return !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
}

__device__ __forceinline__ bool is_candidate(uint2 w) { return (w.x & 0xFFFFu) != 0xFFFFu && (w.y & 0xFFFFu) != 0xFFFFu; }

// Labels of one event's hits from the tracks of its plain search and its number of
// seeding candidates (h1 of modules 2..49 with both windows). One block per event.
__global__ void __launch_bounds__(256) collect_count_kernel(ChainPointers P, uint8_t* labels, uint32_t* counts)
{
  __shared__ uint32_t s_cnt;
  const uint32_t e = blockIdx.x;
  if (!event_runnable(P, e)) {
    if (threadIdx.x == 0) counts[e] = 0;
    return;
  }
  const uint32_t nhits = P.event_hits[e], base = P.event_hit_base[e];
  uint8_t* L = labels + base;
  if (threadIdx.x == 0) s_cnt = 0;
  for (uint32_t h = threadIdx.x; h < nhits; h += blockDim.x) L[h] = 0;
  __syncthreads();
  // a hit is on at most one track (the search marks hits used)
  const uint32_t nt = min(P.event_tracks[e], kMaxTracks);
  const uint16_t* tn = P.scratch.track_n + static_cast<size_t>(e) * kMaxTracks;
  const uint16_t* th = P.scratch.track_hits + static_cast<size_t>(e) * kMaxTracks * kMaxTrackSize;
  for (uint32_t t = threadIdx.x; t < nt; t += blockDim.x) {
    const uint32_t n = tn[t];
    for (uint32_t k = 0; k < n; ++k) L[th[t * kMaxTrackSize + k]] = k >= 3 ? 3u : 1u;
  }
  const uint32_t lo = P.module_start[e * kModules + 2] - base, hi = P.module_start[e * kModules + 50] - base;
  uint32_t c = 0;
  for (uint32_t h = lo + threadIdx.x; h < hi; h += blockDim.x) c += is_candidate(P.windows[base + h]);
  atomicAdd(&s_cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) counts[e] = s_cnt;
}

// Features and labels of the first take[e] candidates of each event, in hit order, at
// offsets[e]. One block of 256 per event.
__global__ void __launch_bounds__(256) collect_write_kernel(ChainPointers P, const uint8_t* labels,
                                                            const uint64_t* offsets, const uint32_t* take, float* feat,
                                                            uint8_t* lab)
{
  __shared__ uint32_t s_ms[kModules + 1];
  __shared__ uint32_t s_warp[8];
  const uint32_t e = blockIdx.x;
  const uint32_t want = take[e];
  if (want == 0) return;
  const uint32_t base = P.event_hit_base[e], nhits = P.event_hits[e];
  if (threadIdx.x < kModules) s_ms[threadIdx.x] = P.module_start[e * kModules + threadIdx.x] - base;
  if (threadIdx.x == 0) s_ms[kModules] = nhits;
  __syncthreads();
  const float4* H = P.hits.xyzp + base;
  const uint8_t* S = P.hit_size + base;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t written = 0;
  for (uint32_t t0 = s_ms[2]; t0 < s_ms[50] && written < want; t0 += 256) {
    const uint32_t h = t0 + threadIdx.x;
    uint2 w = make_uint2(0xFFFFu, 0xFFFFu);
    if (h < s_ms[50]) w = P.windows[base + h];
    const bool cand = h < s_ms[50] && is_candidate(w);
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, cand);
    if (lane == 0) s_warp[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (uint32_t k = 0; k < 8; ++k) {
      before += k < warp ? s_warp[k] : 0u;
      total += s_warp[k];
    }
    const uint32_t rank = written + before + __popc(bal & ((1u << lane) - 1u));
    if (cand && rank < want) {
      uint32_t a = 2, b = 50;
      while (b - a > 1) {
        const uint32_t mid = (a + b) >> 1;
        if (s_ms[mid] <= h) a = mid; else b = mid;
      }
      float f[kMlpFeatures];
      seed_features(H, S, h, a, static_cast<int>(w.x & 0xFFFFu), static_cast<int>(w.x >> 16),
                    static_cast<int>(w.y & 0xFFFFu), static_cast<int>(w.y >> 16), f);
      const uint64_t o = offsets[e] + rank;
      for (int k = 0; k < 12; ++k) feat[o * 12 + k] = f[k];
      lab[o] = labels[base + h] & 3u;
    }
    written += total;
    __syncthreads();
  }
}

}  // namespace

// ============================================================================
// Trainer
// ============================================================================
struct VeloMlpTrainer {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint64_t cap = 0, n = 0;
  float* d_feat = nullptr;
  uint8_t* d_lab = nullptr;
  uint32_t* d_perm = nullptr;
  float *d_master = nullptr, *d_m = nullptr, *d_v = nullptr, *d_norm = nullptr;
  __nv_bfloat16 *d_w = nullptr, *d_w2t = nullptr, *d_w3t = nullptr;
  float *d_partial = nullptr, *d_loss = nullptr, *d_loss_total = nullptr, *d_grad = nullptr;
  uint32_t* d_error = nullptr;
  uint8_t* d_hit_labels = nullptr;
  size_t hit_labels_cap = 0;
  uint32_t grid = 0;
  uint64_t step = 0;
  std::mt19937_64 rng;
  VeloMlpWeights meta{};  // normalisation and thresholds
};

#define TCK(x)                                                                                        \
  do {                                                                                                \
    cudaError_t e_ = (x);                                                                             \
    if (e_ != cudaSuccess) {                                                                          \
      std::fprintf(stderr, "velo_mlp: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return VELO_ERR_CUDA;                                                                           \
    }                                                                                                 \
  } while (0)

namespace {

template<class T>
cudaError_t talloc(T*& p, size_t count)
{
  return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T));
}

void trainer_free(VeloMlpTrainer* t)
{
  void* ptrs[] = {t->d_feat, t->d_lab, t->d_perm, t->d_master, t->d_m, t->d_v, t->d_norm, t->d_w, t->d_w2t, t->d_w3t,
                  t->d_partial, t->d_loss, t->d_loss_total, t->d_grad, t->d_error, t->d_hit_labels};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (t->stream) cudaStreamDestroy(t->stream);
}

// fp32 slots <-> the host struct (weights with the bias in the last column)
void weights_to_slots(const VeloMlpWeights& w, std::vector<float>& slots)
{
  slots.assign(kMlpParams, 0.f);
  for (int j = 0; j < 64; ++j)
    for (int i = 0; i < 13; ++i) slots[kW1 + j * kMlpK1 + i] = w.w1[j][i];
  for (int j = 0; j < 64; ++j)
    for (int i = 0; i < 65; ++i) slots[kW2 + j * kMlpK2 + i] = w.w2[j][i];
  for (int o = 0; o < 2; ++o)
    for (int i = 0; i < 65; ++i) slots[kW3 + o * kMlpK2 + i] = w.w3[o][i];
}
void slots_to_weights(const float* slots, VeloMlpWeights& w)
{
  for (int j = 0; j < 64; ++j)
    for (int i = 0; i < 13; ++i) w.w1[j][i] = slots[kW1 + j * kMlpK1 + i];
  for (int j = 0; j < 64; ++j)
    for (int i = 0; i < 65; ++i) w.w2[j][i] = slots[kW2 + j * kMlpK2 + i];
  for (int o = 0; o < 2; ++o)
    for (int i = 0; i < 65; ++i) w.w3[o][i] = slots[kW3 + o * kMlpK2 + i];
}

int upload_norm(VeloMlpTrainer* t)
{
  float norm[32] = {};
  for (int k = 0; k < 12; ++k) {
    norm[k] = t->meta.mean[k];
    norm[16 + k] = t->meta.inv_std[k];
  }
  TCK(cudaMemcpyAsync(t->d_norm, norm, sizeof norm, cudaMemcpyHostToDevice, t->stream));
  TCK(cudaStreamSynchronize(t->stream));  // the host array goes out of scope
  return 0;
}

// Publishes the bf16 copies of the master weights (Adam kernel; without `update` no step
// is taken); with `grad` the summed partials of `parts` CTAs are also written there.
int publish(VeloMlpTrainer* t, uint32_t parts, float* grad, int update, float lr)
{
  AdamArgs a{};
  a.master = t->d_master;
  a.m = t->d_m;
  a.v = t->d_v;
  a.partial = t->d_partial;
  a.parts = parts;
  a.lr = lr;
  a.beta1 = 0.9f;
  a.beta2 = 0.999f;
  a.eps = 1e-8f;
  a.bias1 = 1.f - std::pow(0.9f, static_cast<float>(std::max<uint64_t>(t->step, 1)));
  a.bias2 = 1.f - std::pow(0.999f, static_cast<float>(std::max<uint64_t>(t->step, 1)));
  a.update = update;
  a.w = t->d_w;
  a.w2t = t->d_w2t;
  a.w3t = t->d_w3t;
  a.grad_out = grad;
  a.loss = t->d_loss;
  a.loss_total = parts ? t->d_loss_total : nullptr;
  mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, t->stream>>>(a);
  TCK(cudaGetLastError());
  return 0;
}

int train_step(VeloMlpTrainer* t, const float* feat, const uint8_t* lab, const uint32_t* perm, uint64_t first,
               uint32_t batch, uint32_t* parts)
{
  TrainArgs a{};
  a.feat = feat;
  a.lab = lab;
  a.perm = perm;
  a.first = first;
  a.batch = batch;
  a.inv_count = 1.f / (2.f * static_cast<float>(batch));
  a.w = t->d_w;
  a.w2t = t->d_w2t;
  a.w3t = t->d_w3t;
  a.norm = t->d_norm;
  a.partial = t->d_partial;
  a.loss = t->d_loss;
  a.error = t->d_error;
  const uint32_t tiles = (batch + kMlpTile - 1) / kMlpTile;
  const uint32_t grid = std::min(t->grid, tiles);
  mlp_train_kernel<<<grid, kMlpTile, kTrainSmem, t->stream>>>(a);
  TCK(cudaGetLastError());
  *parts = grid;
  return 0;
}

int check_error(VeloMlpTrainer* t)
{
  uint32_t err = 0;
  TCK(cudaMemcpyAsync(&err, t->d_error, 4, cudaMemcpyDeviceToHost, t->stream));
  TCK(cudaStreamSynchronize(t->stream));
  return err ? VELO_ERR_DEVICE_TIMEOUT : 0;
}

}  // namespace

extern "C" {

int velo_mlp_trainer_create(int device, uint64_t max_samples, uint64_t seed, VeloMlpTrainer** out)
{
  if (!out || max_samples == 0) return VELO_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return VELO_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return VELO_ERR_INVALID;
  auto* t = new VeloMlpTrainer();
  t->device = device;
  t->cap = max_samples;
  t->rng.seed(seed);
  auto fail = [&](int code) {
    trainer_free(t);
    delete t;
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fail(VELO_ERR_CUDA);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  t->grid = static_cast<uint32_t>(std::max(1, sms));
  bool ok = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok &= talloc(t->d_feat, max_samples * 12) == cudaSuccess;
  ok &= talloc(t->d_lab, max_samples) == cudaSuccess;
  ok &= talloc(t->d_perm, max_samples) == cudaSuccess;
  ok &= talloc(t->d_master, kMlpParams) == cudaSuccess;
  ok &= talloc(t->d_m, kMlpParams) == cudaSuccess;
  ok &= talloc(t->d_v, kMlpParams) == cudaSuccess;
  ok &= talloc(t->d_norm, 32) == cudaSuccess;
  ok &= talloc(t->d_w, kMlpParams) == cudaSuccess;
  ok &= talloc(t->d_w2t, 64 * 64) == cudaSuccess;
  ok &= talloc(t->d_w3t, 64 * 16) == cudaSuccess;
  ok &= talloc(t->d_partial, static_cast<size_t>(t->grid) * kMlpParams) == cudaSuccess;
  ok &= talloc(t->d_loss, t->grid) == cudaSuccess;
  ok &= talloc(t->d_loss_total, 1) == cudaSuccess;
  ok &= talloc(t->d_grad, kMlpParams) == cudaSuccess;
  ok &= talloc(t->d_error, 1) == cudaSuccess;
  if (!ok) return fail(VELO_ERR_CUDA);
  ok &= cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kTrainSmem)) == cudaSuccess;
  ok &= cudaFuncSetAttribute(mlp_infer_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kMlpInferSmem)) == cudaSuccess;
  ok &= cudaMemset(t->d_error, 0, 4) == cudaSuccess;
  if (!ok) return fail(VELO_ERR_CUDA);
  // defaults: identity normalisation, seeded uniform(+-1/sqrt(fan_in)) weights, zero biases
  for (int k = 0; k < 12; ++k) {
    t->meta.mean[k] = 0.f;
    t->meta.inv_std[k] = 1.f;
  }
  t->meta.seed_threshold = 0.5f;
  t->meta.ext_threshold = 0.f;
  t->meta.max_event_clusters = 0xFFFFFFFFu;
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  VeloMlpWeights w = t->meta;
  for (int j = 0; j < 64; ++j) {
    for (int i = 0; i < 12; ++i) w.w1[j][i] = u(t->rng) / std::sqrt(12.f);
    w.w1[j][12] = 0.f;
    for (int i = 0; i < 64; ++i) w.w2[j][i] = u(t->rng) / 8.f;
    w.w2[j][64] = 0.f;
  }
  for (int o = 0; o < 2; ++o) {
    for (int i = 0; i < 64; ++i) w.w3[o][i] = u(t->rng) / 8.f;
    w.w3[o][64] = 0.f;
  }
  const int rc = velo_mlp_set_weights(t, &w);
  if (rc != 0) return fail(rc);
  *out = t;
  return 0;
}

int velo_mlp_trainer_destroy(VeloMlpTrainer* t)
{
  if (!t) return VELO_ERR_INVALID;
  cudaSetDevice(t->device);
  cudaStreamSynchronize(t->stream);
  trainer_free(t);
  delete t;
  return 0;
}

int velo_mlp_set_weights(VeloMlpTrainer* t, const VeloMlpWeights* w)
{
  if (!t || !w) return VELO_ERR_INVALID;
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  t->meta = *w;
  std::vector<float> slots;
  weights_to_slots(*w, slots);
  TCK(cudaMemcpyAsync(t->d_master, slots.data(), kMlpParams * 4, cudaMemcpyHostToDevice, t->stream));
  TCK(cudaMemsetAsync(t->d_m, 0, kMlpParams * 4, t->stream));
  TCK(cudaMemsetAsync(t->d_v, 0, kMlpParams * 4, t->stream));
  t->step = 0;
  int rc = upload_norm(t);  // synchronises the stream: `slots` may go
  if (rc) return rc;
  rc = publish(t, 0, nullptr, 0, 0.f);
  if (rc) return rc;
  TCK(cudaStreamSynchronize(t->stream));
  return 0;
}

int velo_mlp_get_weights(VeloMlpTrainer* t, VeloMlpWeights* w)
{
  if (!t || !w) return VELO_ERR_INVALID;
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  std::vector<float> slots(kMlpParams);
  TCK(cudaMemcpyAsync(slots.data(), t->d_master, kMlpParams * 4, cudaMemcpyDeviceToHost, t->stream));
  TCK(cudaStreamSynchronize(t->stream));
  *w = t->meta;
  slots_to_weights(slots.data(), *w);
  return 0;
}

int velo_mlp_collect(VeloMlpTrainer* t, VeloCtx* ctx, uint64_t* n_total)
{
  if (!t || !ctx) return VELO_ERR_INVALID;
  ChainPointers P;
  cudaStream_t cs;
  int dev;
  if (!velo_ctx_last_run(ctx, &P, &cs, &dev)) return VELO_ERR_STATE;
  if (dev != t->device) return VELO_ERR_INVALID;
  if (P.keep) return VELO_ERR_STATE;  // labels come from the plain search only
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  const uint32_t N = P.n_grid;  // the last run's events (its kernels were sized for them)
  if (N == 0 || t->n >= t->cap) {
    if (n_total) *n_total = t->n;
    return 0;
  }
  TCK(cudaStreamSynchronize(cs));
  if (t->hit_labels_cap < P.hit_capacity) {
    if (t->d_hit_labels) cudaFree(t->d_hit_labels);
    t->d_hit_labels = nullptr;
    TCK(talloc(t->d_hit_labels, P.hit_capacity));
    t->hit_labels_cap = P.hit_capacity;
  }
  uint32_t* d_counts = nullptr;
  uint64_t* d_offsets = nullptr;
  TCK(talloc(d_counts, 2ull * N));
  TCK(talloc(d_offsets, N));
  collect_count_kernel<<<N, 256, 0, t->stream>>>(P, t->d_hit_labels, d_counts);
  TCK(cudaGetLastError());
  std::vector<uint32_t> counts(N), take(N);
  std::vector<uint64_t> offsets(N);
  TCK(cudaMemcpyAsync(counts.data(), d_counts, 4ull * N, cudaMemcpyDeviceToHost, t->stream));
  TCK(cudaStreamSynchronize(t->stream));
  uint64_t pos = t->n;
  for (uint32_t e = 0; e < N; ++e) {
    offsets[e] = pos;
    take[e] = static_cast<uint32_t>(std::min<uint64_t>(counts[e], t->cap - pos));
    pos += take[e];
  }
  TCK(cudaMemcpyAsync(d_counts + N, take.data(), 4ull * N, cudaMemcpyHostToDevice, t->stream));
  TCK(cudaMemcpyAsync(d_offsets, offsets.data(), 8ull * N, cudaMemcpyHostToDevice, t->stream));
  collect_write_kernel<<<N, 256, 0, t->stream>>>(P, t->d_hit_labels, d_offsets, d_counts + N, t->d_feat, t->d_lab);
  TCK(cudaGetLastError());
  TCK(cudaStreamSynchronize(t->stream));
  cudaFree(d_counts);
  cudaFree(d_offsets);
  t->n = pos;
  if (n_total) *n_total = t->n;
  return 0;
}

int velo_mlp_samples(VeloMlpTrainer* t, uint64_t first, uint32_t n, float* features, uint8_t* labels)
{
  if (!t || (n && (!features || !labels)) || first + n > t->n) return VELO_ERR_INVALID;
  if (n == 0) return 0;
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  TCK(cudaMemcpyAsync(features, t->d_feat + first * 12, 48ull * n, cudaMemcpyDeviceToHost, t->stream));
  TCK(cudaMemcpyAsync(labels, t->d_lab + first, n, cudaMemcpyDeviceToHost, t->stream));
  TCK(cudaStreamSynchronize(t->stream));
  return 0;
}

int velo_mlp_normalize(VeloMlpTrainer* t)
{
  if (!t || t->n == 0) return VELO_ERR_STATE;
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  const uint64_t n = std::min<uint64_t>(t->n, 1u << 21);  // the first 2M samples suffice
  std::vector<float> f(n * 12);
  TCK(cudaMemcpyAsync(f.data(), t->d_feat, 48ull * n, cudaMemcpyDeviceToHost, t->stream));
  TCK(cudaStreamSynchronize(t->stream));
  for (int k = 0; k < 12; ++k) {
    double s = 0, s2 = 0;
    for (uint64_t i = 0; i < n; ++i) {
      const double v = f[i * 12 + k];
      s += v;
      s2 += v * v;
    }
    const double mean = s / n, var = std::max(s2 / n - mean * mean, 1e-12);
    t->meta.mean[k] = static_cast<float>(mean);
    t->meta.inv_std[k] = static_cast<float>(1.0 / std::sqrt(var));
  }
  return upload_norm(t);
}

int velo_mlp_train(VeloMlpTrainer* t, uint32_t epochs, uint32_t batch, float lr, float* last_loss)
{
  if (!t || batch == 0 || t->n == 0) return VELO_ERR_INVALID;
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  std::vector<uint32_t> perm(t->n);
  for (uint64_t i = 0; i < t->n; ++i) perm[i] = static_cast<uint32_t>(i);
  float loss = 0.f;
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), t->rng);
    TCK(cudaMemcpyAsync(t->d_perm, perm.data(), 4ull * t->n, cudaMemcpyHostToDevice, t->stream));
    TCK(cudaMemsetAsync(t->d_loss_total, 0, 4, t->stream));
    for (uint64_t first = 0; first < t->n; first += batch) {
      const uint32_t b = static_cast<uint32_t>(std::min<uint64_t>(batch, t->n - first));
      uint32_t parts = 0;
      int rc = train_step(t, t->d_feat, t->d_lab, t->d_perm, first, b, &parts);
      if (rc) return rc;
      ++t->step;
      rc = publish(t, parts, nullptr, 1, lr);
      if (rc) return rc;
    }
    float total = 0.f;
    TCK(cudaMemcpyAsync(&total, t->d_loss_total, 4, cudaMemcpyDeviceToHost, t->stream));
    TCK(cudaStreamSynchronize(t->stream));  // also orders the next epoch's perm upload
    loss = total / (2.f * static_cast<float>(t->n));
  }
  if (last_loss) *last_loss = loss;
  return check_error(t);
}

int velo_mlp_gradient(VeloMlpTrainer* t, const float* features, const uint8_t* labels, uint32_t n,
                      VeloMlpWeights* grad, float* loss)
{
  if (!t || !features || !labels || !grad || n == 0) return VELO_ERR_INVALID;
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  float* d_f = nullptr;
  uint8_t* d_l = nullptr;
  uint32_t* d_p = nullptr;
  TCK(talloc(d_f, 12ull * n));
  TCK(talloc(d_l, n));
  TCK(talloc(d_p, n));
  std::vector<uint32_t> perm(n);
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  TCK(cudaMemcpyAsync(d_f, features, 48ull * n, cudaMemcpyHostToDevice, t->stream));
  TCK(cudaMemcpyAsync(d_l, labels, n, cudaMemcpyHostToDevice, t->stream));
  TCK(cudaMemcpyAsync(d_p, perm.data(), 4ull * n, cudaMemcpyHostToDevice, t->stream));
  TCK(cudaMemsetAsync(t->d_loss_total, 0, 4, t->stream));
  uint32_t parts = 0;
  int rc = train_step(t, d_f, d_l, d_p, 0, n, &parts);
  if (!rc) rc = publish(t, parts, t->d_grad, 0, 0.f);
  std::vector<float> g(kMlpParams);
  float total = 0.f;
  if (!rc) {
    TCK(cudaMemcpyAsync(g.data(), t->d_grad, kMlpParams * 4, cudaMemcpyDeviceToHost, t->stream));
    TCK(cudaMemcpyAsync(&total, t->d_loss_total, 4, cudaMemcpyDeviceToHost, t->stream));
  }
  TCK(cudaStreamSynchronize(t->stream));
  cudaFree(d_f);
  cudaFree(d_l);
  cudaFree(d_p);
  if (rc) return rc;
  std::memset(grad, 0, sizeof(*grad));
  slots_to_weights(g.data(), *grad);
  if (loss) *loss = total / (2.f * static_cast<float>(n));
  return check_error(t);
}

int velo_mlp_infer(VeloMlpTrainer* t, const float* features, uint32_t n, float* logits)
{
  if (!t || !features || !logits || n == 0) return VELO_ERR_INVALID;
  if (cudaSetDevice(t->device) != cudaSuccess) return VELO_ERR_CUDA;
  float *d_f = nullptr, *d_z = nullptr;
  TCK(talloc(d_f, 12ull * n));
  TCK(talloc(d_z, 2ull * n));
  TCK(cudaMemcpyAsync(d_f, features, 48ull * n, cudaMemcpyHostToDevice, t->stream));
  MlpDevice m{};
  m.w = t->d_w;
  m.norm = t->d_norm;
  const uint32_t tiles = (n + kMlpTile - 1) / kMlpTile;
  mlp_infer_rows_kernel<<<std::min<uint32_t>(tiles, 4 * t->grid), kMlpTile, kMlpInferSmem, t->stream>>>(
    m, d_f, n, d_z, t->d_error);
  const cudaError_t le = cudaGetLastError();
  if (le == cudaSuccess) TCK(cudaMemcpyAsync(logits, d_z, 8ull * n, cudaMemcpyDeviceToHost, t->stream));
  TCK(cudaStreamSynchronize(t->stream));
  cudaFree(d_f);
  cudaFree(d_z);
  TCK(le);
  return check_error(t);
}

}  // extern "C"
