// Learned seed / extension scorer: a 12 -> 64 -> 64 -> 2 MLP run on the 5th-generation
// tensor cores (tcgen05) with bf16 operands and fp32 accumulators in tensor memory.
//
// No counterpart in the reference: search_by_triplet (TrackSeeding.cu:7-200) tries every
// (h0, h2) pair in the phi windows of every unused h1. The scorer sees one cheap proxy
// triplet per h1 (the hits bracketing phi(h1) in its two windows) and predicts whether the
// plain search keeps h1 on a final track (output 0, "seed keep") and whether it appends h1
// to a track as an extension hit (output 1, "extension keep"); the pruned search seeds only
// from kept h1.
//
// Layout of one 128-row tile (one row per thread of a 128-thread CTA):
//   X   [128][16]  features 0..11, 1.0 in column 12 (bias), zeros
//   H   [128][80]  hidden units 0..63, 1.0 in column 64 (bias), zeros
//   W1  [64][16], W2 [64][80], W3 [16][80] (rows 2..15 zero): weights with the bias in the
//       ones column, so every layer is one K-major GEMM D = A * B^T.
// Tiles live in shared memory in the no-swizzle canonical K-major layout: 8-row x 16-byte
// core matrices, 128 B apart along K and `sbo` bytes apart along rows.
#pragma once
#include <cuda_bf16.h>

#include "velo_kernels.cuh"

namespace velo {

constexpr uint32_t kMlpFeatures = 12;
constexpr uint32_t kMlpK1 = 16;      // features + ones column, padded to one MMA K step
constexpr uint32_t kMlpHidden = 64;
constexpr uint32_t kMlpK2 = 80;      // hidden + ones column, padded to a multiple of 16
constexpr uint32_t kMlpOutPad = 16;  // two outputs padded to the smallest N of an M=128 MMA
constexpr uint32_t kMlpTile = 128;
constexpr uint32_t kMlpW1 = kMlpHidden * kMlpK1;
constexpr uint32_t kMlpW2 = kMlpHidden * kMlpK2;
constexpr uint32_t kMlpW3 = kMlpOutPad * kMlpK2;
constexpr uint32_t kMlpParams = kMlpW1 + kMlpW2 + kMlpW3;  // 7424 slots, 5122 trainable
constexpr uint32_t kMbarSpinLimit = 1u << 22;               // bounded waits on MMA completion

// ---------------------------------------------------------------------------------
// tcgen05 / mbarrier primitives
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm_100 format, version 1) of a K-major, no-swizzle tile.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: bf16 A and B (K-major), fp32 D, shape M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(uint32_t M, uint32_t N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
    "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init1(uint64_t* mbar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the phase `parity` of the barrier to complete; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait_parity(uint64_t* mbar, uint32_t parity, uint32_t limit = kMbarSpinLimit)
{
  const uint32_t a = smem_u32(mbar);
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-wide: allocates `ncols` tensor-memory columns, address written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (32x32b shape: warp w reads
// lanes 32w..32w+31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
      "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
    : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of the 16-byte chunk `kb` (K elements 8kb..8kb+7) of row `row` in a
// canonical K-major tile whose 8-row groups are `sbo` bytes apart.
__device__ __forceinline__ uint32_t canon_off(uint32_t row, uint32_t kb, uint32_t sbo)
{
  return (row >> 3) * sbo + kb * 128u + (row & 7u) * 16u;
}
// Byte offset of element (row, k).
__device__ __forceinline__ uint32_t canon_elem(uint32_t row, uint32_t k, uint32_t sbo)
{
  return canon_off(row, k >> 3, sbo) + (k & 7u) * 2u;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Copies a row-major bf16 [rows][k] matrix from global memory into the canonical layout.
__device__ __forceinline__ void load_canon(uint8_t* dst, const __nv_bfloat16* src, uint32_t rows, uint32_t k)
{
  const uint32_t kbs = k / 8, sbo = kbs * 128u;
  for (uint32_t c = threadIdx.x; c < rows * kbs; c += blockDim.x) {
    const uint32_t row = c / kbs, kb = c % kbs;
    const uint4 v = *reinterpret_cast<const uint4*>(src + row * k + kb * 8);
    *reinterpret_cast<uint4*>(dst + canon_off(row, kb, sbo)) = v;
  }
}

// Bulk copy (no tensor map) of `bytes` from global memory into shared memory, completing
// on `mbar` with the byte count; 16-byte aligned addresses, size a multiple of 16.
__device__ __forceinline__ void bulk_load_smem(void* dst, const void* src, uint32_t bytes, uint64_t* mbar)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                 smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}

// Makes the shared-memory writes of every thread visible to the tensor core and orders
// earlier tensor-memory reads before the MMAs issued next.
__device__ __forceinline__ void umma_stage_barrier()
{
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// D(tmem) (+)= A * B^T over K = k (k/16 MMAs of M = 128, N = n); A and B K-major canonical
// tiles in shared memory. Called by one thread.
__device__ __forceinline__ void umma_issue(uint32_t d_tmem, const uint8_t* a, uint32_t a_sbo, const uint8_t* b,
                                           uint32_t b_sbo, uint32_t k, uint32_t n, bool accumulate)
{
  const uint32_t idesc = umma_idesc_bf16(kMlpTile, n);
  for (uint32_t kk = 0; kk < k / 16; ++kk)
    umma_bf16(d_tmem, umma_desc(smem_u32(a) + kk * 256u, 128u, a_sbo), umma_desc(smem_u32(b) + kk * 256u, 128u, b_sbo),
              idesc, (accumulate || kk > 0) ? 1u : 0u);
}

// Waits (all threads) for the MMAs committed to `mbar`; `phase` is the barrier phase each
// thread tracks. False, uniformly over the CTA, if completion did not come in time.
__device__ __forceinline__ bool umma_wait(uint64_t* mbar, uint32_t& phase)
{
  const bool ok = mbar_wait_parity(mbar, phase);
  phase ^= 1u;
  tc_fence_after();
  return __syncthreads_and(ok);
}

// ---------------------------------------------------------------------------------
// Inference on 128-row tiles (128 threads, one row each): the trainer's row inference. The
// chain's scorer (score_candidates_kernel) runs two tiles per CTA with all three layers on
// the tensor core instead.
// ---------------------------------------------------------------------------------
// This inference keeps the hidden layer at K = 64 (the layer-2 bias is added in fp32 in the
// epilogue: the same bf16 value the training's ones column multiplies by 1) and computes the
// two-output head on the CUDA cores, so it needs neither the padded H columns nor a W3 tile.
struct __align__(128) MlpInferSmem {
  uint8_t w1[kMlpW1 * 2];
  uint8_t w2[kMlpHidden * kMlpHidden * 2];
  uint8_t x[kMlpTile * kMlpK1 * 2];
  uint8_t h[kMlpTile * kMlpHidden * 2];
  uint64_t mbar;
  uint32_t tmem;
  float norm[32];
  float b2[kMlpHidden];
  float2 w3[kMlpHidden + 1];  // head weights (output 0, output 1) per hidden unit, bias last
};

constexpr uint32_t kSbo1 = (kMlpK1 / 8) * 128;      // 256
constexpr uint32_t kSbo2 = (kMlpK2 / 8) * 128;      // 1280 (training tiles, K = 80)
constexpr uint32_t kSboH = (kMlpHidden / 8) * 128;  // 1024 (inference hidden tile, K = 64)
constexpr uint32_t kMlpInferTmemCols = 64;       // D1, D2 and D3 share columns 0..63
constexpr uint32_t kMlpInferSmem = sizeof(MlpInferSmem) + 128;  // dynamic size, 128-byte aligned

// Warp 0 allocates tensor memory, thread 0 sets up the barrier; weights to shared memory.
__device__ __forceinline__ void mlp_infer_setup(MlpInferSmem& s, const MlpDevice& mlp)
{
  if (threadIdx.x < 32) tmem_alloc(&s.tmem, kMlpInferTmemCols);
  if (threadIdx.x == 0) mbar_init1(&s.mbar);
  if (threadIdx.x < 32) s.norm[threadIdx.x] = mlp.norm[threadIdx.x];
  load_canon(s.w1, mlp.w, kMlpHidden, kMlpK1);
  // W2 without its bias column: rows of 80, first 64 columns
  for (uint32_t c = threadIdx.x; c < kMlpHidden * 8; c += blockDim.x) {
    const uint32_t row = c / 8, kb = c % 8;
    *reinterpret_cast<uint4*>(s.w2 + canon_off(row, kb, kSboH)) =
      *reinterpret_cast<const uint4*>(mlp.w + kMlpW1 + row * kMlpK2 + kb * 8);
  }
  for (uint32_t j = threadIdx.x; j <= kMlpHidden; j += blockDim.x) {
    const __nv_bfloat16* w3 = mlp.w + kMlpW1 + kMlpW2;
    s.w3[j] = make_float2(__bfloat162float(w3[j]), __bfloat162float(w3[kMlpK2 + j]));
    if (j < kMlpHidden) s.b2[j] = __bfloat162float(mlp.w[kMlpW1 + j * kMlpK2 + kMlpHidden]);
  }
  umma_stage_barrier();
}

__device__ __forceinline__ void mlp_infer_teardown(MlpInferSmem& s)
{
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) tmem_dealloc(s.tmem, kMlpInferTmemCols);
}

// Row `row` of an X tile at `tile` (shared or global memory): normalised features in
// bf16 (norm: mean[16], inv_std[16]), 1.0 bias column, zero padding.
__device__ __forceinline__ void store_feature_row(uint8_t* tile, uint32_t row, const float (&f)[kMlpFeatures],
                                                  const float* norm)
{
  float n[16];
#pragma unroll
  for (int i = 0; i < 12; ++i) n[i] = (f[i] - norm[i]) * norm[16 + i];
  n[12] = 1.f;
  n[13] = n[14] = n[15] = 0.f;
#pragma unroll
  for (uint32_t kb = 0; kb < 2; ++kb) {
    uint4 v;
    v.x = pack_bf16x2(n[8 * kb + 0], n[8 * kb + 1]);
    v.y = pack_bf16x2(n[8 * kb + 2], n[8 * kb + 3]);
    v.z = pack_bf16x2(n[8 * kb + 4], n[8 * kb + 5]);
    v.w = pack_bf16x2(n[8 * kb + 6], n[8 * kb + 7]);
    *reinterpret_cast<uint4*>(tile + canon_off(row, kb, kSbo1)) = v;
  }
}

// Writes this thread's row of X: normalised features in bf16, 1.0 bias column.
__device__ __forceinline__ void mlp_store_features(MlpInferSmem& s, const float (&f)[kMlpFeatures], bool valid)
{
  float n[16];
#pragma unroll
  for (int i = 0; i < 12; ++i) n[i] = valid ? (f[i] - s.norm[i]) * s.norm[16 + i] : 0.f;
  n[12] = 1.f;
  n[13] = n[14] = n[15] = 0.f;
  const uint32_t row = threadIdx.x;
#pragma unroll
  for (uint32_t kb = 0; kb < 2; ++kb) {
    uint4 v;
    v.x = pack_bf16x2(n[8 * kb + 0], n[8 * kb + 1]);
    v.y = pack_bf16x2(n[8 * kb + 2], n[8 * kb + 3]);
    v.z = pack_bf16x2(n[8 * kb + 4], n[8 * kb + 5]);
    v.w = pack_bf16x2(n[8 * kb + 6], n[8 * kb + 7]);
    *reinterpret_cast<uint4*>(s.x + canon_off(row, kb, kSbo1)) = v;
  }
}

// Reads this thread's 64 accumulator columns, applies ReLU and writes the bf16 row of H
// (inference layout: 64 columns, no bias column).
__device__ __forceinline__ void mlp_hidden_epilogue(uint8_t* h, uint32_t taddr_row)
{
  const uint32_t row = threadIdx.x;
  float v[64];
#pragma unroll
  for (int c = 0; c < 4; ++c) tmem_ld16(taddr_row + 16 * c, *reinterpret_cast<float(*)[16]>(v + 16 * c));
  tmem_ld_wait();
#pragma unroll
  for (uint32_t kb = 0; kb < 8; ++kb) {
    uint4 q;
    q.x = pack_bf16x2(fmaxf(v[8 * kb + 0], 0.f), fmaxf(v[8 * kb + 1], 0.f));
    q.y = pack_bf16x2(fmaxf(v[8 * kb + 2], 0.f), fmaxf(v[8 * kb + 3], 0.f));
    q.z = pack_bf16x2(fmaxf(v[8 * kb + 4], 0.f), fmaxf(v[8 * kb + 5], 0.f));
    q.w = pack_bf16x2(fmaxf(v[8 * kb + 6], 0.f), fmaxf(v[8 * kb + 7], 0.f));
    *reinterpret_cast<uint4*>(h + canon_off(row, kb, kSboH)) = q;
  }
}

// The two-output head on the CUDA cores, fused into the epilogue of layer 2: relu of this
// thread's 64 accumulators, rounded to bf16 as the tensor core would read them, dotted with
// the bf16 head weights in fp32 (2.5% of the network's multiply-adds: a third tensor-core
// round trip would cost more than the arithmetic).
__device__ __forceinline__ void mlp_head_epilogue(const MlpInferSmem& s, uint32_t taddr_row, float& z0, float& z1)
{
  float v[64];
#pragma unroll
  for (int c = 0; c < 4; ++c) tmem_ld16(taddr_row + 16 * c, *reinterpret_cast<float(*)[16]>(v + 16 * c));
  tmem_ld_wait();
  const float2 bias = s.w3[kMlpHidden];
  float a0 = bias.x, a1 = bias.y;
#pragma unroll
  for (int j = 0; j < 64; ++j) {
    const float h = __bfloat162float(__float2bfloat16_rn(fmaxf(v[j] + s.b2[j], 0.f)));
    const float2 w = s.w3[j];
    a0 = fmaf(h, w.x, a0);
    a1 = fmaf(h, w.y, a1);
  }
  z0 = a0;
  z1 = a1;
}

// One layer of the inference tile: D(cols 0..n) = A * B^T, then wait.
__device__ __forceinline__ bool mlp_layer(MlpInferSmem& s, uint32_t& phase, const uint8_t* a, uint32_t a_sbo,
                                          const uint8_t* b, uint32_t b_sbo, uint32_t k, uint32_t n)
{
  umma_stage_barrier();
  if (threadIdx.x == 0) {
    umma_issue(s.tmem, a, a_sbo, b, b_sbo, k, n, false);
    umma_commit(&s.mbar);
  }
  return umma_wait(&s.mbar, phase);
}

// Forward pass of the X tile at `x` (shared memory, canonical layout; s.x by default);
// logits of this thread's row. False on timeout.
__device__ __forceinline__ bool mlp_tile_forward(MlpInferSmem& s, uint32_t& phase, float& z0, float& z1,
                                                 const uint8_t* x = nullptr)
{
  const uint32_t taddr_row = s.tmem + ((threadIdx.x & ~31u) << 16);
  if (!mlp_layer(s, phase, x ? x : s.x, kSbo1, s.w1, kSbo1, kMlpK1, kMlpHidden)) return false;
  mlp_hidden_epilogue(s.h, taddr_row);
  if (!mlp_layer(s, phase, s.h, kSboH, s.w2, kSboH, kMlpHidden, kMlpHidden)) return false;
  mlp_head_epilogue(s, taddr_row, z0, z1);
  return true;
}

// ---------------------------------------------------------------------------------
// Features of the proxy triplet of h1
// ---------------------------------------------------------------------------------
// The hits of window [f, l) of a phi-sorted module that bracket phi1: the last with
// phi < phi1 and the first with phi >= phi1 (one of them when phi1 is outside the window).
__device__ __forceinline__ void bracket(const float4* H, int f, int l, float phi1, int& a, int& b)
{
  int lo = f, hi = l;  // first index in [f, l) with phi >= phi1
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (H[mid].w < phi1) lo = mid + 1; else hi = mid;
  }
  a = lo - 1 >= f ? lo - 1 : lo;
  b = lo < l ? lo : lo - 1;
}

// Twelve features of h1 (module m) with windows [f0, l0) in module m+2 and [f2, l2) in
// module m-2 (both non-empty): the proxy triplet is the pair of bracketing hits with the
// smallest seeding scatter (TrackSeeding.cu:137-152 formula).
__device__ __forceinline__ void seed_features(const float4* H, const uint8_t* size, uint32_t h1, uint32_t m, int f0,
                                              int l0, int f2, int l2, float (&f)[kMlpFeatures])
{
  const float4 p1 = H[h1];
  int a0, b0, a2, b2;
  bracket(H, f0, l0, p1.w, a0, b0);
  bracket(H, f2, l2, p1.w, a2, b2);
  const int c0[2] = {a0, b0}, c2[2] = {a2, b2};
  float best = 3.402823466e+38f;
  int h0 = a0, h2 = a2;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const float4 q0 = H[c0[i]], q2 = H[c2[j]];
      const float z2_tz = (q2.z - q0.z) / (p1.z - q0.z);
      const float x = q0.x + (p1.x - q0.x) * z2_tz;
      const float y = q0.y + (p1.y - q0.y) * z2_tz;
      const float dx = x - q2.x, dy = y - q2.y;
      const float sc = (dx * dx + dy * dy) / ((q2.z - p1.z) * (q2.z - p1.z));
      if (sc < best) {
        best = sc;
        h0 = c0[i];
        h2 = c2[j];
      }
    }
  const float4 q0 = H[h0], q2 = H[h2];
  const float dz = q0.z - q2.z;
  f[0] = (q0.x - q2.x) / dz;
  f[1] = (q0.y - q2.y) / dz;
  f[2] = log1pf(fminf(best, 1e6f) * 1000.f);
  f[3] = q0.w - p1.w;
  f[4] = p1.w - q2.w;
  f[5] = static_cast<float>(m);
  f[6] = static_cast<float>(l0 - f0);
  f[7] = static_cast<float>(l2 - f2);
  f[8] = sqrtf(p1.x * p1.x + p1.y * p1.y);
  f[9] = static_cast<float>(size[h1]);
  f[10] = static_cast<float>(size[h0]);
  f[11] = static_cast<float>(size[h2]);
}

}  // namespace velo
