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
// whose work overlaps on a device race with each other (keep them on one stream). The first
// call on a device looks up the array's device address (cudaGetSymbolAddress) and caches it
// for the CUDA context current at the time (another context, or a reset device, gets the
// look-up again); that first call should come before any stream capture.
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

// Warp per event, events pulled from the counter at the head of the scratch. The search of
// each event is the chain's warp search (search_event_warp, velo_search.cuh), with its seeding
// windows computed in place instead of read from fill_candidates' output.
__global__ void __launch_bounds__(128) search_static_kernel(StaticSearchArgs A)
{
  __shared__ SearchWarpShared s_warp[4];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  SearchWarpShared& sw = s_warp[warp];
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
    uint32_t n_tracks = 0;
    const bool runnable = !(status & (kStatusBadRawEvent | kStatusHitOverflow)) && nhits <= kEventHitCap && nhits > 0;
    if (nhits > kEventHitCap) flags |= kStatusHitOverflow;
    if (runnable) {
      search_event_setup(sw, A.module_start + e * kModules, A.module_num + e * kModules, base, nhits);
      const float4* H = A.xyzp + base;
      uint8_t* ev_scratch = A.scratch + kStaticHeaderBytes + static_cast<size_t>(e) * kEventScratchBytes;
      const EventScratch sc{A.track_n + static_cast<size_t>(e) * kMaxTracks,
                            A.track_hits + static_cast<size_t>(e) * kMaxTracks * kMaxTrackSize,
                            reinterpret_cast<uint16_t*>(ev_scratch),
                            reinterpret_cast<uint32_t*>(ev_scratch + kTrackletBytes),
                            reinterpret_cast<uint16_t*>(ev_scratch + kTrackletBytes + kTtfBytes)};
      n_tracks = search_event_warp(sw, H, ComputedWindows{H, sw.mstart, sw.mnum}, nullptr, sc, flags);
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

// The scratch address of one device as seen from one CUDA context (module globals exist per
// context: a caller that makes another context current on the same device, or resets the
// device, gets a fresh set-up).
struct SymbolEntry {
  void* context = nullptr;
  void* address = nullptr;
};
std::mutex g_symbol_mutex;
SymbolEntry g_symbol[64];

// The calling thread's current CUDA context (driver handle), or null when none is current;
// looked up through the runtime so that the library needs no link-time driver dependency.
void* current_context()
{
  using CtxGetCurrent = int (*)(void**);
  static const CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Device address of velo_static_scratch on device `dev` (current). Set-up, once per device
// and context: cudaGetSymbolAddress with that device current.
int static_scratch_address(int dev, void** out)
{
  std::lock_guard<std::mutex> lock(g_symbol_mutex);
  SymbolEntry& entry = g_symbol[dev];
  const void* ctx = current_context();
  if (entry.address && ctx && ctx == entry.context) {
    *out = entry.address;
    return 0;
  }
  void* address = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&address, velo_static_scratch);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "velo_search_static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
    entry = SymbolEntry{};
    return VELO_ERR_CUDA;
  }
  entry.address = address;
  entry.context = current_context();  // the set-up made the device's context current if none was
  *out = address;
  return 0;
}

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
  const int rc = static_scratch_address(dev, &scratch);
  if (rc != 0) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the work-queue counter starts at zero; the rings are written before they are read
  if (cudaMemsetAsync(scratch, 0, kStaticHeaderBytes, s) != cudaSuccess) return VELO_ERR_CUDA;
  StaticSearchArgs A{reinterpret_cast<const float4*>(hit_xyzp), module_hit_start, module_hit_num, status_in,
                     n_events, track_n, track_hits, event_tracks, status_out, static_cast<uint8_t*>(scratch)};
  const uint32_t blocks = (n_events + 3) / 4;
  search_static_kernel<<<blocks, 128, 0, s>>>(A);
  return cudaGetLastError() == cudaSuccess ? 0 : VELO_ERR_CUDA;
}
