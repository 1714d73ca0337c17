// ORACLE — test infrastructure only. C wrapper around the reference's own x86 VELO
// clustering (x86/velo/clustering/src/Clustering.cpp:3 `clustering`,
// CudaClusteringCpuOptimized.cpp:4 `cuda_clustering_cpu_optimized`), compiled from the
// reference tree by oracle/build.py into oracle/_ref/libvelo_ref_x86.so. Used for the
// reference CPU timing and as an independent clustering cross-check.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "Clustering.h"

extern "C" {

// The reference's SuperPixel tables (x86/velo/clustering/src/ClusteringCommon.cpp:3-101).
void ref_x86_sp_patterns(uint8_t* patterns, uint8_t* sizes, float* fx, float* fy)
{
  std::vector<unsigned char> p(256, 0), s(256, 0);
  std::vector<float> x(512, 0), y(512, 0);
  cache_sp_patterns(p, s, x, y);
  std::memcpy(patterns, p.data(), 256);
  std::memcpy(sizes, s.data(), 256);
  std::memcpy(fx, x.data(), 512 * sizeof(float));
  std::memcpy(fy, y.data(), 512 * sizeof(float));
}

// algo: 0 = clustering (classic flood fill), 1 = cuda_clustering_cpu_optimized.
// Splits the events into contiguous slices, one reference call per slice, over n_threads
// host threads. counts[N] receives the clusters per event; ids (optional, capacity
// ids_capacity) the LHCb ids in the reference's output order, id_offsets[N+1] their offsets.
int ref_x86_clustering(const void* raw, const uint32_t* offsets, uint32_t n_events, const void* geometry, int algo,
                       int n_threads, uint32_t* counts, uint32_t* ids, uint64_t ids_capacity, uint64_t* id_offsets)
{
  if (!raw || !offsets || !geometry || !counts) return -1;
  const std::vector<char> geo(static_cast<const char*>(geometry), static_cast<const char*>(geometry) + 19456);
  if (n_threads <= 0) n_threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  const uint32_t per = (n_events + n_threads - 1) / n_threads;
  std::vector<std::vector<std::vector<uint32_t>>> results(n_threads);
  auto work = [&](int t) {
    const uint32_t a = std::min<uint32_t>(n_events, t * per), b = std::min<uint32_t>(n_events, a + per);
    if (a >= b) return;
    const char* base = static_cast<const char*>(raw);
    std::vector<char> events(base + offsets[a], base + offsets[b]);
    std::vector<unsigned int> offs(b - a + 1);
    for (uint32_t i = a; i <= b; ++i) offs[i - a] = offsets[i] - offsets[a];
    results[t] = algo == 0 ? clustering(geo, events, offs, false)
                           : cuda_clustering_cpu_optimized(geo, events, offs, false, logger::error);
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  uint64_t o = 0;
  uint32_t e = 0;
  for (int t = 0; t < n_threads; ++t)
    for (const auto& ev : results[t]) {
      counts[e] = static_cast<uint32_t>(ev.size());
      if (id_offsets) id_offsets[e] = o;
      if (ids && o + ev.size() <= ids_capacity) std::memcpy(ids + o, ev.data(), 4 * ev.size());
      o += ev.size();
      ++e;
    }
  if (id_offsets) id_offsets[e] = o;
  return e == n_events ? 0 : -2;
}
}
