// Device memory cache for the library's stream-ordered buffers.
//
// A fit allocates a few hundred MB of short-lived buffers (membership rows, sort buffers,
// the edge slices).  Growing the CUDA stream-ordered pool for them costs 100-200 ms per
// large allocation, so freed blocks are kept here, bucketed by rounded size, and reused by
// later allocations of the same rounded size.  A block freed on stream A carries an event
// recorded on A after its last use; a stream that reuses it waits on that event first, so
// reuse across streams keeps stream order.  Blocks are returned to the pool only when an
// allocation fails (then the cache is flushed and the allocation retried) or when
// umap_release_cached_memory() is called.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include "ub_internal.hpp"

namespace ub {
namespace {

struct Block {
  void* p;
  cudaEvent_t ready;
};

struct DeviceCache {
  std::multimap<uint64_t, Block> free_blocks;  // rounded size -> block
  std::vector<cudaEvent_t> spare_events;
  uint64_t cached_bytes = 0;
};

// Never destroyed: handles may be freed during process teardown after static destructors.
std::mutex& g_mu = *new std::mutex;
std::map<int, DeviceCache>& g_cache = *new std::map<int, DeviceCache>;

uint64_t round_size(uint64_t bytes) {
  if (bytes <= (1ull << 20)) {
    uint64_t r = 512;
    while (r < bytes) r <<= 1;
    return r;
  }
  const uint64_t g = 2ull << 20;
  return (bytes + g - 1) / g * g;
}

// Returns every cached block of `dev` to the pool (caller holds g_mu).
void flush_locked(int dev) {
  auto it = g_cache.find(dev);
  if (it == g_cache.end()) return;
  for (auto& kv : it->second.free_blocks) {
    (void)cudaEventSynchronize(kv.second.ready);
    (void)cudaFreeAsync(kv.second.p, 0);
    it->second.spare_events.push_back(kv.second.ready);
  }
  it->second.free_blocks.clear();
  it->second.cached_bytes = 0;
}

}  // namespace

void* dev_alloc(uint64_t bytes, cudaStream_t s) {
  if (bytes == 0) return nullptr;
  int dev = 0;
  UB_CUDA(cudaGetDevice(&dev));
  const uint64_t rs = round_size(bytes);
  {
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceCache& c = g_cache[dev];
    auto it = c.free_blocks.lower_bound(rs);
    if (it != c.free_blocks.end() && it->first == rs) {
      Block b = it->second;
      c.free_blocks.erase(it);
      c.cached_bytes -= rs;
      UB_CUDA(cudaStreamWaitEvent(s, b.ready, 0));
      c.spare_events.push_back(b.ready);
      return b.p;
    }
  }
  const bool timed = alloc_log_enabled();
  const auto t0 = timed ? std::chrono::steady_clock::now() : std::chrono::steady_clock::time_point{};
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, rs, s);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    {
      std::lock_guard<std::mutex> lock(g_mu);
      flush_locked(dev);
    }
    e = cudaMallocAsync(&p, rs, s);
  }
  if (timed) {
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (ms > 1.0) log_slow_alloc(rs, ms);
  }
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    throw Error(OUT_OF_MEMORY, "device allocation of " + std::to_string(rs) + " bytes failed");
  }
  cuda_check(e, "cudaMallocAsync", __FILE__, __LINE__);
  return p;
}

void dev_free(void* p, uint64_t bytes, cudaStream_t s) noexcept {
  if (!p) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  const uint64_t rs = round_size(bytes);
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceCache& c = g_cache[dev];
  cudaEvent_t ev = nullptr;
  if (!c.spare_events.empty()) {
    ev = c.spare_events.back();
    c.spare_events.pop_back();
  } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    (void)cudaGetLastError();
    (void)cudaFreeAsync(p, s);
    return;
  }
  if (cudaEventRecord(ev, s) != cudaSuccess) {
    (void)cudaGetLastError();
    c.spare_events.push_back(ev);
    (void)cudaFreeAsync(p, s);
    return;
  }
  c.free_blocks.emplace(rs, Block{p, ev});
  c.cached_bytes += rs;
}

uint64_t release_cached_memory() {
  std::lock_guard<std::mutex> lock(g_mu);
  uint64_t total = 0;
  int cur = 0;
  (void)cudaGetDevice(&cur);
  for (auto& kv : g_cache) {
    total += kv.second.cached_bytes;
    (void)cudaSetDevice(kv.first);
    flush_locked(kv.first);
  }
  (void)cudaSetDevice(cur);
  (void)cudaGetLastError();
  return total;
}

}  // namespace ub
