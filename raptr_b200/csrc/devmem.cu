// Device memory for the library's large buffers (system matrices, their
// transposes, transpose staging, build scratch), kept for reuse when freed.
//
// A reconstruction job allocates and frees tens of GB per build and
// transpose, and a few dozen smaller blocks (row pointers, channel lists,
// row orders, counters); cudaFree costs 30-600 ms of host time for the
// large blocks and, at times, as much for a block of a few MB or bytes
// (one transpose's release of its counters took 765 ms), during which the
// device idles; a job that follows reallocates the same sizes.  Blocks are
// therefore not returned to the driver when the library frees them but
// parked per device, and a later request of a similar size (up to 25 %
// smaller) takes the smallest fitting parked block.  Parked bytes per device are capped at two thirds
// of the device's memory, which holds every block of a full reconstruction
// job (matrix, transpose and the transpose's staging, ~107 GB at 70^3 x
// 5.14M channels), so that the next job of the same size allocates nothing
// from the driver; when an allocation fails, the device's parked blocks
// are released and the allocation is retried once.  raptr_trim_memory()
// releases them on request (before a caller allocates much memory by other
// means, say).
//
// The environment variable RAPTR_DEVICE_MEMORY_LIMIT (bytes, read once)
// caps what the library holds on a device (blocks in use and parked): an
// allocation beyond it fails like one the device cannot satisfy, so that a
// process sharing the device can keep the rest, and the callers that fall
// back on a smaller working set (raptr_reco_host rebuilding rows in every
// iteration) do so within the cap.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <unordered_map>

#include "internal.h"

namespace raptr {

namespace {

struct Block {
  size_t bytes;
  int device;
};

std::mutex g_mu;
std::unordered_map<void*, Block> g_live;                 // blocks handed out
std::map<int, size_t> g_in_use;                          // device -> bytes handed out
std::map<int, std::multimap<size_t, void*>> g_parked;    // device -> size -> block
std::map<int, size_t> g_parked_bytes;
std::map<int, size_t> g_total;                           // device -> memory size

// Releases the parked blocks of `device` (all devices for -1).  Holds g_mu.
void release_locked(int device) {
  int cur = -1;
  cudaGetDevice(&cur);
  for (auto it = g_parked.begin(); it != g_parked.end(); ++it) {
    if (device >= 0 && it->first != device) continue;
    cudaSetDevice(it->first);
    for (auto& kv : it->second) cudaFree(kv.second);
    it->second.clear();
    g_parked_bytes[it->first] = 0;
  }
  if (cur >= 0) cudaSetDevice(cur);
}

size_t memory_limit() {
  static const size_t lim = [] {
    const char* v = std::getenv("RAPTR_DEVICE_MEMORY_LIMIT");
    return v ? size_t(std::strtoull(v, nullptr, 10)) : size_t(0);
  }();
  return lim;
}

// Whether `bytes` more may be handed out on `device` under the limit
// (parked blocks released first when they are what stands in the way).
// Holds g_mu.
bool within_limit_locked(int device, size_t bytes) {
  const size_t lim = memory_limit();
  if (lim == 0) return true;
  if (g_in_use[device] + g_parked_bytes[device] + bytes <= lim) return true;
  release_locked(device);
  return g_in_use[device] + bytes <= lim;
}

}  // namespace

size_t dev_available(int device) {
  size_t free_b = 0, total_b = 0;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    (void)cudaGetLastError();
    free_b = 0;
  }
  if (cur >= 0 && cur != device) cudaSetDevice(cur);
  std::lock_guard<std::mutex> lock(g_mu);
  size_t avail = free_b + g_parked_bytes[device];  // parked blocks can be given back
  const size_t lim = memory_limit();
  if (lim > 0) avail = std::min(avail, lim > g_in_use[device] ? lim - g_in_use[device] : size_t(0));
  return avail;
}

cudaError_t dev_alloc(void** p, size_t bytes) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_mu);
  auto& parked = g_parked[dev];
  auto it = parked.lower_bound(bytes);
  if (it != parked.end() && it->first <= bytes + bytes / 4) {
    *p = it->second;
    g_live[*p] = Block{it->first, dev};
    g_parked_bytes[dev] -= it->first;
    g_in_use[dev] += it->first;
    parked.erase(it);
    return cudaSuccess;
  }
  if (!within_limit_locked(dev, bytes)) return cudaErrorMemoryAllocation;
  const double t0 = trace_on() ? trace_ms() : 0.0;
  e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation && !parked.empty()) {
    (void)cudaGetLastError();
    release_locked(dev);
    e = cudaMalloc(p, bytes);
  }
  if (trace_on())
    trace("dev_alloc: %zu bytes from the driver in %.2f ms (%zu bytes parked on device %d)", bytes,
          trace_ms() - t0, g_parked_bytes[dev], dev);
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  g_live[*p] = Block{bytes, dev};
  g_in_use[dev] += bytes;
  return cudaSuccess;
}

void dev_free(void* p) {
  if (!p) return;
  Block b{};
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_live.find(p);
    if (it != g_live.end()) {
      b = it->second;
      g_live.erase(it);
      g_in_use[b.device] -= b.bytes;
    }
  }
  if (b.bytes == 0) {
    // not from dev_alloc
    cudaFree(p);
    return;
  }
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != b.device) cudaSetDevice(b.device);
  // Like cudaFree, wait for the device's work (which may still use the
  // block) before the block can be handed out again.  The wait runs without
  // the lock, so that other threads' allocations do not wait for it too.
  const double t0 = trace_on() ? trace_ms() : 0.0;
  bool ok = cudaDeviceSynchronize() == cudaSuccess;
  const double t1 = trace_on() ? trace_ms() : 0.0;
  size_t total = 0, freeb = 0;
  bool park = false;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (ok && !g_total.count(b.device)) {
      ok = cudaMemGetInfo(&freeb, &total) == cudaSuccess;
      if (ok) g_total[b.device] = total;
    }
    if (ok) {
      total = g_total[b.device];
      park = g_parked_bytes[b.device] + b.bytes <= total / 3 * 2;
      if (park) {
        g_parked[b.device].emplace(b.bytes, p);
        g_parked_bytes[b.device] += b.bytes;
      }
    }
  }
  if (!park) {
    // a failed wait (a stream being captured, a device error) leaves the
    // block's use unknown: hand it back to the driver, never to the cache
    (void)cudaGetLastError();
    const cudaError_t e = cudaFree(p);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      trace("dev_free: cudaFree of a %zu-byte block failed (%s); the block is leaked", b.bytes,
            cudaGetErrorString(e));
    }
  }
  if (trace_on())
    trace("dev_free: %zu bytes %s (device wait %.2f ms, then %.2f ms)", b.bytes,
          park ? "parked" : "returned to the driver", t1 - t0, trace_ms() - t1);
  if (cur >= 0 && cur != b.device) cudaSetDevice(cur);
}

void dev_release(int device) {
  std::lock_guard<std::mutex> lock(g_mu);
  release_locked(device);
}

}  // namespace raptr
