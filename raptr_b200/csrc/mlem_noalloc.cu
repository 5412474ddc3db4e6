// MLEM iterations that allocate no device memory.
//
// raptr_mlem keeps its per-call workspace (the correction image and an FP64
// accumulator) in context scratch that it grows with cudaMalloc.  Some
// callers cannot allocate at the point where they reconstruct: a serving
// process that reserves its whole HBM budget up front in its own pool, where
// any further cudaMalloc can fail, and callers that cannot accept the device
// synchronisation cudaMalloc/cudaFree imply in the middle of a pipeline.
// raptr_mlem_noalloc serves them with the same one-pass iteration (row
// projection with the back projection scattered into the correction image,
// then the update and normalisation), its workspace in the fixed device
// array below.
//
// The array holds the correction image of at most kMaxVoxels voxels (4 MiB)
// and the accumulator; every GPU that loads the library keeps it until the
// process exits.  All calls on a device share it, and it keeps the last
// call's contents: each call clears what must start at zero, and calls whose
// work overlaps on the GPU (other streams, other host threads) race on it.
#include <cstdint>
#include <mutex>
#include <string>

#include "internal.h"

namespace raptr {

namespace {

constexpr int64_t kMaxVoxels = int64_t(1) << 20;
constexpr size_t kImageBytes = size_t(kMaxVoxels) * sizeof(float);
constexpr size_t kScratchBytes = kImageBytes + 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the array on the current device, looked up once per
// device (host code cannot use the symbol itself as a device pointer).  The
// address belongs to the device's primary context: after cudaDeviceReset
// the library's device state (this address, contexts, cached blocks) is
// gone, so the library must not be used across a reset.
cudaError_t scratch_address(int dev, void** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

thread_local std::string g_noalloc_error;

}  // namespace

raptr_status mlem_noalloc(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val,
                          const float* y, const float* s, float* x, int32_t n_iter, cudaStream_t st,
                          std::string* err) {
  if (m < 0 || n <= 0 || n_iter < 0 || !rp || !y || !s || !x) {
    *err = "raptr_mlem_noalloc: bad argument";
    return RAPTR_ERR_INVALID;
  }
  if (m > 0 && (!col || !val)) {
    // the row pointers alone cannot tell whether the rows hold entries
    *err = "raptr_mlem_noalloc: null column or value array for a matrix with rows";
    return RAPTR_ERR_INVALID;
  }
  if (n > kMaxVoxels) {
    *err = "raptr_mlem_noalloc: " + std::to_string(n) + " voxels exceed its fixed workspace of " +
           std::to_string(kMaxVoxels) + " voxels; use raptr_mlem";
    return RAPTR_ERR_INVALID;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess && (dev < 0 || dev >= kMaxDevices)) {
    *err = "device ordinal above the supported range";
    return RAPTR_ERR_UNSUPPORTED;
  }
  void* base = nullptr;
  if (e == cudaSuccess) e = scratch_address(dev, &base);
  float* c = static_cast<float*>(base);
  double* acc = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + kImageBytes);
  // The correction image must start at zero; the previous call may have
  // left anything in it.  The normalisation pass clears it again after
  // every iteration.
  if (e == cudaSuccess) e = cudaMemsetAsync(c, 0, size_t(n) * sizeof(float), st);
  for (int32_t it = 0; it < n_iter && e == cudaSuccess; it++) {
    e = launch_mlem_project(m, rp, col, val, y, x, c, nullptr, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(double), st);
    if (e == cudaSuccess) e = launch_mlem_update(n, x, c, s, acc, st);
    if (e == cudaSuccess) e = launch_mlem_normalise(n, x, c, acc, st);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *err = std::string("raptr_mlem_noalloc: ") + cudaGetErrorString(e);
    return RAPTR_ERR_CUDA;
  }
  return RAPTR_OK;
}

}  // namespace raptr
