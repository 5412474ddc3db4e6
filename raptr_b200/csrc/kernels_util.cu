// Device-wide scan and sparse-format utilities.
#include <atomic>
#include <cstdint>

#include "internal.h"

namespace raptr {

namespace {
std::atomic<long long> g_launches{0};
}

void note_launches(long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ long long warp_inclusive(long long x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Exclusive block scan of one value per thread (kScanThreads threads).
__device__ __forceinline__ long long block_excl(long long v, long long* total, long long* ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long x = warp_inclusive(v);
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    long long w = (lane < kScanThreads / 32) ? ws[lane] : 0;
    w = warp_inclusive(w);
    if (lane < kScanThreads / 32) ws[lane] = w;
  }
  __syncthreads();
  long long r = (warp > 0 ? ws[warp - 1] : 0) + x - v;
  *total = ws[kScanThreads / 32 - 1];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) scan_partials(const int64_t* __restrict__ in, int64_t n,
                                                              int64_t* __restrict__ partial) {
  __shared__ long long ws[32];
  const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++)
    if (base + k < n) s += in[base + k];
  long long tot;
  block_excl(s, &tot, ws);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) scan_spine(int64_t* __restrict__ partial, int64_t nb) {
  __shared__ long long ws[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t t0 = 0; t0 < nb; t0 += kScanThreads) {
    int64_t i = t0 + threadIdx.x;
    long long v = (i < nb) ? partial[i] : 0;
    long long tot;
    long long ex = block_excl(v, &tot, ws);
    if (i < nb) partial[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[nb] = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply(const int64_t* __restrict__ in, int64_t n,
                                                           const int64_t* __restrict__ partial,
                                                           int64_t* __restrict__ out, int64_t nb) {
  __shared__ long long ws[32];
  const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
  long long v[kScanItems];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  long long tot;
  long long ex = block_excl(s, &tot, ws) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = partial[nb];
}

__global__ void coo2csr_kernel(const int32_t* __restrict__ rows, int64_t nnz, int64_t m, int64_t* __restrict__ rp) {
  for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r <= m; r += int64_t(gridDim.x) * blockDim.x) {
    int64_t lo = 0, hi = nnz;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (rows[mid] < r) lo = mid + 1;
      else hi = mid;
    }
    rp[r] = lo;
  }
}

__global__ void csr2ecsr_kernel(int64_t* __restrict__ ecsr, const int32_t* __restrict__ yrow, int64_t nnzr,
                                const int64_t* __restrict__ csr, int64_t m) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i <= nnzr; i += int64_t(gridDim.x) * blockDim.x)
    ecsr[i] = (i < nnzr) ? csr[yrow[i]] : csr[m];
}

__global__ void iota_kernel(int32_t* __restrict__ p, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = int32_t(i);
}

__global__ void fill_kernel(float* __restrict__ p, float v, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = v;
}

__global__ void narrow_kernel(const int64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = int32_t(in[i]);
}

__global__ void widen32_kernel(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = in[i];
}

unsigned grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return unsigned(b);
}

}  // namespace

cudaError_t launch_iota(int32_t* p, int64_t n, cudaStream_t s) {
  if (n > 0) {
    iota_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, n);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_fill(float* p, float v, int64_t n, cudaStream_t s) {
  if (n > 0) {
    fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, v, n);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_narrow_i64(const int64_t* in, int64_t n, int32_t* out, cudaStream_t s) {
  if (n > 0) {
    narrow_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, n, out);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_widen_i32(const int32_t* in, int64_t n, int64_t* out, cudaStream_t s) {
  if (n > 0) {
    widen32_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, n, out);
    note_launches(1);
  }
  return cudaGetLastError();
}

// ---- back-projection order of channels ------------------------------------
//
// A channel joins crystal (z0, y0) of head 0 to (z1, y1) of head 1.  Sorting
// channels by (angle, z0+z1, y0+y1, z0-z1, y0-y1) groups lines by their
// midpoint before their slope, so the channels that cross one voxel sit in
// few short runs: a column of the transpose then reads a vector laid out in
// this order in dense runs instead of scattered words.
__device__ __forceinline__ int64_t channel_order_key(const DGeom& g, int cnl) {
  const ChannelIds c = channel_split(g, cnl);
  const int64_t sz = g.n0z + g.n1z - 1, sy = g.n0y + g.n1y - 1;
  int64_t k = c.ida;
  k = k * sz + (c.id0z + c.id1z);
  k = k * sy + (c.id0y + c.id1y);
  k = k * sz + (c.id0z - c.id1z + g.n1z - 1);
  k = k * sy + (c.id0y - c.id1y + g.n1y - 1);
  return k;
}

__global__ void order_mark_kernel(DGeom g, int64_t m, const int32_t* __restrict__ cnl, int64_t nkeys,
                                  unsigned long long* __restrict__ mark, int32_t* __restrict__ bad) {
  const int64_t nch = int64_t(g.na) * g.n0z * g.n0y * g.n1z * g.n1y;
  for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < m; r += int64_t(gridDim.x) * blockDim.x) {
    const int c = cnl[r];
    if (c < 0 || c >= nch) {
      atomicOr(bad, 1);
      continue;
    }
    const int64_t k = channel_order_key(g, c);
    if (k < 0 || k >= nkeys || atomicAdd(mark + k, 1ull) != 0ull) atomicOr(bad, 1);
  }
}

__global__ void order_rank_kernel(DGeom g, int64_t m, const int32_t* __restrict__ cnl,
                                  const int64_t* __restrict__ prefix, int32_t* __restrict__ rank,
                                  int32_t* __restrict__ order) {
  for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < m; r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t k = prefix[channel_order_key(g, cnl[r])];
    rank[r] = int32_t(k);
    order[k] = int32_t(r);
  }
}

int64_t channel_order_keys(const DGeom& g) {
  const int64_t sz = g.n0z + g.n1z - 1, sy = g.n0y + g.n1y - 1;
  return int64_t(g.na) * sz * sz * sy * sy;
}

cudaError_t launch_channel_order_mark(const DGeom& g, int64_t m, const int32_t* cnl, unsigned long long* mark,
                                      int32_t* bad, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(mark, 0, size_t(channel_order_keys(g)) * sizeof(unsigned long long), s);
  if (e != cudaSuccess || m <= 0) return e;
  order_mark_kernel<<<grid_for(m, 256), 256, 0, s>>>(g, m, cnl, channel_order_keys(g), mark, bad);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_channel_order_rank(const DGeom& g, int64_t m, const int32_t* cnl, const int64_t* prefix,
                                      int32_t* rank, int32_t* order, cudaStream_t s) {
  if (m <= 0) return cudaSuccess;
  order_rank_kernel<<<grid_for(m, 256), 256, 0, s>>>(g, m, cnl, prefix, rank, order);
  note_launches(1);
  return cudaGetLastError();
}

int64_t scan_temp_elems(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

cudaError_t launch_scan_i64(const int64_t* in, int64_t n, int64_t* out, int64_t* temp, cudaStream_t s) {
  int64_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) {
    return cudaMemsetAsync(out, 0, sizeof(int64_t), s);
  }
  scan_partials<<<unsigned(nb), kScanThreads, 0, s>>>(in, n, temp);
  note_launches(1);
  scan_spine<<<1, kScanThreads, 0, s>>>(temp, nb);
  note_launches(1);
  scan_apply<<<unsigned(nb), kScanThreads, 0, s>>>(in, n, temp, out, nb);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_coo2csr(const int32_t* rows, int64_t nnz, int64_t m, int64_t* row_ptr, int64_t*, cudaStream_t s) {
  coo2csr_kernel<<<grid_for(m + 1, 256), 256, 0, s>>>(rows, nnz, m, row_ptr);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_csr2ecsr(int64_t* ecsr, const int32_t* yrow, int64_t nnzr, const int64_t* csr, int64_t m,
                            cudaStream_t s) {
  csr2ecsr_kernel<<<grid_for(nnzr + 1, 256), 256, 0, s>>>(ecsr, yrow, nnzr, csr, m);
  note_launches(1);
  return cudaGetLastError();
}

}  // namespace raptr
