// Batched MLEM for sm_100a: K frames that share one system matrix run as
// one multi-right-hand-side pass per half-iteration (SpMM), so every matrix
// entry is read once per frame tile instead of once per frame.
//
// Layout: images X (n x K) and measurements Y (m x K) are frame-minor
// (X[j*K + f]); the ratios E (m x K) sit at the rows' positions in the
// transpose's order, like the single-frame e.  A pass handles a tile of KT
// consecutive frames.  Within a warp, lanes split into EPW entry slots of
// LPE lanes, each lane owning VEC frames (LPE*VEC = KT, EPW*LPE = 32): per
// step a warp reads EPW matrix entries and gathers EPW rows of KT frames,
// coalesced.  The value type is binary16 (with the per-row scale folded
// into E, as in the FP16 single-frame form) or float.  Grids are sized to
// the GPU and every warp loops over rows / columns (persistent CTAs).  The
// back pass can take the columns in a given order: voxels in compact
// (y, z) tubes along x keep the ratio rows that concurrent warps gather
// (the channels crossing those voxels) within L2.
#include <cstdint>

#include <cuda_fp16.h>

#include "internal.h"

namespace raptr {

namespace {

constexpr int kThreads = 256;

// Blocks of a pass: one warp per item up to 64 blocks per SM, so that
// blocks are short enough for the scheduler to interleave the kernels of
// other streams (batches of other geometries served at the same time).
unsigned grid_warps(int64_t items) {
  int64_t b = (items * 32 + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return unsigned(b);
}

constexpr int kColsPerWarp = 48;  // back pass: columns a warp takes before its block ends

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }

// Four frames per lane (one 16-byte gather), KT/4 lanes per entry slot.
template <int KT>
struct Split {
  static constexpr int VEC = 4;
  static constexpr int LPE = KT / VEC;
  static constexpr int EPW = 32 / LPE;
};

__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

__device__ __forceinline__ void fma4(float (&a)[4], float w, float4 x) {
  a[0] += w * x.x;
  a[1] += w * x.y;
  a[2] += w * x.z;
  a[3] += w * x.w;
}

// Forward: E[rank_i*K + f] = sc_i * Y[i*K + f] / (sc_i * sum_j v_ij X[j*K + f])
// for the frames f of the tile (0 where Y == 0); sc = rscale (FP16) or 1.
template <int KT, typename VT>
__global__ void __launch_bounds__(kThreads) batch_forward_kernel(int64_t m, int K, int f0,
                                                                 const int64_t* __restrict__ rp,
                                                                 const int32_t* __restrict__ col,
                                                                 const VT* __restrict__ val,
                                                                 const float* __restrict__ rscale,
                                                                 const float* __restrict__ Y,
                                                                 const float* __restrict__ X,
                                                                 const int32_t* __restrict__ rank,
                                                                 float* __restrict__ E) {
  using S = Split<KT>;
  const int lane = threadIdx.x & 31;
  const int es = lane / S::LPE, fg = lane % S::LPE;
  const int fbase = f0 + fg * S::VEC;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    float acc[S::VEC];
#pragma unroll
    for (int v = 0; v < S::VEC; v++) acc[v] = 0.f;
    const int64_t b = rp[r], e = rp[r + 1];
    int64_t k = b + es;
    // two entries per slot in flight
    for (; k + S::EPW < e; k += 2 * S::EPW) {
      const int c0 = __ldg(col + k), c1 = __ldg(col + k + S::EPW);
      const float w0 = to_f(val[k]), w1 = to_f(val[k + S::EPW]);
      const float4 x0 = ld4(X + int64_t(c0) * K + fbase);
      const float4 x1 = ld4(X + int64_t(c1) * K + fbase);
      fma4(acc, w0, x0);
      fma4(acc, w1, x1);
    }
    if (k < e) fma4(acc, to_f(val[k]), ld4(X + int64_t(__ldg(col + k)) * K + fbase));
#pragma unroll
    for (int o = S::LPE; o < 32; o <<= 1)
#pragma unroll
      for (int v = 0; v < S::VEC; v++) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
    if (es == 0) {
      const float sc = rscale ? __ldg(rscale + r) : 1.f;
      const int64_t dst = rank ? int64_t(__ldg(rank + r)) : r;
#pragma unroll
      for (int v = 0; v < S::VEC; v++) {
        const float yi = __ldg(Y + r * K + fbase + v);
        E[dst * K + fbase + v] = yi == 0.f ? 0.f : sc * __fdiv_rn(yi, sc * acc[v]);
      }
    }
  }
}

// Back projection and update for the frames of the tile:
// c = sum_k v_kj E[k*K + f] (FP32; the FP16 values dominate its error),
// XX = X*c/(S+(S==0)), acc[f] += sum_j XX (FP64).  Warps take columns from
// the counter *next (zero at launch).
template <int KT, typename VT>
__global__ void __launch_bounds__(kThreads) batch_back_kernel(int64_t n, int K, int f0, unsigned long long* next,
                                                              const int64_t* __restrict__ cp,
                                                              const int32_t* __restrict__ trow,
                                                              const VT* __restrict__ tval,
                                                              const float* __restrict__ E,
                                                              const float* __restrict__ X,
                                                              const float* __restrict__ sens,
                                                              const int32_t* __restrict__ col_order,
                                                              float* __restrict__ XX, double* __restrict__ acc) {
  using S = Split<KT>;
  const int lane = threadIdx.x & 31;
  const int es = lane / S::LPE, fg = lane % S::LPE;
  const int fbase = f0 + fg * S::VEC;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double fsum[S::VEC];
#pragma unroll
  for (int v = 0; v < S::VEC; v++) fsum[v] = 0.0;
  __shared__ double red[KT];  // the block's image sums per frame of the tile
  for (int i = threadIdx.x; i < KT; i += blockDim.x) red[i] = 0.0;
  __syncthreads();
  (void)nw;
  for (int taken = 0; taken < kColsPerWarp; taken++) {
    // columns are handed out one at a time (their lengths vary ~20-fold)
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(next, 1ull);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= (unsigned long long)n) break;
    const int64_t j = col_order ? int64_t(__ldg(col_order + q)) : int64_t(q);
    float s[S::VEC];
#pragma unroll
    for (int v = 0; v < S::VEC; v++) s[v] = 0.f;
    const int64_t b = cp[j], e = cp[j + 1];
    int64_t p = b + es;
    for (; p + S::EPW < e; p += 2 * S::EPW) {
      const int k0 = __ldg(trow + p), k1 = __ldg(trow + p + S::EPW);
      const float w0 = to_f(tval[p]), w1 = to_f(tval[p + S::EPW]);
      const float4 e0 = ld4(E + int64_t(k0) * K + fbase);
      const float4 e1 = ld4(E + int64_t(k1) * K + fbase);
      fma4(s, w0, e0);
      fma4(s, w1, e1);
    }
    if (p < e) fma4(s, to_f(tval[p]), ld4(E + int64_t(__ldg(trow + p)) * K + fbase));
#pragma unroll
    for (int o = S::LPE; o < 32; o <<= 1)
#pragma unroll
      for (int v = 0; v < S::VEC; v++) s[v] += __shfl_xor_sync(0xffffffffu, s[v], o);
    if (es == 0) {
      float dvs = __ldg(sens + j);
      dvs += float(dvs == 0.f);
#pragma unroll
      for (int v = 0; v < S::VEC; v++) {
        const float xx = __fdiv_rn(__fmul_rn(X[j * K + fbase + v], s[v]), dvs);
        XX[j * K + fbase + v] = xx;
        fsum[v] += double(xx);
      }
    }
  }
  if (es == 0)
#pragma unroll
    for (int v = 0; v < S::VEC; v++)
      if (fsum[v] != 0.0) atomicAdd(red + (fbase - f0) + v, fsum[v]);
  __syncthreads();
  for (int i = threadIdx.x; i < KT; i += blockDim.x)
    if (red[i] != 0.0) atomicAdd(acc + f0 + i, red[i]);
}

// X = XX * (1 / acc[f]) for all frames; then acc = 0 for the next pass.
__global__ void batch_normalise_kernel(int64_t n, int K, float* __restrict__ X, const float* __restrict__ XX,
                                       const double* __restrict__ acc) {
  const int64_t total = n * K;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int f = int(i % K);
    X[i] = XX[i] * float(1.0 / acc[f]);
  }
}

template <int KT, typename VT>
cudaError_t launch_tile(bool forward, int64_t m, int64_t n, int K, int f0, const int64_t* rp, const int32_t* col,
                        const void* val, const float* rscale, const int64_t* cp, const int32_t* trow,
                        const void* tval, const int32_t* rank, const int32_t* col_order, const float* Y,
                        const float* S, float* X, float* E, float* XX, double* acc, unsigned long long* next,
                        cudaStream_t s) {
  if (forward)
    batch_forward_kernel<KT, VT><<<grid_warps(m), kThreads, 0, s>>>(m, K, f0, rp, col, static_cast<const VT*>(val),
                                                                    rscale, Y, X, rank, E);
  else
    batch_back_kernel<KT, VT><<<unsigned((n + kColsPerWarp * (kThreads / 32) - 1) / (kColsPerWarp * (kThreads / 32))),
                                kThreads, 0, s>>>(n, K, f0, next, cp, trow, static_cast<const VT*>(tval),
                                                                 E, X, S, col_order, XX, acc);
  note_launches(1);
  return cudaGetLastError();
}

template <typename VT>
cudaError_t launch_tile_kt(int kt, bool forward, int64_t m, int64_t n, int K, int f0, const int64_t* rp,
                           const int32_t* col, const void* val, const float* rscale, const int64_t* cp,
                           const int32_t* trow, const void* tval, const int32_t* rank, const int32_t* col_order,
                           const float* Y, const float* S, float* X, float* E, float* XX, double* acc,
                           unsigned long long* next, cudaStream_t s) {
  switch (kt) {
    case 4:
      return launch_tile<4, VT>(forward, m, n, K, f0, rp, col, val, rscale, cp, trow, tval, rank, col_order, Y, S, X, E, XX, acc, next, s);
    case 8:
      return launch_tile<8, VT>(forward, m, n, K, f0, rp, col, val, rscale, cp, trow, tval, rank, col_order, Y, S, X, E, XX, acc, next, s);
    case 16:
      return launch_tile<16, VT>(forward, m, n, K, f0, rp, col, val, rscale, cp, trow, tval, rank, col_order, Y, S, X, E,
                                 XX, acc, next, s);
    case 32:
      return launch_tile<32, VT>(forward, m, n, K, f0, rp, col, val, rscale, cp, trow, tval, rank, col_order, Y, S, X, E,
                                 XX, acc, next, s);
    case 64:
      return launch_tile<64, VT>(forward, m, n, K, f0, rp, col, val, rscale, cp, trow, tval, rank, col_order, Y, S, X, E,
                                 XX, acc, next, s);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace

bool batch_tile_supported(int K, int kt) {
  return (kt == 4 || kt == 8 || kt == 16 || kt == 32 || kt == 64) && K > 0 && K % 4 == 0;
}

int batch_tile_at(int K, int kt, int f0) {
  int t = kt;
  while (t > K - f0) t >>= 1;
  return t;
}

cudaError_t launch_batch_iteration(const BatchArgs& a, int kt, double* acc, unsigned long long* next, cudaStream_t s,
                                   cudaEvent_t ev_mid) {
  // Tiles of kt frames while that many remain, then the largest power of
  // two (>= 4, since K is a multiple of 4) that fits: 40 frames at kt = 32
  // run as 32 + 8, so no frame slot is computed for nothing.
  cudaError_t e = cudaMemsetAsync(acc, 0, size_t(a.K) * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(next, 0, size_t(a.K / 4) * sizeof(unsigned long long), s);
  for (int f0 = 0; f0 < a.K && e == cudaSuccess; f0 += batch_tile_at(a.K, kt, f0)) {
    const int t = batch_tile_at(a.K, kt, f0);
    e = a.half ? launch_tile_kt<__half>(t, true, a.m, a.n, a.K, f0, a.rp, a.col, a.val, a.rscale, a.cp, a.trow,
                                        a.tval, a.rank, a.col_order, a.Y, a.S, a.X, a.E, a.XX, acc, nullptr, s)
               : launch_tile_kt<float>(t, true, a.m, a.n, a.K, f0, a.rp, a.col, a.val, nullptr, a.cp, a.trow,
                                       a.tval, a.rank, a.col_order, a.Y, a.S, a.X, a.E, a.XX, acc, nullptr, s);
  }
  if (e == cudaSuccess && ev_mid) e = cudaEventRecord(ev_mid, s);
  for (int f0 = 0, tile = 0; f0 < a.K && e == cudaSuccess; f0 += batch_tile_at(a.K, kt, f0), tile++) {
    const int t = batch_tile_at(a.K, kt, f0);
    e = a.half ? launch_tile_kt<__half>(t, false, a.m, a.n, a.K, f0, a.rp, a.col, a.val, a.rscale, a.cp, a.trow,
                                        a.tval, a.rank, a.col_order, a.Y, a.S, a.X, a.E, a.XX, acc, next + tile, s)
               : launch_tile_kt<float>(t, false, a.m, a.n, a.K, f0, a.rp, a.col, a.val, nullptr, a.cp, a.trow,
                                       a.tval, a.rank, a.col_order, a.Y, a.S, a.X, a.E, a.XX, acc, next + tile, s);
  }
  if (e == cudaSuccess) {
    const int64_t total = a.n * a.K;
    int64_t blocks = (total + kThreads - 1) / kThreads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    batch_normalise_kernel<<<unsigned(blocks), kThreads, 0, s>>>(a.n, a.K, a.X, a.XX, acc);
    note_launches(1);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace raptr
