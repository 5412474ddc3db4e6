// The precision forms of the MLEM iteration for sm_100a.
//
// FP16 system matrix: a_ij ~= scale_i * h_ij, h in IEEE binary16 with the
// row scale scale_i = max_j |a_ij| * 2^-15 (an exact power-of-two scaling of
// the row maximum), so every h of a row lies in [0, 32768] and keeps
// binary16's full 11-bit significand down to 2^-9 of the row maximum.  The
// transpose stores the same h; the forward pass folds scale_i into the
// ratio it writes (e'_i = scale_i * y_i / (A x)_i), so the back projection
// needs no scale: c_j = sum_i h_ij e'_i.  Accumulation is FP32; the back
// projection's is compensated (Neumaier's two-sum variant).  Matrix bytes
// per entry: 4 (index) + 2 (value) instead of 4 + 4.
//
// FP64 reference: the same iteration with FP32 matrix values and FP64
// vectors and accumulation, the yardstick for the FP32 and FP16 images.
#include <cstdint>

#include <cuda_fp16.h>

#include "internal.h"

namespace raptr {

namespace {

constexpr int kThreads = 256;

unsigned grid_rows(int64_t m) {
  int64_t b = (m * 32 + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return unsigned(b);
}

unsigned grid_elems(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148 * 8) b = 148 * 8;
  return unsigned(b);
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void block_add_d(double v, double* dst) {
  __shared__ double ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum_d(v);
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double w = (lane < int(blockDim.x >> 5)) ? ws[lane] : 0.0;
    w = warp_sum_d(w);
    if (lane == 0 && w != 0.0) atomicAdd(dst, w);
  }
}

__device__ __forceinline__ float h2f(uint16_t h) { return __half2float(__ushort_as_half(h)); }

// Neumaier compensated addition: (s, c) += v.
__device__ __forceinline__ void two_sum_add(float& s, float& c, float v) {
  const float t = s + v;
  if (fabsf(s) >= fabsf(v))
    c += (s - t) + v;
  else
    c += (v - t) + s;
  s = t;
}

// ---- conversion ------------------------------------------------------------

__global__ void __launch_bounds__(kThreads) half_rows_kernel(int64_t m, const int64_t* __restrict__ rp,
                                                             const float* __restrict__ val,
                                                             float* __restrict__ rscale, uint16_t* __restrict__ hval) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const int64_t b = rp[r], e = rp[r + 1];
    float mx = 0.f;
    for (int64_t k = b + lane; k < e; k += 32) mx = fmaxf(mx, fabsf(val[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const float sc = mx > 0.f ? ldexpf(mx, -15) : 1.f;
    if (lane == 0) rscale[r] = sc;
    for (int64_t k = b + lane; k < e; k += 32) hval[k] = __half_as_ushort(__float2half_rn(__fdiv_rn(val[k], sc)));
  }
}

// The transpose's values as h of the same rows (position k -> row order[k]).
__global__ void half_csc_kernel(int64_t nnz, const int32_t* __restrict__ trow, const float* __restrict__ tval,
                                const int32_t* __restrict__ order, const float* __restrict__ rscale,
                                uint16_t* __restrict__ htval) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += int64_t(gridDim.x) * blockDim.x) {
    const int k = trow[p];
    const int r = order ? order[k] : k;
    htval[p] = __half_as_ushort(__float2half_rn(__fdiv_rn(tval[p], rscale[r])));
  }
}

__global__ void pscale_kernel(int64_t m, const int32_t* __restrict__ order, const float* __restrict__ rscale,
                              float* __restrict__ pscale) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < m; k += int64_t(gridDim.x) * blockDim.x)
    pscale[k] = rscale[order ? order[k] : k];
}

// ---- FP16 iteration --------------------------------------------------------

// Row dot with binary16 values, lanes on consecutive entries (as the FP32
// forward pass).
__device__ __forceinline__ float row_dot_half(const int32_t* __restrict__ col, const uint16_t* __restrict__ hv,
                                              int64_t b, int64_t e, const float* __restrict__ x, int lane) {
  constexpr int U = 8;
  float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
  const int64_t nfull = (e - b) / (32 * U);
  int64_t k = b + lane;
  for (int64_t i = 0; i < nfull; i++, k += 32 * U) {
    int c[U];
    uint16_t v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      c[u] = __ldcs(col + k + 32 * u);
      v[u] = __ldcs(reinterpret_cast<const unsigned short*>(hv) + k + 32 * u);
    }
#pragma unroll
    for (int u = 0; u < U; u += 4) {
      acc0 += h2f(v[u]) * __ldg(x + c[u]);
      acc1 += h2f(v[u + 1]) * __ldg(x + c[u + 1]);
      acc2 += h2f(v[u + 2]) * __ldg(x + c[u + 2]);
      acc3 += h2f(v[u + 3]) * __ldg(x + c[u + 3]);
    }
  }
  if (k < e) {
    // the rest of the row as one more step with predicated loads
    int c[U];
    uint16_t v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool in = k + 32 * u < e;
      c[u] = in ? __ldcs(col + k + 32 * u) : 0;
      v[u] = in ? __ldcs(reinterpret_cast<const unsigned short*>(hv) + k + 32 * u) : uint16_t(0);
    }
#pragma unroll
    for (int u = 0; u < U; u += 4) {
      acc0 += h2f(v[u]) * __ldg(x + c[u]);
      acc1 += h2f(v[u + 1]) * __ldg(x + c[u + 1]);
      acc2 += h2f(v[u + 2]) * __ldg(x + c[u + 2]);
      acc3 += h2f(v[u + 3]) * __ldg(x + c[u + 3]);
    }
  }
  return warp_sum_f((acc0 + acc1) + (acc2 + acc3));
}

// e'[rank_i] = scale_i * y_i / (A x)_i, 0 where y_i == 0.
__global__ void __launch_bounds__(kThreads) mlem_forward_half_kernel(
    int64_t m, const int64_t* __restrict__ rp, const int32_t* __restrict__ col, const uint16_t* __restrict__ hval,
    const float* __restrict__ rscale, const float* __restrict__ y, const float* __restrict__ x,
    const int32_t* __restrict__ rank, float* __restrict__ e, double* __restrict__ ll, unsigned long long* next) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double ly = 0.0, lt = 0.0;
  // rows drawn kRowChunk at a time from `next` when given, as the FP32 pass
  int64_t r0 = next ? warp_next(next, lane) * kRowChunk : (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  for (; r0 < m; r0 = next ? warp_next(next, lane) * kRowChunk : r0 + nw)
  for (int64_t r = r0, r1 = next ? min(r0 + kRowChunk, m) : r0 + 1; r < r1; r++) {
    const float yi = __ldg(y + r);
    const int64_t dst = rank ? int64_t(__ldg(rank + r)) : r;
    if (yi == 0.f) {
      if (lane == 0) e[dst] = 0.f;
      continue;
    }
    const float sc = __ldg(rscale + r);
    const float yt = sc * row_dot_half(col, hval, rp[r], rp[r + 1], x, lane);
    if (lane == 0) {
      e[dst] = sc * __fdiv_rn(yi, yt);
      if (ll) {
        ly += double(yi) * log(double(yt));
        lt += double(yt);
      }
    }
  }
  if (ll) {
    block_add_d(ly, ll);
    __syncthreads();
    block_add_d(lt, ll + 1);
  }
}

// Column dot with binary16 values and compensated accumulation; lane q
// takes quads q, q+32, ... (four consecutive entries: 16-byte index load,
// 8-byte value load), each quad summed in FP32 and added with a two-sum.
// Four quads per lane are loaded and gathered together (3-4 % faster than
// two on the 70^3 x 5.14M matrix).
__device__ __forceinline__ float col_dot_half(const int32_t* __restrict__ trow, const uint16_t* __restrict__ hv,
                                              int64_t b, int64_t e, const float* __restrict__ ev, int lane) {
  float s = 0.f, c = 0.f;
  int64_t a = (b + 3) & ~int64_t(3);
  if (a > e) a = e;
  if (b + lane < a) two_sum_add(s, c, h2f(hv[b + lane]) * __ldg(ev + __ldg(trow + b + lane)));
  const int64_t nq = (e - a) >> 2;
  const int4* t4 = reinterpret_cast<const int4*>(trow + a);
  const uint2* h4 = reinterpret_cast<const uint2*>(hv + a);
  int64_t q = lane;
  for (; q + 96 < nq; q += 128) {
    const int4 r0 = __ldcs(t4 + q), r1 = __ldcs(t4 + q + 32), r2 = __ldcs(t4 + q + 64), r3 = __ldcs(t4 + q + 96);
    const uint2 w0 = __ldcs(h4 + q), w1 = __ldcs(h4 + q + 32), w2 = __ldcs(h4 + q + 64), w3 = __ldcs(h4 + q + 96);
    const float g0 = __ldg(ev + r0.x), g1 = __ldg(ev + r0.y), g2 = __ldg(ev + r0.z), g3 = __ldg(ev + r0.w);
    const float g4 = __ldg(ev + r1.x), g5 = __ldg(ev + r1.y), g6 = __ldg(ev + r1.z), g7 = __ldg(ev + r1.w);
    const float g8 = __ldg(ev + r2.x), g9 = __ldg(ev + r2.y), g10 = __ldg(ev + r2.z), g11 = __ldg(ev + r2.w);
    const float g12 = __ldg(ev + r3.x), g13 = __ldg(ev + r3.y), g14 = __ldg(ev + r3.z), g15 = __ldg(ev + r3.w);
    const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&w0.x));
    const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&w0.y));
    const float2 f2 = __half22float2(*reinterpret_cast<const __half2*>(&w1.x));
    const float2 f3 = __half22float2(*reinterpret_cast<const __half2*>(&w1.y));
    const float2 f4 = __half22float2(*reinterpret_cast<const __half2*>(&w2.x));
    const float2 f5 = __half22float2(*reinterpret_cast<const __half2*>(&w2.y));
    const float2 f6 = __half22float2(*reinterpret_cast<const __half2*>(&w3.x));
    const float2 f7 = __half22float2(*reinterpret_cast<const __half2*>(&w3.y));
    two_sum_add(s, c, (f0.x * g0 + f0.y * g1) + (f1.x * g2 + f1.y * g3));
    two_sum_add(s, c, (f2.x * g4 + f2.y * g5) + (f3.x * g6 + f3.y * g7));
    two_sum_add(s, c, (f4.x * g8 + f4.y * g9) + (f5.x * g10 + f5.y * g11));
    two_sum_add(s, c, (f6.x * g12 + f6.y * g13) + (f7.x * g14 + f7.y * g15));
  }
  for (; q + 32 < nq; q += 64) {
    const int4 r0 = __ldcs(t4 + q), r1 = __ldcs(t4 + q + 32);
    const uint2 w0 = __ldcs(h4 + q), w1 = __ldcs(h4 + q + 32);
    const float g0 = __ldg(ev + r0.x), g1 = __ldg(ev + r0.y), g2 = __ldg(ev + r0.z), g3 = __ldg(ev + r0.w);
    const float g4 = __ldg(ev + r1.x), g5 = __ldg(ev + r1.y), g6 = __ldg(ev + r1.z), g7 = __ldg(ev + r1.w);
    const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&w0.x));
    const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&w0.y));
    const float2 f2 = __half22float2(*reinterpret_cast<const __half2*>(&w1.x));
    const float2 f3 = __half22float2(*reinterpret_cast<const __half2*>(&w1.y));
    two_sum_add(s, c, (f0.x * g0 + f0.y * g1) + (f1.x * g2 + f1.y * g3));
    two_sum_add(s, c, (f2.x * g4 + f2.y * g5) + (f3.x * g6 + f3.y * g7));
  }
  for (; q < nq; q += 32) {
    const int4 r0 = __ldcs(t4 + q);
    const uint2 w0 = __ldcs(h4 + q);
    const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&w0.x));
    const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&w0.y));
    two_sum_add(s, c, (f0.x * __ldg(ev + r0.x) + f0.y * __ldg(ev + r0.y)) +
                          (f1.x * __ldg(ev + r0.z) + f1.y * __ldg(ev + r0.w)));
  }
  const int64_t t = a + (nq << 2) + lane;
  if (t < e) two_sum_add(s, c, h2f(hv[t]) * __ldg(ev + __ldg(trow + t)));
  // combine the lanes' (sum, compensation) pairs, compensated too
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float so = __shfl_xor_sync(0xffffffffu, s, o);
    const float co = __shfl_xor_sync(0xffffffffu, c, o);
    two_sum_add(s, c, so);
    c += co;
  }
  return s + c;
}

// Columns are drawn from the counter at `next` when it is given (see
// mlem_back_kernel), else taken by a grid stride.
template <bool UPDATE>
__global__ void __launch_bounds__(kThreads) mlem_back_half_kernel(int64_t n, const int64_t* __restrict__ cp,
                                                                  const int32_t* __restrict__ trow,
                                                                  const uint16_t* __restrict__ htval,
                                                                  const float* __restrict__ e,
                                                                  const float* __restrict__ x,
                                                                  const float* __restrict__ sens,
                                                                  float* __restrict__ out, double* __restrict__ acc,
                                                                  unsigned long long* next) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double sum = 0.0;
  int64_t j = next ? warp_next(next, lane) : (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  for (; j < n; j = next ? warp_next(next, lane) : j + nw) {
    const float c = col_dot_half(trow, htval, cp[j], cp[j + 1], e, lane);
    if (lane == 0) {
      if (UPDATE) {
        float dvs = sens[j];
        dvs += float(dvs == 0.f);
        const float xx = __fdiv_rn(__fmul_rn(x[j], c), dvs);
        out[j] = xx;
        sum += double(xx);
      } else {
        out[j] = c;
      }
    }
  }
  if (UPDATE) block_add_d(sum, acc);
}

// FP64 column sums of the FP16 matrix: s_j = sum_k h_kj * pscale_k.
__global__ void __launch_bounds__(kThreads) sens_half_kernel(int64_t n, const int64_t* __restrict__ cp,
                                                             const int32_t* __restrict__ trow,
                                                             const uint16_t* __restrict__ htval,
                                                             const float* __restrict__ pscale,
                                                             double* __restrict__ s64) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; j < n; j += nw) {
    double a = 0.0;
    for (int64_t p = cp[j] + lane; p < cp[j + 1]; p += 32) a += double(h2f(htval[p])) * double(pscale[trow[p]]);
    a = warp_sum_d(a);
    if (lane == 0) s64[j] = a;
  }
}

// ---- FP64 reference iteration --------------------------------------------

__global__ void __launch_bounds__(kThreads) mlem_forward_f64_kernel(
    int64_t m, const int64_t* __restrict__ rp, const int32_t* __restrict__ col, const float* __restrict__ val,
    const float* __restrict__ y, const double* __restrict__ x, const int32_t* __restrict__ rank,
    double* __restrict__ e, double* __restrict__ ll) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double ly = 0.0, lt = 0.0;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const double yi = __ldg(y + r);
    const int64_t dst = rank ? int64_t(__ldg(rank + r)) : r;
    if (yi == 0.0) {
      if (lane == 0) e[dst] = 0.0;
      continue;
    }
    double a = 0.0;
    for (int64_t k = rp[r] + lane; k < rp[r + 1]; k += 32) a += double(__ldcs(val + k)) * __ldg(x + __ldcs(col + k));
    a = warp_sum_d(a);
    if (lane == 0) {
      e[dst] = yi / a;
      if (ll) {
        ly += yi * log(a);
        lt += a;
      }
    }
  }
  if (ll) {
    block_add_d(ly, ll);
    __syncthreads();
    block_add_d(lt, ll + 1);
  }
}

__global__ void __launch_bounds__(kThreads) mlem_back_f64_kernel(int64_t n, const int64_t* __restrict__ cp,
                                                                 const int32_t* __restrict__ trow,
                                                                 const float* __restrict__ tval,
                                                                 const double* __restrict__ e,
                                                                 const double* __restrict__ x,
                                                                 const double* __restrict__ sens,
                                                                 double* __restrict__ out, double* __restrict__ acc) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double sum = 0.0;
  for (int64_t j = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; j < n; j += nw) {
    double c = 0.0;
    for (int64_t p = cp[j] + lane; p < cp[j + 1]; p += 32) c += double(__ldcs(tval + p)) * __ldg(e + __ldcs(trow + p));
    c = warp_sum_d(c);
    if (lane == 0) {
      double dvs = sens[j];
      dvs += double(dvs == 0.0);
      const double xx = x[j] * c / dvs;
      out[j] = xx;
      sum += xx;
    }
  }
  block_add_d(sum, acc);
}

__global__ void normalise_f64_kernel(int64_t n, double* __restrict__ x, const double* __restrict__ xx,
                                     const double* __restrict__ acc) {
  const double scale = 1.0 / *acc;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] = xx[i] * scale;
}


// ---- delta-coded FP16 form -------------------------------------------------
//
// Each row of the FP16 matrix (or column of its transpose) as a run of
// 32-bit words, word = (h << 16) | d: h the entry's binary16 value, d the
// step of its column (row position) from the previous word's index, the
// first word's from the run's anchor, which is the first index (d = 0).  A
// step above 65535 is split: words of step 65535 and value 0 come before
// the entry's own word; words with value 0 (those, and the padding) make no
// gather.  Runs start on 16-byte boundaries: offsets count
// quads of four words, and the last quad is padded with words 0.  4 bytes
// per entry instead of 6 (index 4 + value 2).
//
// A warp reads a run as quads, lane l taking quads l, l+32, ...: one
// 16-byte load per four entries.  The indices follow from the steps by a
// prefix sum: four steps within the lane, then across the lanes with a
// warp scan of the lanes' sums, then across the warp's steps through the
// carried last index.

constexpr int kMaxStep = 65535;

__device__ __forceinline__ int step_escapes(int d) { return d > kMaxStep ? (d - 1) / kMaxStep : 0; }

// Words per run (entries plus escapes), as quads; *bad on a descending index.
__global__ void __launch_bounds__(kThreads) pack_count_kernel(int64_t cnt, const int64_t* __restrict__ ptr,
                                                             const int32_t* __restrict__ idx,
                                                             int64_t* __restrict__ quads, int32_t* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < cnt; r += nw) {
    const int64_t b = ptr[r], e = ptr[r + 1];
    int64_t words = 0;
    for (int64_t k = b + lane; k < e; k += 32) {
      const int d = k == b ? 0 : idx[k] - idx[k - 1];
      if (d < 0) atomicOr(bad, 1);
      words += 1 + step_escapes(d);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) words += __shfl_xor_sync(0xffffffffu, words, o);
    if (lane == 0) quads[r] = (words + 3) >> 2;
  }
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// The runs' anchors and words (run r from word 4*qoff[r]).
__global__ void __launch_bounds__(kThreads) pack_fill_kernel(int64_t cnt, const int64_t* __restrict__ ptr,
                                                            const int32_t* __restrict__ idx,
                                                            const uint16_t* __restrict__ hv,
                                                            const int64_t* __restrict__ qoff,
                                                            int32_t* __restrict__ anchor,
                                                            uint32_t* __restrict__ words) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < cnt; r += nw) {
    const int64_t b = ptr[r], e = ptr[r + 1];
    if (lane == 0) anchor[r] = e > b ? idx[b] : 0;
    int64_t pos = qoff[r] * 4;
    for (int64_t k0 = b; k0 < e; k0 += 32) {
      const int64_t k = k0 + lane;
      const int d = k < e ? (k == b ? 0 : idx[k] - idx[k - 1]) : 0;
      const int esc = step_escapes(d);
      const int c = k < e ? 1 + esc : 0;
      const int incl = warp_incl_scan(c, lane);
      int64_t w = pos + incl - c;
      for (int j = 0; j < esc; j++) words[w++] = uint32_t(kMaxStep);
      if (k < e) words[w] = (uint32_t(hv[k]) << 16) | uint32_t(d - esc * kMaxStep);
      pos += __shfl_sync(0xffffffffu, incl, 31);
    }
    for (int64_t w = pos + lane; w < qoff[r + 1] * 4; w += 32) words[w] = 0u;
  }
}

__device__ __forceinline__ float word_h(uint32_t w) { return __half2float(__ushort_as_half(uint16_t(w >> 16))); }

// v at the word's index, read only for a word with a value: the steps above
// 65535 and the padding read nothing, so that a vector entry the run does
// not hold (a ratio y/0 of a row without entries) cannot reach the sum.
__device__ __forceinline__ float word_v(uint32_t w, const float* __restrict__ v, int i) {
  return (w >> 16) ? __ldg(v + i) : 0.f;
}

// The indices of the QPL quads a[] the lanes hold (quad u of lane l is the
// run's quad q + 32u + l), given the index before them (carry, updated to
// the last index the warp's quads reach).  Steps of quads past the run's
// end are 0.
template <int QPL>
__device__ __forceinline__ void quad_indices(const uint4 (&a)[QPL], int& carry, int lane, int (&i)[QPL][4]) {
  int sum[QPL], incl[QPL];
#pragma unroll
  for (int u = 0; u < QPL; u++) {
    sum[u] = int(a[u].x & 0xffffu) + int(a[u].y & 0xffffu) + int(a[u].z & 0xffffu) + int(a[u].w & 0xffffu);
    incl[u] = sum[u];
  }
  // the QPL scans are independent; their latencies overlap
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int u = 0; u < QPL; u++) {
      const int t = __shfl_up_sync(0xffffffffu, incl[u], o);
      if (lane >= o) incl[u] += t;
    }
  }
#pragma unroll
  for (int u = 0; u < QPL; u++) {
    const int b = carry + incl[u] - sum[u];
    i[u][0] = b + int(a[u].x & 0xffffu);
    i[u][1] = i[u][0] + int(a[u].y & 0xffffu);
    i[u][2] = i[u][1] + int(a[u].z & 0xffffu);
    i[u][3] = i[u][2] + int(a[u].w & 0xffffu);
    carry += __shfl_sync(0xffffffffu, incl[u], 31);
  }
}

constexpr int kPackedQuads = 4;  // quads per lane in flight (16 entries)

// Loads the QPL quads of lane `lane` from quad q on (zeros past q1).
template <int QPL>
__device__ __forceinline__ void load_quads(const uint4* __restrict__ w, int64_t q, int64_t q1, int lane,
                                           uint4 (&a)[QPL]) {
#pragma unroll
  for (int u = 0; u < QPL; u++) {
    const int64_t k = q + 32 * u + lane;
    a[u] = k < q1 ? __ldcs(w + k) : make_uint4(0u, 0u, 0u, 0u);
  }
}

// Dot product of the run in quads [q0, q1) with v (FP32 accumulation).
__device__ __forceinline__ float packed_row_dot(const uint4* __restrict__ w, int64_t q0, int64_t q1, int anchor,
                                                const float* __restrict__ v, int lane) {
  constexpr int Q = kPackedQuads;
  float acc[Q];
#pragma unroll
  for (int u = 0; u < Q; u++) acc[u] = 0.f;
  int carry = anchor;
  for (int64_t q = q0; q < q1; q += 32 * Q) {
    uint4 a[Q];
    load_quads<Q>(w, q, q1, lane, a);
    int i[Q][4];
    quad_indices<Q>(a, carry, lane, i);
#pragma unroll
    for (int u = 0; u < Q; u++)
      acc[u] += (word_h(a[u].x) * word_v(a[u].x, v, i[u][0]) + word_h(a[u].y) * word_v(a[u].y, v, i[u][1])) +
                (word_h(a[u].z) * word_v(a[u].z, v, i[u][2]) + word_h(a[u].w) * word_v(a[u].w, v, i[u][3]));
  }
  float t = 0.f;
#pragma unroll
  for (int u = 0; u < Q; u++) t += acc[u];
  return warp_sum_f(t);
}

// Column dot of a run with e, compensated as col_dot_half: each quad summed
// in FP32 and added with a two-sum.
__device__ __forceinline__ float packed_col_dot(const uint4* __restrict__ w, int64_t q0, int64_t q1, int anchor,
                                                const float* __restrict__ ev, int lane) {
  constexpr int Q = kPackedQuads;
  float s = 0.f, c = 0.f;
  int carry = anchor;
  for (int64_t q = q0; q < q1; q += 32 * Q) {
    uint4 a[Q];
    load_quads<Q>(w, q, q1, lane, a);
    int i[Q][4];
    quad_indices<Q>(a, carry, lane, i);
#pragma unroll
    for (int u = 0; u < Q; u++)
      two_sum_add(s, c, (word_h(a[u].x) * word_v(a[u].x, ev, i[u][0]) + word_h(a[u].y) * word_v(a[u].y, ev, i[u][1])) +
                            (word_h(a[u].z) * word_v(a[u].z, ev, i[u][2]) + word_h(a[u].w) * word_v(a[u].w, ev, i[u][3])));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float so = __shfl_xor_sync(0xffffffffu, s, o);
    const float co = __shfl_xor_sync(0xffffffffu, c, o);
    two_sum_add(s, c, so);
    c += co;
  }
  return s + c;
}

// The FP16 forward pass over delta-coded rows: e'[rank_i] = rscale_i * y_i /
// (A x)_i, rows drawn kRowChunk at a time from `next` (zero at launch).
__global__ void __launch_bounds__(kThreads) mlem_forward_packed_kernel(
    int64_t m, const int64_t* __restrict__ seg, const int32_t* __restrict__ anchor, const uint4* __restrict__ words,
    const float* __restrict__ rscale, const float* __restrict__ y, const float* __restrict__ x,
    const int32_t* __restrict__ rank, float* __restrict__ e, double* __restrict__ ll, unsigned long long* next) {
  const int lane = threadIdx.x & 31;
  double ly = 0.0, lt = 0.0;
  for (int64_t r0 = warp_next(next, lane) * kRowChunk; r0 < m; r0 = warp_next(next, lane) * kRowChunk)
    for (int64_t r = r0, r1 = min(r0 + kRowChunk, m); r < r1; r++) {
      const float yi = __ldg(y + r);
      const int64_t dst = rank ? int64_t(__ldg(rank + r)) : r;
      if (yi == 0.f) {
        if (lane == 0) e[dst] = 0.f;
        continue;
      }
      const float sc = __ldg(rscale + r);
      const float yt = sc * packed_row_dot(words, seg[r], seg[r + 1], __ldg(anchor + r), x, lane);
      if (lane == 0) {
        e[dst] = sc * __fdiv_rn(yi, yt);
        if (ll) {
          ly += double(yi) * log(double(yt));
          lt += double(yt);
        }
      }
    }
  if (ll) {
    block_add_d(ly, ll);
    __syncthreads();
    block_add_d(lt, ll + 1);
  }
}

// The FP16 back projection over delta-coded columns, columns drawn from
// `next`; with UPDATE the MLEM update in the epilogue as mlem_back_half_kernel.
template <bool UPDATE>
__global__ void __launch_bounds__(kThreads) mlem_back_packed_kernel(
    int64_t n, const int64_t* __restrict__ seg, const int32_t* __restrict__ anchor, const uint4* __restrict__ words,
    const float* __restrict__ e, const float* __restrict__ x, const float* __restrict__ sens,
    float* __restrict__ out, double* __restrict__ acc, unsigned long long* next) {
  const int lane = threadIdx.x & 31;
  double sum = 0.0;
  for (int64_t j = warp_next(next, lane); j < n; j = warp_next(next, lane)) {
    const float c = packed_col_dot(words, seg[j], seg[j + 1], __ldg(anchor + j), e, lane);
    if (lane == 0) {
      if (UPDATE) {
        float dvs = sens[j];
        dvs += float(dvs == 0.f);
        const float xx = __fdiv_rn(__fmul_rn(x[j], c), dvs);
        out[j] = xx;
        sum += double(xx);
      } else {
        out[j] = c;
      }
    }
  }
  if (UPDATE) block_add_d(sum, acc);
}

}  // namespace

cudaError_t launch_half_convert(int64_t m, int64_t nnz, const int64_t* rp, const float* val, const int32_t* trow,
                                const float* tval, const int32_t* order, float* rscale, uint16_t* hval,
                                uint16_t* htval, float* pscale, cudaStream_t s) {
  if (m <= 0) return cudaSuccess;
  half_rows_kernel<<<grid_rows(m), kThreads, 0, s>>>(m, rp, val, rscale, hval);
  note_launches(1);
  if (nnz > 0 && trow) {
    half_csc_kernel<<<148 * 16, kThreads, 0, s>>>(nnz, trow, tval, order, rscale, htval);
    note_launches(1);
  }
  pscale_kernel<<<grid_elems(m), kThreads, 0, s>>>(m, order, rscale, pscale);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_sens_half(int64_t n, const int64_t* cp, const int32_t* trow, const uint16_t* htval,
                             const float* pscale, double* s64, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  sens_half_kernel<<<grid_rows(n), kThreads, 0, s>>>(n, cp, trow, htval, pscale, s64);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mlem_forward_half(int64_t m, const int64_t* rp, const int32_t* col, const uint16_t* hval,
                                     const float* rscale, const float* y, const float* x, const int32_t* rank,
                                     float* e, double* d_ll, cudaStream_t s, unsigned long long* next) {
  if (m <= 0) return cudaSuccess;
  mlem_forward_half_kernel<<<grid_rows(m), kThreads, 0, s>>>(m, rp, col, hval, rscale, y, x, rank, e, d_ll, next);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mlem_back_half(int64_t n, const int64_t* cp, const int32_t* trow, const uint16_t* htval,
                                  const float* e, const float* x, const float* sens, float* out, double* d_acc,
                                  bool update, cudaStream_t s, unsigned long long* next) {
  if (n <= 0) return cudaSuccess;
  if (update)
    mlem_back_half_kernel<true><<<grid_rows(n), kThreads, 0, s>>>(n, cp, trow, htval, e, x, sens, out, d_acc, next);
  else
    mlem_back_half_kernel<false><<<grid_rows(n), kThreads, 0, s>>>(n, cp, trow, htval, e, x, sens, out, d_acc, next);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mlem_f64_iteration(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val,
                                      const int64_t* cp, const int32_t* trow, const float* tval, const int32_t* rank,
                                      const float* y, const double* s64, double* x, double* e, double* xx,
                                      double* acc, double* d_ll, cudaStream_t s) {
  cudaError_t err = cudaMemsetAsync(acc, 0, sizeof(double), s);
  if (err != cudaSuccess) return err;
  mlem_forward_f64_kernel<<<grid_rows(m), kThreads, 0, s>>>(m, rp, col, val, y, x, rank, e, d_ll);
  mlem_back_f64_kernel<<<grid_rows(n), kThreads, 0, s>>>(n, cp, trow, tval, e, x, s64, xx, acc);
  normalise_f64_kernel<<<grid_elems(n), kThreads, 0, s>>>(n, x, xx, acc);
  note_launches(3);
  return cudaGetLastError();
}

cudaError_t launch_pack_count(int64_t cnt, const int64_t* ptr, const int32_t* idx, int64_t* quads, int32_t* bad,
                              cudaStream_t s) {
  if (cnt <= 0) return cudaSuccess;
  pack_count_kernel<<<grid_rows(cnt), kThreads, 0, s>>>(cnt, ptr, idx, quads, bad);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_pack_fill(int64_t cnt, const int64_t* ptr, const int32_t* idx, const uint16_t* hv,
                             const int64_t* qoff, int32_t* anchor, uint32_t* words, cudaStream_t s) {
  if (cnt <= 0) return cudaSuccess;
  pack_fill_kernel<<<grid_rows(cnt), kThreads, 0, s>>>(cnt, ptr, idx, hv, qoff, anchor, words);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mlem_forward_packed(int64_t m, const int64_t* seg, const int32_t* anchor, const uint32_t* words,
                                       const float* rscale, const float* y, const float* x, const int32_t* rank,
                                       float* e, double* d_ll, unsigned long long* next, cudaStream_t s) {
  if (m <= 0) return cudaSuccess;
  mlem_forward_packed_kernel<<<grid_rows(m), kThreads, 0, s>>>(
      m, seg, anchor, reinterpret_cast<const uint4*>(words), rscale, y, x, rank, e, d_ll, next);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mlem_back_packed(int64_t n, const int64_t* seg, const int32_t* anchor, const uint32_t* words,
                                    const float* e, const float* x, const float* sens, float* out, double* d_acc,
                                    bool update, unsigned long long* next, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const uint4* w = reinterpret_cast<const uint4*>(words);
  if (update)
    mlem_back_packed_kernel<true><<<grid_rows(n), kThreads, 0, s>>>(n, seg, anchor, w, e, x, sens, out, d_acc, next);
  else
    mlem_back_packed_kernel<false><<<grid_rows(n), kThreads, 0, s>>>(n, seg, anchor, w, e, x, sens, out, d_acc, next);
  note_launches(1);
  return cudaGetLastError();
}

}  // namespace raptr
