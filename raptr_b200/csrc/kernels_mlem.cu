// CSR SpMV (forward and back projection), the MLEM element-wise operations
// and the fused MLEM projection for sm_100a.
//
// All kernels here are HBM-bandwidth bound: the matrix streams once per
// call with 16-byte vector loads (four columns + four values per lane), the
// image x (a few MB) stays in L2, and back projection accumulates with
// fire-and-forget float reductions (red.global.add.f32) into the image,
// which is also L2-resident.
#include <algorithm>
#include <cstdint>

#include "internal.h"

namespace raptr {

namespace {

constexpr int kThreads = 256;
// CTAs per SM the FP32 MLEM passes are compiled for: 5 (48 registers) runs
// them 2-4 % faster than the 4 their unbounded register use (60-62) allows;
// 6 (40 registers, with spills) is slower.
constexpr int kPassBlocks = 5;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block reduction of a double into *dst (one atomic per block).
__device__ __forceinline__ void block_add_double(double v, double* dst) {
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

// Dot product of CSR row [b, e) with x, computed by one warp; every lane
// returns the sum.  Head and tail are scalar, the aligned body uses
// 16-byte loads of four columns and four values per lane.
template <bool VEC>
__device__ __forceinline__ float row_dot(const int32_t* __restrict__ col, const float* __restrict__ val, int64_t b,
                                         int64_t e, const float* __restrict__ x, int lane) {
  float acc = 0.f;
  if (!VEC) {
    for (int64_t k = b + lane; k < e; k += 32) acc += __ldg(val + k) * __ldg(x + __ldg(col + k));
    return warp_sum(acc);
  }
  int64_t a = (b + 3) & ~int64_t(3);
  if (a > e) a = e;
  if (b + lane < a) acc += __ldg(val + b + lane) * __ldg(x + __ldg(col + b + lane));
  const int64_t nq = (e - a) >> 2;
  const int4* c4 = reinterpret_cast<const int4*>(col + a);
  const float4* v4 = reinterpret_cast<const float4*>(val + a);
  int64_t q = lane;
  // Four quads (16 entries) per lane per step: 8 independent 16-byte loads,
  // then 16 independent gathers, kept in flight together.
  float acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
  for (; q + 96 < nq; q += 128) {
    const int4 c0 = __ldg(c4 + q), c1 = __ldg(c4 + q + 32), c2 = __ldg(c4 + q + 64), c3 = __ldg(c4 + q + 96);
    const float4 w0 = __ldg(v4 + q), w1 = __ldg(v4 + q + 32), w2 = __ldg(v4 + q + 64), w3 = __ldg(v4 + q + 96);
    const float g00 = __ldg(x + c0.x), g01 = __ldg(x + c0.y), g02 = __ldg(x + c0.z), g03 = __ldg(x + c0.w);
    const float g10 = __ldg(x + c1.x), g11 = __ldg(x + c1.y), g12 = __ldg(x + c1.z), g13 = __ldg(x + c1.w);
    const float g20 = __ldg(x + c2.x), g21 = __ldg(x + c2.y), g22 = __ldg(x + c2.z), g23 = __ldg(x + c2.w);
    const float g30 = __ldg(x + c3.x), g31 = __ldg(x + c3.y), g32 = __ldg(x + c3.z), g33 = __ldg(x + c3.w);
    acc += w0.x * g00 + w0.y * g01 + w0.z * g02 + w0.w * g03;
    acc1 += w1.x * g10 + w1.y * g11 + w1.z * g12 + w1.w * g13;
    acc2 += w2.x * g20 + w2.y * g21 + w2.z * g22 + w2.w * g23;
    acc3 += w3.x * g30 + w3.y * g31 + w3.z * g32 + w3.w * g33;
  }
  for (; q < nq; q += 32) {
    const int4 c0 = __ldg(c4 + q);
    const float4 w0 = __ldg(v4 + q);
    acc += w0.x * __ldg(x + c0.x) + w0.y * __ldg(x + c0.y) + w0.z * __ldg(x + c0.z) + w0.w * __ldg(x + c0.w);
  }
  const int64_t t = a + (nq << 2) + lane;
  if (t < e) acc += __ldg(val + t) * __ldg(x + __ldg(col + t));
  return warp_sum((acc + acc1) + (acc2 + acc3));
}

// Dot product of CSR row [b, e) with x, one warp, lanes on consecutive
// entries: each step loads U entries per lane (32*U consecutive entries per
// warp, coalesced, streamed past the caches) and then gathers x for all of
// them; one gather instruction covers 32 neighbouring columns of the row,
// which sit in few cache lines because a row's voxels are sorted.
template <int U>
__device__ __forceinline__ float row_dot_seq(const int32_t* __restrict__ col, const float* __restrict__ val, int64_t b,
                                             int64_t e, const float* __restrict__ x, int lane) {
  static_assert(U % 4 == 0, "U is a multiple of 4");
  float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
  const int64_t nfull = (e - b) / (32 * U);
  int64_t k = b + lane;
  for (int64_t i = 0; i < nfull; i++, k += 32 * U) {
    int c[U];
    float v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      c[u] = __ldcs(col + k + 32 * u);
      v[u] = __ldcs(val + k + 32 * u);
    }
#pragma unroll
    for (int u = 0; u < U; u += 4) {
      acc0 += v[u] * __ldg(x + c[u]);
      acc1 += v[u + 1] * __ldg(x + c[u + 1]);
      acc2 += v[u + 2] * __ldg(x + c[u + 2]);
      acc3 += v[u + 3] * __ldg(x + c[u + 3]);
    }
  }
  if (k < e) {
    // the rest of the row (fewer than 32*U entries) as one more step with
    // predicated loads, so that its loads are in flight together
    int c[U];
    float v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool in = k + 32 * u < e;
      c[u] = in ? __ldcs(col + k + 32 * u) : 0;
      v[u] = in ? __ldcs(val + k + 32 * u) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < U; u += 4) {
      acc0 += v[u] * __ldg(x + c[u]);
      acc1 += v[u + 1] * __ldg(x + c[u + 1]);
      acc2 += v[u + 2] * __ldg(x + c[u + 2]);
      acc3 += v[u + 3] * __ldg(x + c[u + 3]);
    }
  }
  return warp_sum((acc0 + acc1) + (acc2 + acc3));
}

// y[col] += f * val over CSR row [b, e), by one warp.  Streaming loads:
// this is the last use of the row in the pass.
template <bool VEC>
__device__ __forceinline__ void row_scatter(const int32_t* __restrict__ col, const float* __restrict__ val, int64_t b,
                                            int64_t e, float f, float* __restrict__ y, int lane) {
  if (!VEC) {
    for (int64_t k = b + lane; k < e; k += 32) atomicAdd(y + __ldcs(col + k), __ldcs(val + k) * f);
    return;
  }
  int64_t a = (b + 3) & ~int64_t(3);
  if (a > e) a = e;
  if (b + lane < a) atomicAdd(y + __ldcs(col + b + lane), __ldcs(val + b + lane) * f);
  const int64_t nq = (e - a) >> 2;
  const int4* c4 = reinterpret_cast<const int4*>(col + a);
  const float4* v4 = reinterpret_cast<const float4*>(val + a);
  for (int64_t q = lane; q < nq; q += 32) {
    int4 c = __ldcs(c4 + q);
    float4 w = __ldcs(v4 + q);
    atomicAdd(y + c.x, w.x * f);
    atomicAdd(y + c.y, w.y * f);
    atomicAdd(y + c.z, w.z * f);
    atomicAdd(y + c.w, w.w * f);
  }
  const int64_t t = a + (nq << 2) + lane;
  if (t < e) atomicAdd(y + __ldcs(col + t), __ldcs(val + t) * f);
}

__global__ void __launch_bounds__(kThreads) spmv_n_kernel(int64_t m, const int64_t* __restrict__ rp,
                                                          const int32_t* __restrict__ col,
                                                          const float* __restrict__ val, float alpha,
                                                          const float* __restrict__ x, float beta,
                                                          float* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    float d = row_dot_seq<8>(col, val, rp[r], rp[r + 1], x, lane);
    if (lane == 0) y[r] = (beta == 0.f) ? alpha * d : alpha * d + beta * y[r];
  }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads) spmv_t_kernel(int64_t m, const int64_t* __restrict__ rp,
                                                          const int32_t* __restrict__ col,
                                                          const float* __restrict__ val, float alpha,
                                                          const float* __restrict__ x, float* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    float f = alpha * x[r];
    if (f != 0.f) row_scatter<VEC>(col, val, rp[r], rp[r + 1], f, y, lane);
  }
}

__global__ void scale_kernel(float* __restrict__ y, float beta, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = (beta == 0.f) ? 0.f : beta * y[i];
}

__global__ void divides_kernel(float* __restrict__ r, const float* __restrict__ a, const float* __restrict__ b,
                               int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    r[i] = a[i] / b[i];
}

// result = a * b / (c + (c == 0)) (src/mlemOperations.hpp:61-76).
__global__ void divmul_kernel(float* __restrict__ r, const float* __restrict__ a, const float* __restrict__ b,
                              const float* __restrict__ c, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    float dvs = c[i];
    dvs += float(dvs == 0.f);
    r[i] = __fdiv_rn(__fmul_rn(a[i], b[i]), dvs);
  }
}

__global__ void scales_kernel(float* __restrict__ x, float alpha, int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    x[i] = __fmul_rn(alpha, x[i]);
}

__global__ void __launch_bounds__(kThreads) sum_kernel(const float* __restrict__ x, int64_t n, double* acc) {
  double s = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += double(x[i]);
  block_add_double(s, acc);
}

__global__ void __launch_bounds__(kThreads) sum_f64_kernel(const double* __restrict__ x, int64_t n, double* acc) {
  double s = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += x[i];
  block_add_double(s, acc);
}

__global__ void __launch_bounds__(kThreads) colsum_kernel(int64_t m, const int64_t* __restrict__ rp,
                                                          const int32_t* __restrict__ col,
                                                          const float* __restrict__ val, double* __restrict__ s) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const int64_t b = rp[r], e = rp[r + 1];
    for (int64_t k = b + lane; k < e; k += 32) atomicAdd(s + __ldcs(col + k), double(__ldcs(val + k)));
  }
}

// The same column sums through the transpose: a warp per column, lanes on
// strided entries summed in FP64 and combined in a fixed order (no atomics,
// the same result on every run); the values stream once (4 bytes per entry).
__global__ void __launch_bounds__(kThreads) colsum_csc_kernel(int64_t n, const int64_t* __restrict__ cp,
                                                              const float* __restrict__ tval,
                                                              double* __restrict__ s) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; j < n; j += nw) {
    double a = 0.0;
    for (int64_t k = cp[j] + lane; k < cp[j + 1]; k += 32) a += double(__ldcs(tval + k));
    a = warp_sum_d(a);
    if (lane == 0) s[j] = a;
  }
}

// s32 = s64 / sum(s64) in one CTA of kNormThreads: the FP64 sum in a fixed
// order (each thread's stride, then a tree over the threads), so the result
// does not depend on scheduling, and no device scratch is needed.  Reads
// s64 twice from one SM: ~0.1 ms at 10^6 voxels.
constexpr int kNormThreads = 1024;
__global__ void __launch_bounds__(kNormThreads) sens_norm_self_kernel(int64_t n, const double* __restrict__ s64,
                                                                      float* __restrict__ s32) {
  __shared__ double part[kNormThreads];
  double a = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kNormThreads) a += s64[i];
  part[threadIdx.x] = a;
  __syncthreads();
  for (int w = kNormThreads / 2; w > 0; w >>= 1) {
    if (int(threadIdx.x) < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  const double t = part[0];
  for (int64_t i = threadIdx.x; i < n; i += kNormThreads) s32[i] = float(s64[i] / t);
}

// Fused MLEM projection: per measured row, yt = <a_i, x>, e = y_i / yt
// (no zero guard, src/mlemOperations.hpp:44-54), c += e * a_i.  A row with
// y_i == 0 is not part of the measurement (the reference's matrix has no row
// for it) and is skipped.
template <bool VEC>
__global__ void __launch_bounds__(kThreads) mlem_project_kernel(int64_t m, const int64_t* __restrict__ rp,
                                                                const int32_t* __restrict__ col,
                                                                const float* __restrict__ val,
                                                                const float* __restrict__ y,
                                                                const float* __restrict__ x, float* __restrict__ c,
                                                                double* __restrict__ ll) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double ly = 0.0, lt = 0.0;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    const float yi = __ldg(y + r);
    if (yi == 0.f) continue;
    const int64_t b = rp[r], e = rp[r + 1];
    const float yt = row_dot<VEC>(col, val, b, e, x, lane);
    const float f = __fdiv_rn(yi, yt);
    if (ll && lane == 0) {
      ly += double(yi) * log(double(yt));
      lt += double(yt);
    }
    row_scatter<VEC>(col, val, b, e, f, c, lane);
  }
  if (ll) {
    block_add_double(ly, ll);
    __syncthreads();
    block_add_double(lt, ll + 1);
  }
}

// The same projection for rows still in the build's staging slots (row i:
// entries st_col/st_val[i*cap, i*cap + row_nnz[i]), columns ascending), so
// that rows rebuilt in every iteration are projected without being placed
// into a CSR first.  Rows with row_nnz[i] < 0 (not built) are skipped.
// With s64 non-null every built row's entries are also added to the FP64
// column sums s64 (the sensitivity), measured or not.
__global__ void __launch_bounds__(kThreads) stage_project_kernel(int64_t nrows, const int32_t* __restrict__ st_col,
                                                                 const float* __restrict__ st_val, int cap,
                                                                 const int32_t* __restrict__ row_nnz,
                                                                 const float* __restrict__ y,
                                                                 const float* __restrict__ x, float* __restrict__ c,
                                                                 double* __restrict__ s64) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < nrows; r += nw) {
    const int cnt = __ldg(row_nnz + r);
    if (cnt <= 0) continue;
    const int32_t* rc = st_col + size_t(r) * cap;
    const float* rv = st_val + size_t(r) * cap;
    if (s64)
      for (int k = lane; k < cnt; k += 32) atomicAdd(s64 + __ldg(rc + k), double(__ldg(rv + k)));
    const float yi = __ldg(y + r);
    if (yi == 0.f) continue;
    float acc = 0.f;
    for (int k = lane; k < cnt; k += 32) acc += __ldg(rv + k) * __ldg(x + __ldg(rc + k));
    const float f = __fdiv_rn(yi, warp_sum(acc));
    for (int k = lane; k < cnt; k += 32) atomicAdd(c + __ldg(rc + k), __ldg(rv + k) * f);
  }
}

__global__ void __launch_bounds__(kThreads) mlem_update_kernel(int64_t n, float* __restrict__ x,
                                                               const float* __restrict__ c,
                                                               const float* __restrict__ s, double* __restrict__ acc) {
  double sum = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    float dvs = s[i];
    dvs += float(dvs == 0.f);
    float xx = __fdiv_rn(__fmul_rn(x[i], c[i]), dvs);
    x[i] = xx;
    sum += double(xx);
  }
  block_add_double(sum, acc);
}

// x = scale * xx with scale = float(1/float(sum)) as src/tests/reco.cu:300-302
// (norm = sum(x); scales(x, val_t(1./norm))); clears c when given.
__global__ void mlem_normalise_kernel(int64_t n, float* __restrict__ x, const float* __restrict__ xx,
                                      float* __restrict__ c, const double* __restrict__ acc) {
  const float norm = float(*acc);
  const float scale = float(1.0 / double(norm));
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] = __fmul_rn(scale, xx[i]);
    if (c) c[i] = 0.f;
  }
}

// ---- transpose (CSC) and the two-pass MLEM iteration ------------------------

// Deterministic transpose.  The rows, taken in a given order (k -> row
// order[k], or k itself), are cut into B contiguous blocks, one warp each.
// Pass 1 counts the entries of every (column, block) pair, pass 2 turns the
// counts of each column into exclusive offsets over the blocks, and pass 3
// has every warp walk its rows in order and append each entry at its
// (column, block) cursor, with a warp barrier between rows.  Within a column
// the entries therefore come out in the order of k, whatever the
// scheduling.  cnt is column-major (cnt[j*B + b]).  Entries with a column
// outside [0, n) or an order entry outside [0, m) are skipped and flagged.
__device__ __forceinline__ int64_t block_begin(int64_t m, int B, int b) { return m * b / B; }

__global__ void __launch_bounds__(kThreads) tblock_count_kernel(int64_t m, int64_t n, int B,
                                                                const int64_t* __restrict__ rp,
                                                                const int32_t* __restrict__ col,
                                                                const int32_t* __restrict__ order,
                                                                int32_t* __restrict__ cnt, int32_t* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int nw = int((int64_t(gridDim.x) * blockDim.x) >> 5);
  for (int b = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); b < B; b += nw) {
    const int64_t k1 = block_begin(m, B, b + 1);
    for (int64_t k = block_begin(m, B, b); k < k1; k++) {
      const int64_t r = order ? int64_t(__ldg(order + k)) : k;
      if (r < 0 || r >= m) {
        if (lane == 0) atomicOr(bad, 1);
        continue;
      }
      const int64_t e = rp[r + 1];
      for (int64_t q = rp[r] + lane; q < e; q += 32) {
        const int j = __ldcs(col + q);
        if (j < 0 || j >= n) {
          atomicOr(bad, 1);
          continue;
        }
        atomicAdd(cnt + int64_t(j) * B + b, 1);
      }
    }
  }
}

// One warp per column: cnt[j*B .. j*B+B) becomes its exclusive prefix sum,
// colcount[j] the column total.
__global__ void __launch_bounds__(kThreads) tblock_scan_kernel(int64_t n, int B, int32_t* __restrict__ cnt,
                                                               int64_t* __restrict__ colcount) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; j < n; j += nw) {
    int32_t* c = cnt + j * B;
    int run = 0;
    for (int b0 = 0; b0 < B; b0 += 32) {
      const int v = (b0 + lane < B) ? c[b0 + lane] : 0;
      int x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (b0 + lane < B) c[b0 + lane] = run + x - v;
      run += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) colcount[j] = run;
  }
}

// Pass 3: entry (row order[k], j) goes to cp[j] + cursor(j, block of k);
// its row id is k when POSITIONS, else the row itself.
template <bool POSITIONS>
__global__ void __launch_bounds__(kThreads) tblock_fill_kernel(int64_t m, int64_t n, int B,
                                                               const int64_t* __restrict__ rp,
                                                               const int32_t* __restrict__ col,
                                                               const float* __restrict__ val,
                                                               const int32_t* __restrict__ order,
                                                               const int64_t* __restrict__ cp,
                                                               int32_t* __restrict__ cur, int32_t* __restrict__ trow,
                                                               float* __restrict__ tval) {
  const int lane = threadIdx.x & 31;
  const int nw = int((int64_t(gridDim.x) * blockDim.x) >> 5);
  for (int b = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); b < B; b += nw) {
    const int64_t k1 = block_begin(m, B, b + 1);
    for (int64_t k = block_begin(m, B, b); k < k1; k++) {
      const int64_t r = order ? int64_t(__ldg(order + k)) : k;
      if (r >= 0 && r < m) {
        const int32_t id = int32_t(POSITIONS ? k : r);
        const int64_t e = rp[r + 1];
        // four entries per lane in flight; a row's columns are distinct, so
        // their cursors are too
        for (int64_t q = rp[r] + lane; q < e; q += 128) {
          int j[4];
          float v[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int64_t qq = q + 32 * u;
            j[u] = -1;
            if (qq < e) {
              j[u] = __ldcs(col + qq);
              v[u] = __ldcs(val + qq);
              if (j[u] >= n) j[u] = -1;
            }
          }
          int64_t pos[4];
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (j[u] >= 0) pos[u] = cp[j[u]] + atomicAdd(cur + int64_t(j[u]) * B + b, 1);
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (j[u] >= 0) {
              trow[pos[u]] = id;
              tval[pos[u]] = v[u];
            }
        }
      }
      __syncwarp();
    }
  }
}

// Forward projection with the ratio: e_i = y_i / <a_i, x> for measured rows
// (y_i != 0), e_i = 0 otherwise.  With rank, e_i is stored at rank[i] (the
// layout a transpose in that order reads).
__global__ void __launch_bounds__(kThreads, kPassBlocks) mlem_forward_kernel(int64_t m, const int64_t* __restrict__ rp,
                                                                const int32_t* __restrict__ col,
                                                                const float* __restrict__ val,
                                                                const float* __restrict__ y,
                                                                const float* __restrict__ x,
                                                                const int32_t* __restrict__ rank,
                                                                float* __restrict__ e, double* __restrict__ ll,
                                                                unsigned long long* next) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double ly = 0.0, lt = 0.0;
  // rows [r0, r1): kRowChunk rows drawn from the counter at `next`, or one
  // row by a grid stride
  int64_t r0 = next ? warp_next(next, lane) * kRowChunk : (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  for (; r0 < m; r0 = next ? warp_next(next, lane) * kRowChunk : r0 + nw)
  for (int64_t r = r0, r1 = next ? min(r0 + kRowChunk, m) : r0 + 1; r < r1; r++) {
    const float yi = __ldg(y + r);
    const int64_t dst = rank ? int64_t(__ldg(rank + r)) : r;
    if (yi == 0.f) {
      if (lane == 0) e[dst] = 0.f;
      continue;
    }
    const float yt = row_dot_seq<8>(col, val, rp[r], rp[r + 1], x, lane);
    if (lane == 0) {
      e[dst] = __fdiv_rn(yi, yt);
      if (ll) {
        ly += double(yi) * log(double(yt));
        lt += double(yt);
      }
    }
  }
  if (ll) {
    block_add_double(ly, ll);
    __syncthreads();
    block_add_double(lt, ll + 1);
  }
}

// Back projection by columns: c_j = <column j of A, e>.  With UPDATE the
// MLEM update follows in the epilogue: xx_j = x_j*c_j/(s_j + (s_j==0)) and
// acc += sum xx (FP64); without it c_j is stored.  With a column counter
// (`next`, zero at launch) each warp draws its next column from it, so that
// warps whose columns were short take more of them: columns run from a few
// entries at the edge of the field of view to ~10^4 at its centre, and a
// grid stride leaves the kernel waiting on the warps that drew the longest
// (0.85 instead of 0.72 of HBM on the 70^3 x 5.14M matrix).  Without it the
// columns go by a grid stride.
template <bool VEC, bool UPDATE>
__global__ void __launch_bounds__(kThreads, kPassBlocks) mlem_back_kernel(int64_t n, const int64_t* __restrict__ cp,
                                                             const int32_t* __restrict__ trow,
                                                             const float* __restrict__ tval,
                                                             const float* __restrict__ e,
                                                             const float* __restrict__ x,
                                                             const float* __restrict__ sens, float* __restrict__ out,
                                                             double* __restrict__ acc, unsigned long long* next) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double sum = 0.0;
  int64_t j = next ? warp_next(next, lane) : (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  for (; j < n; j = next ? warp_next(next, lane) : j + nw) {
    const float c = row_dot<VEC>(trow, tval, cp[j], cp[j + 1], e, lane);
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
  if (UPDATE) block_add_double(sum, acc);
}

// The 16-byte vector path needs 16-byte aligned column and value arrays.
bool aligned16(const void* a, const void* b) {
  return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15u) == 0;
}

unsigned ew_grid(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148 * 8) b = 148 * 8;
  return unsigned(b);
}

unsigned row_grid(int64_t m) {
  int64_t b = (m * 32 + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return unsigned(b);
}

}  // namespace

cudaError_t launch_spmv(int op, int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val,
                        float alpha, const float* x, float beta, float* y, cudaStream_t s) {
  if (op == RAPTR_OP_N) {
    if (m > 0) {
      spmv_n_kernel<<<row_grid(m), kThreads, 0, s>>>(m, rp, col, val, alpha, x, beta, y);
      note_launches(1);
    }
  } else {
    if (beta != 1.f && n > 0) {
      scale_kernel<<<ew_grid(n), kThreads, 0, s>>>(y, beta, n);
      note_launches(1);
    }
    if (m > 0) {
      if (aligned16(col, val)) {
        spmv_t_kernel<true><<<row_grid(m), kThreads, 0, s>>>(m, rp, col, val, alpha, x, y);
        note_launches(1);
      }
      else {
        spmv_t_kernel<false><<<row_grid(m), kThreads, 0, s>>>(m, rp, col, val, alpha, x, y);
        note_launches(1);
      }
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_divides(float* r, const float* a, const float* b, int64_t n, cudaStream_t s) {
  if (n > 0) {
    divides_kernel<<<ew_grid(n), kThreads, 0, s>>>(r, a, b, n);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_divides_multiplies(float* r, const float* a, const float* b, const float* c, int64_t n,
                                      cudaStream_t s) {
  if (n > 0) {
    divmul_kernel<<<ew_grid(n), kThreads, 0, s>>>(r, a, b, c, n);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_scales(float* x, float alpha, int64_t n, cudaStream_t s) {
  if (n > 0) {
    scales_kernel<<<ew_grid(n), kThreads, 0, s>>>(x, alpha, n);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_sum(const float* x, int64_t n, double* d_acc, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_acc, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    sum_kernel<<<ew_grid(n), kThreads, 0, s>>>(x, n, d_acc);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_sum_f64(const double* x, int64_t n, double* d_acc, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_acc, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    sum_f64_kernel<<<ew_grid(n), kThreads, 0, s>>>(x, n, d_acc);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_column_sums(int64_t m, const int64_t* rp, const int32_t* col, const float* val, double* s64,
                               cudaStream_t s) {
  if (m > 0) {
    colsum_kernel<<<row_grid(m), kThreads, 0, s>>>(m, rp, col, val, s64);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_column_sums_csc(int64_t n, const int64_t* cp, const float* tval, double* s64, cudaStream_t s) {
  if (n > 0) {
    colsum_csc_kernel<<<row_grid(n), kThreads, 0, s>>>(n, cp, tval, s64);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_sens_normalise_self(int64_t n, const double* s64, float* s32, cudaStream_t s) {
  if (n > 0) {
    sens_norm_self_kernel<<<1, kNormThreads, 0, s>>>(n, s64, s32);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_mlem_project(int64_t m, const int64_t* rp, const int32_t* col, const float* val, const float* y,
                                const float* x, float* c, double* d_ll, cudaStream_t s) {
  if (m > 0) {
    if (aligned16(col, val)) {
      mlem_project_kernel<true><<<row_grid(m), kThreads, 0, s>>>(m, rp, col, val, y, x, c, d_ll);
      note_launches(1);
    }
    else {
      mlem_project_kernel<false><<<row_grid(m), kThreads, 0, s>>>(m, rp, col, val, y, x, c, d_ll);
      note_launches(1);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_stage_project(int64_t nrows, const int32_t* st_col, const float* st_val, int cap,
                                 const int32_t* row_nnz, const float* y, const float* x, float* c, double* s64,
                                 cudaStream_t s) {
  if (nrows > 0) {
    stage_project_kernel<<<row_grid(nrows), kThreads, 0, s>>>(nrows, st_col, st_val, cap, row_nnz, y, x, c, s64);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_mlem_update(int64_t n, float* x, const float* c, const float* sens, double* d_acc, cudaStream_t s) {
  if (n > 0) {
    mlem_update_kernel<<<ew_grid(n), kThreads, 0, s>>>(n, x, c, sens, d_acc);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_mlem_normalise(int64_t n, float* x, float* c, double* d_acc, cudaStream_t s) {
  if (n > 0) {
    mlem_normalise_kernel<<<ew_grid(n), kThreads, 0, s>>>(n, x, x, c, d_acc);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_mlem_normalise_from(int64_t n, float* x, const float* xx, double* d_acc, cudaStream_t s) {
  if (n > 0) {
    mlem_normalise_kernel<<<ew_grid(n), kThreads, 0, s>>>(n, x, xx, nullptr, d_acc);
    note_launches(1);
  }
  return cudaGetLastError();
}

int transpose_blocks(int64_t m, int64_t n) {
  // enough warps to fill the GPU, with the count table (B x n int32) kept
  // under 4 GiB
  int64_t B = (int64_t(4) << 30) / (4 * std::max<int64_t>(n, 1));
  B = std::min<int64_t>(B, 4096);
  B = std::max<int64_t>(B & ~int64_t(31), 32);
  B = std::min<int64_t>(B, std::max<int64_t>(m, 1));
  return int(B);
}

cudaError_t launch_transpose_blocked(int64_t m, int64_t n, int B, const int64_t* rp, const int32_t* col,
                                     const float* val, const int32_t* order, bool positions, int32_t* cnt,
                                     int64_t* colcount, int64_t* scan_tmp, int32_t* bad, int64_t* cp, int32_t* trow,
                                     float* tval, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(cnt, 0, size_t(B) * size_t(n) * sizeof(int32_t), s);
  if (e != cudaSuccess) return e;
  const unsigned gb = unsigned((int64_t(B) * 32 + kThreads - 1) / kThreads);
  if (m > 0) {
    tblock_count_kernel<<<gb, kThreads, 0, s>>>(m, n, B, rp, col, order, cnt, bad);
    note_launches(1);
  }
  tblock_scan_kernel<<<row_grid(n), kThreads, 0, s>>>(n, B, cnt, colcount);
  note_launches(1);
  e = launch_scan_i64(colcount, n, cp, scan_tmp, s);
  if (e != cudaSuccess) return e;
  if (m > 0) {
    if (positions)
      tblock_fill_kernel<true><<<gb, kThreads, 0, s>>>(m, n, B, rp, col, val, order, cp, cnt, trow, tval);
    else
      tblock_fill_kernel<false><<<gb, kThreads, 0, s>>>(m, n, B, rp, col, val, order, cp, cnt, trow, tval);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_mlem_forward(int64_t m, const int64_t* rp, const int32_t* col, const float* val, const float* y,
                                const float* x, const int32_t* rank, float* e, double* d_ll, cudaStream_t s,
                                unsigned long long* next) {
  if (m > 0) {
    mlem_forward_kernel<<<row_grid(m), kThreads, 0, s>>>(m, rp, col, val, y, x, rank, e, d_ll, next);
    note_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_mlem_back(int64_t n, const int64_t* cp, const int32_t* trow, const float* tval, const float* e,
                             const float* x, const float* sens, float* out, double* d_acc, bool update,
                             cudaStream_t s, unsigned long long* next) {
  if (n <= 0) return cudaSuccess;
  const bool v = aligned16(trow, tval);
  if (update) {
    if (v) {
      mlem_back_kernel<true, true><<<row_grid(n), kThreads, 0, s>>>(n, cp, trow, tval, e, x, sens, out, d_acc, next);
      note_launches(1);
    }
    else {
      mlem_back_kernel<false, true><<<row_grid(n), kThreads, 0, s>>>(n, cp, trow, tval, e, x, sens, out, d_acc, next);
      note_launches(1);
    }
  } else {
    if (v) {
      mlem_back_kernel<true, false><<<row_grid(n), kThreads, 0, s>>>(n, cp, trow, tval, e, x, sens, out, d_acc, next);
      note_launches(1);
    }
    else {
      mlem_back_kernel<false, false><<<row_grid(n), kThreads, 0, s>>>(n, cp, trow, tval, e, x, sens, out, d_acc, next);
      note_launches(1);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_zero_f64(double* p, int64_t n, cudaStream_t s) {
  return cudaMemsetAsync(p, 0, size_t(n) * sizeof(double), s);
}

}  // namespace raptr
