// Batched MLEM for sm_100a: K frames that share one system matrix run as
// one multi-right-hand-side pass per half-iteration (SpMM), so every matrix
// entry is read once per frame tile instead of once per frame.
//
// Layout: images X (n x K) and measurements Y (m x K) are frame-minor
// (X[j*K + f]); the ratios E sit at the rows' positions in the transpose's
// order, like the single-frame e, in one block per tile: the tile of KT
// frames from f0 holds E[f0*m + k*KT + (f - f0)], so that the back pass
// over a tile gathers from m*KT floats (82 MB for 4 frames at 5.14M rows,
// inside L2) instead of 16 bytes out of each row of an m x K array, whose
// sectors for a 4-frame tile spread over 164 MB and missed L2 (33 ms per
// 4-frame back pass, against 3.9 ms for one frame).  A pass handles a tile
// of KT consecutive frames.  Within a warp, lanes split into EPW entry slots of
// LPE lanes, each lane owning VEC frames (LPE*VEC = KT, EPW*LPE = 32): per
// step a warp reads EPW matrix entries and gathers EPW rows of KT frames,
// coalesced.  The value type is binary16 (with the per-row scale folded
// into E, as in the FP16 single-frame form) or float.  Grids are sized to
// the GPU and every warp loops over rows / columns (persistent CTAs).  The
// back pass can take the columns in a given order: voxels in compact
// (y, z) tubes along x keep the ratio rows that concurrent warps gather
// (the channels crossing those voxels) within L2.
#include <algorithm>
#include <cstdint>
#include <vector>

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
// CTAs per SM both passes are compiled for: with 5 (48 registers) the back
// pass runs 10-35 % faster for every frame tile than compiled without a
// bound (40 registers, 6 CTAs per SM), the forward pass 1-6 % (8: slower)
constexpr int kBatchBlocks = 5;
constexpr double kBackGroupBytes = 48.0 * (1 << 20);  // ratios of a back-pass row-block group

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

// Forward: Et[rank_i*KT + f - f0] = sc_i * Y[i*K + f] / (sc_i * sum_j v_ij
// X[j*K + f]) for the frames f of the tile (0 where Y == 0), Et = E + f0*m
// the tile's block of ratios; sc = rscale (FP16) or 1.  The images are gathered from Xg with row stride xs:
// X + f0 and K, or a compact copy of the tile's frames and KT (a 4-frame
// tile then gathers from n*16 bytes instead of 16 bytes of each 256-byte
// row of a 64-frame X).
template <int KT, typename VT>
__global__ void __launch_bounds__(kThreads, kBatchBlocks) batch_forward_kernel(int64_t m, int K, int f0,
                                                                 const int64_t* __restrict__ rp,
                                                                 const int32_t* __restrict__ col,
                                                                 const VT* __restrict__ val,
                                                                 const float* __restrict__ rscale,
                                                                 const float* __restrict__ Y,
                                                                 const float* __restrict__ Xg, int xs,
                                                                 const int32_t* __restrict__ rank,
                                                                 float* __restrict__ Et) {
  using S = Split<KT>;
  const int lane = threadIdx.x & 31;
  const int es = lane / S::LPE, fg = lane % S::LPE;
  const int fbase = f0 + fg * S::VEC;
  const float* __restrict__ X = Xg + fg * S::VEC;  // the lane's four frames
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
      const float4 x0 = ld4(X + int64_t(c0) * xs);
      const float4 x1 = ld4(X + int64_t(c1) * xs);
      fma4(acc, w0, x0);
      fma4(acc, w1, x1);
    }
    if (k < e) fma4(acc, to_f(val[k]), ld4(X + int64_t(__ldg(col + k)) * xs));
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
        Et[dst * KT + fg * S::VEC + v] = yi == 0.f ? 0.f : sc * __fdiv_rn(yi, sc * acc[v]);
      }
    }
  }
}

// Back projection and update for the frames of the tile:
// c = sum_k v_kj Eb[k*KT + f - f0] (Eb = E + f0*m, the tile's block of
// ratios; FP32, the FP16 values dominate its error),
// XX = X*c/(S+(S==0)), acc[f] += sum_j XX (FP64).  Warps take columns from
// the counter *next (zero at launch).
//
// With a row-block group (seg non-null), only the column's entries whose
// rows lie in blocks [b0, b1) of the transpose's row order are summed
// (entries seg[j*segw + b0] .. seg[j*segw + b1] of column j): the ratios of
// those rows then stay in L2 while every column reads them.  The partial
// sums of all but the last group go to P (n x KT, tile-local frames); the
// last group adds them and finishes as above.  mode: 0 = the whole column
// at once, 1 = first group, 2 = a middle group, 3 = the last group.
template <int KT, typename VT>
__global__ void __launch_bounds__(kThreads, kBatchBlocks) batch_back_kernel(int64_t n, int K, int f0, unsigned long long* next,
                                                              const int64_t* __restrict__ cp,
                                                              const int32_t* __restrict__ trow,
                                                              const VT* __restrict__ tval,
                                                              const float* __restrict__ Eb,
                                                              const float* __restrict__ X,
                                                              const float* __restrict__ sens,
                                                              const int32_t* __restrict__ col_order,
                                                              float* __restrict__ XX, double* __restrict__ acc,
                                                              const int32_t* __restrict__ seg, int segw, int b0,
                                                              int b1, int mode, float* __restrict__ P) {
  using S = Split<KT>;
  const int lane = threadIdx.x & 31;
  const int es = lane / S::LPE, fg = lane % S::LPE;
  const int fbase = f0 + fg * S::VEC;
  // the lane's four frames of this tile's block of ratios
  const float* __restrict__ Et = Eb + fg * S::VEC;
  double fsum[S::VEC];
#pragma unroll
  for (int v = 0; v < S::VEC; v++) fsum[v] = 0.0;
  __shared__ double red[KT];  // the block's image sums per frame of the tile
  for (int i = threadIdx.x; i < KT; i += blockDim.x) red[i] = 0.0;
  __syncthreads();
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
    int64_t b = cp[j], e = cp[j + 1];
    if (seg) {
      const int64_t c0 = b;
      b = c0 + __ldg(seg + j * segw + b0);
      e = c0 + __ldg(seg + j * segw + b1);
    }
    int64_t p = b + es;
    for (; p + S::EPW < e; p += 2 * S::EPW) {
      const int k0 = __ldg(trow + p), k1 = __ldg(trow + p + S::EPW);
      const float w0 = to_f(tval[p]), w1 = to_f(tval[p + S::EPW]);
      const float4 e0 = ld4(Et + int64_t(k0) * KT);
      const float4 e1 = ld4(Et + int64_t(k1) * KT);
      fma4(s, w0, e0);
      fma4(s, w1, e1);
    }
    if (p < e) fma4(s, to_f(tval[p]), ld4(Et + int64_t(__ldg(trow + p)) * KT));
#pragma unroll
    for (int o = S::LPE; o < 32; o <<= 1)
#pragma unroll
      for (int v = 0; v < S::VEC; v++) s[v] += __shfl_xor_sync(0xffffffffu, s[v], o);
    if (es == 0 && mode != 0) {
      float4* pp = reinterpret_cast<float4*>(P + j * KT + (fbase - f0));
      if (mode == 2 || mode == 3) {
        const float4 q4 = *pp;
        s[0] += q4.x;
        s[1] += q4.y;
        s[2] += q4.z;
        s[3] += q4.w;
      }
      if (mode != 3) {
        *pp = make_float4(s[0], s[1], s[2], s[3]);
        continue;
      }
    }
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

// Xt[j*t + f'] = X[j*K + f0 + f'], the tile's frames of every image row
// (t a multiple of 4: one 16-byte copy per thread and step).
__global__ void batch_tile_images_kernel(int64_t n, int K, int f0, int t, const float* __restrict__ X,
                                         float* __restrict__ Xt) {
  const int q = t / 4;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n * q; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t j = i / q;
    const int v = int(i - j * q) * 4;
    *reinterpret_cast<float4*>(Xt + j * t + v) = *reinterpret_cast<const float4*>(X + j * K + f0 + v);
  }
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

// A back pass over row blocks [b0, b1) of the transpose (mode as in
// batch_back_kernel; mode 0 = every row at once, without seg).
struct BackGroup {
  int b0 = 0, b1 = 0, mode = 0;
};

template <int KT, typename VT>
cudaError_t launch_tile(const BatchArgs& a, bool forward, int f0, double* acc, unsigned long long* next,
                        const BackGroup& grp, cudaStream_t s) {
  if (forward) {
    const bool compact = a.Xt && KT < a.K;
    if (compact) {
      int64_t blocks = (a.n * (KT / 4) + kThreads - 1) / kThreads;
      if (blocks > 148 * 8) blocks = 148 * 8;
      batch_tile_images_kernel<<<unsigned(std::max<int64_t>(blocks, 1)), kThreads, 0, s>>>(a.n, a.K, f0, KT, a.X,
                                                                                         a.Xt);
      note_launches(1);
    }
    batch_forward_kernel<KT, VT><<<grid_warps(a.m), kThreads, 0, s>>>(
        a.m, a.K, f0, a.rp, a.col, static_cast<const VT*>(a.val), a.half ? a.rscale : nullptr, a.Y,
        compact ? a.Xt : a.X + f0, compact ? KT : a.K, a.rank, a.E + int64_t(f0) * a.m);
  } else {
    batch_back_kernel<KT, VT><<<unsigned((a.n + kColsPerWarp * (kThreads / 32) - 1) / (kColsPerWarp * (kThreads / 32))),
                                kThreads, 0, s>>>(a.n, a.K, f0, next, a.cp, a.trow, static_cast<const VT*>(a.tval),
                                                  a.E + int64_t(f0) * a.m,
                                                  a.X, a.S, a.col_order, a.XX, acc, grp.mode ? a.seg : nullptr,
                                                  a.seg_blocks + 1, grp.b0, grp.b1, grp.mode, a.P);
  }
  note_launches(1);
  return cudaGetLastError();
}

template <typename VT>
cudaError_t launch_tile_kt(int kt, const BatchArgs& a, bool forward, int f0, double* acc, unsigned long long* next,
                           const BackGroup& grp, cudaStream_t s) {
  switch (kt) {
    case 4: return launch_tile<4, VT>(a, forward, f0, acc, next, grp, s);
    case 8: return launch_tile<8, VT>(a, forward, f0, acc, next, grp, s);
    case 16: return launch_tile<16, VT>(a, forward, f0, acc, next, grp, s);
    case 32: return launch_tile<32, VT>(a, forward, f0, acc, next, grp, s);
    case 64: return launch_tile<64, VT>(a, forward, f0, acc, next, grp, s);
    default: return cudaErrorInvalidValue;
  }
}

// seg[j*(B+1) + b] = the offset in column j of its first entry whose row
// (position in the transpose's order) is at least b*m/B: lane b of the
// column's warp searches boundary b (entries ascend within a column).
__global__ void block_seg_kernel(int64_t n, int64_t m, int B, const int64_t* __restrict__ cp,
                                 const int32_t* __restrict__ trow, int32_t* __restrict__ seg) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; j < n; j += nw) {
    const int64_t c0 = cp[j], c1 = cp[j + 1];
    for (int b = lane; b <= B; b += 32) {
      const int64_t kb = m * b / B;
      int64_t lo = c0, hi = c1;  // first entry with trow >= kb
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (int64_t(__ldg(trow + mid)) < kb) lo = mid + 1;
        else hi = mid;
      }
      seg[j * (B + 1) + b] = int32_t(lo - c0);
    }
  }
}

}  // namespace

cudaError_t launch_block_seg(int64_t n, int64_t m, int B, const int64_t* cp, const int32_t* trow, int32_t* seg,
                             cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  block_seg_kernel<<<grid_warps(n), kThreads, 0, s>>>(n, m, B, cp, trow, seg);
  note_launches(1);
  return cudaGetLastError();
}

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
  // Back-pass row-block groups of a tile: the tile's ratios of one group
  // (rows of g blocks of the transpose's order) should fit in about half of
  // L2, so that the column gathers of the group find them there.
  auto groups = [&](int t) {
    std::vector<BackGroup> out;
    if (!a.seg || !a.P || a.seg_blocks < 2) {
      out.push_back(BackGroup{});
      return out;
    }
    const double block_bytes = double(a.m) / a.seg_blocks * t * sizeof(float);
    const int g = std::max(1, int(kBackGroupBytes / std::max(block_bytes, 1.0)));
    if (g >= a.seg_blocks) {
      out.push_back(BackGroup{});
      return out;
    }
    for (int b = 0; b < a.seg_blocks; b += g) {
      BackGroup q;
      q.b0 = b;
      q.b1 = std::min(a.seg_blocks, b + g);
      q.mode = b == 0 ? 1 : (q.b1 == a.seg_blocks ? 3 : 2);
      out.push_back(q);
    }
    return out;
  };
  const int ngroups_max = a.seg_blocks > 0 ? a.seg_blocks : 1;
  cudaError_t e = cudaMemsetAsync(acc, 0, size_t(a.K) * sizeof(double), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(next, 0, size_t(a.K / 4) * size_t(ngroups_max) * sizeof(unsigned long long), s);
  const BackGroup whole;
  for (int f0 = 0; f0 < a.K && e == cudaSuccess; f0 += batch_tile_at(a.K, kt, f0)) {
    const int t = batch_tile_at(a.K, kt, f0);
    e = a.half ? launch_tile_kt<__half>(t, a, true, f0, acc, nullptr, whole, s)
               : launch_tile_kt<float>(t, a, true, f0, acc, nullptr, whole, s);
  }
  if (e == cudaSuccess && ev_mid) e = cudaEventRecord(ev_mid, s);
  int counter = 0;
  for (int f0 = 0; f0 < a.K && e == cudaSuccess; f0 += batch_tile_at(a.K, kt, f0)) {
    const int t = batch_tile_at(a.K, kt, f0);
    for (const BackGroup& q : groups(t)) {
      if (e != cudaSuccess) break;
      e = a.half ? launch_tile_kt<__half>(t, a, false, f0, acc, next + counter, q, s)
                 : launch_tile_kt<float>(t, a, false, f0, acc, next + counter, q, s);
      counter++;
    }
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
