// CSR -> CSC for sm_100a as a least-significant-digit radix sort of the
// entries by column, rows ascending within each column.
//
// Entries enter in the order of their positions k (rows taken in the given
// order); each pass is a stable partition by the next 10 bits of the column,
// so after the passes the entries are sorted by (column, k).  A pass is
// histogram -> scan -> scatter over tiles of ~128K entries, one CTA each:
// the CTA ranks its entries in chunks of 8192 (32 warps x 8 items x 32
// lanes) with __match_any_sync and per-warp digit counters in shared
// memory.  In the first pass a chunk is staged in shared memory in sorted
// order and written out by consecutive threads, so that the stores of a
// warp coalesce (the lanes' entries are neighbours in a row and carry
// different digits); the second pass stores directly.  The first pass reads
// the CSR rows directly (a tile is a range of positions k); the second reads
// the staging written by the first and writes the CSC.  Column pointers come
// from column counts taken in the last pass's histogram.
//
// Scales as (passes x 3) streaming sweeps of the entries; used for matrices
// whose columns fit two passes (n <= 2^20).  The first digit is 9 bits
// where the second (10 bits) still covers the column, so that a chunk of the
// first scatter holds full 32-byte runs per digit.
#include <algorithm>
#include <cstdint>

#include "internal.h"

namespace raptr {

namespace {

constexpr int kRadixBits = 10;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kWarps = 32;
constexpr int kItems = 8;
constexpr int kChunk = kWarps * kItems * 32;  // entries ranked together
constexpr int kMaxTileRows = 1024;
constexpr int64_t kTileEntries = 131072;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

// Entries of a first-pass tile: positions k in [k0, k1); shared arrays hold
// the tile-local start of each row and its global start.
struct RowTile {
  int64_t k0;
  int nrows;
  int nent;
  const int* start;       // nrows + 1 tile-local starts
  const int64_t* gstart;  // nrows global starts (into col / val)

  // tile-local entry e >= start[i] -> the row holding it, scanning forward
  // from row i (a thread's successive entries are close: 32 apart in a
  // scatter chunk, mostly in the same row; one block apart in a histogram,
  // a row or two on)
  __device__ __forceinline__ void advance(int e, int* i, int64_t* q) const {
    int r = *i;
    while (start[r + 1] <= e) r++;
    *i = r;
    *q = gstart[r] + (e - start[r]);
  }

  // tile-local entry e -> (row index i, global entry index)
  __device__ __forceinline__ void locate(int e, int* i, int64_t* q) const {
    int lo = 0, hi = nrows;  // last i with start[i] <= e
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (start[mid] <= e)
        lo = mid;
      else
        hi = mid;
    }
    *i = lo;
    *q = gstart[lo] + (e - start[lo]);
  }
};

// Loads the row layout of first-pass tile t into shared memory.
__device__ void load_row_tile(int64_t m, int rows_per_tile, int t, const int64_t* __restrict__ rp,
                              const int32_t* __restrict__ order, int* sh_start, int64_t* sh_gstart, int* sh_len,
                              RowTile* tile, int32_t* __restrict__ bad) {
  const int64_t k0 = int64_t(t) * rows_per_tile;
  const int nrows = int(m - k0 < rows_per_tile ? m - k0 : rows_per_tile);
  for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
    int64_t r = order ? int64_t(__ldg(order + k0 + i)) : k0 + i;
    int len = 0;
    int64_t g = 0;
    if (r >= 0 && r < m) {
      g = rp[r];
      len = int(rp[r + 1] - g);
    } else {
      atomicOr(bad, 1);
    }
    sh_len[i] = len;
    sh_gstart[i] = g;
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // exclusive scan of the row lengths by warp 0
    const int lane = threadIdx.x;
    int run = 0;
    for (int b = 0; b < nrows; b += 32) {
      const int v = b + lane < nrows ? sh_len[b + lane] : 0;
      int x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (b + lane < nrows) sh_start[b + lane] = run + x - v;
      run += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) sh_start[nrows] = run;
  }
  __syncthreads();
  tile->k0 = k0;
  tile->nrows = nrows;
  tile->nent = sh_start[nrows];
  tile->start = sh_start;
  tile->gstart = sh_gstart;
}

// Histogram of one pass: hist[d * ntiles + t].  The first pass (ROWS)
// checks the columns.  Column counts (colcnt, when given) are taken in the
// last pass.  With two passes its input is sorted by the low digit, so a
// tile holds (nearly) one low digit, that of its first entry: its entries
// of that low digit are counted per high digit in shared memory and added
// to colcnt once per column at the end; any other entry adds to colcnt
// directly.  Each thread loads kHistItems entries before counting them, so
// that their loads are in flight together.
constexpr int kHistItems = 4;

template <bool ROWS>
__global__ void __launch_bounds__(kWarps * 32) rs_hist(int64_t m, int64_t n, int rows_per_tile, int64_t nent_flat,
                                                       const int64_t* __restrict__ rp, const int32_t* __restrict__ key,
                                                       const int32_t* __restrict__ order, int shift, int mask, int ntiles,
                                                       int64_t* __restrict__ hist, int32_t* __restrict__ colcnt,
                                                       int32_t* __restrict__ bad) {
  __shared__ int sh_hist[kRadix];
  __shared__ int sh_col[kRadix];  // last of two passes: counts of the first entry's low digit
  __shared__ int sh_start[kMaxTileRows + 1];
  __shared__ int64_t sh_gstart[kMaxTileRows];
  __shared__ int sh_len[kMaxTileRows];
  const int t = blockIdx.x;
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
    sh_hist[d] = 0;
    sh_col[d] = 0;
  }
  RowTile tile{};
  int64_t e0 = 0;
  int nent;
  if (ROWS) {
    load_row_tile(m, rows_per_tile, t, rp, order, sh_start, sh_gstart, sh_len, &tile, bad);
    nent = tile.nent;
  } else {
    e0 = int64_t(t) * kTileEntries;
    nent = int(nent_flat - e0 < kTileEntries ? nent_flat - e0 : kTileEntries);
    __syncthreads();
  }
  const int lmask = (1 << shift) - 1;
  const int low0 = (!ROWS && colcnt && nent > 0) ? (__ldg(key + e0) & lmask) : 0;
  int row = -1;  // ROWS: row of this thread's previous entry
  for (int b = threadIdx.x; b < nent; b += kHistItems * blockDim.x) {
    int c[kHistItems];
#pragma unroll
    for (int u = 0; u < kHistItems; u++) {
      const int e = b + u * int(blockDim.x);
      c[u] = 0;
      if (e < nent) {
        int64_t q;
        if (ROWS) {
          if (row < 0)
            tile.locate(e, &row, &q);
          else
            tile.advance(e, &row, &q);
        } else {
          q = e0 + e;
        }
        c[u] = __ldg(key + q);
      }
    }
#pragma unroll
    for (int u = 0; u < kHistItems; u++) {
      if (b + u * int(blockDim.x) >= nent) break;
      const int cu = c[u];
      const int d = (cu >> shift) & mask;
      if (ROWS) {
        if (cu < 0 || cu >= n) {
          atomicOr(bad, 1);
          continue;
        }
        if (colcnt) atomicAdd(colcnt + cu, 1);
      } else if (colcnt) {
        if ((cu & lmask) == low0)
          atomicAdd(sh_col + d, 1);
        else
          atomicAdd(colcnt + cu, 1);
      }
      atomicAdd(sh_hist + d, 1);
    }
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
    hist[int64_t(d) * ntiles + t] = sh_hist[d];
    if (!ROWS && colcnt && sh_col[d] > 0) atomicAdd(colcnt + ((d << shift) | low0), sh_col[d]);
  }
}

// Scatter of one pass.  Positions: off[d * ntiles + t] + rank of the entry
// among the tile's entries of digit d (in input order).  Writes the key
// (when out_key is non-null), the position k and the value.
template <bool ROWS>
__global__ void __launch_bounds__(kWarps * 32, 1) rs_scatter(int64_t m, int64_t n, int rows_per_tile, int64_t nent_flat,
                                                          const int64_t* __restrict__ rp,
                                                          const int32_t* __restrict__ key,
                                                          const int32_t* __restrict__ kin,
                                                          const float* __restrict__ vin,
                                                          const int32_t* __restrict__ order, int shift, int mask, int ntiles,
                                                          const int64_t* __restrict__ off,
                                                          int32_t* __restrict__ out_key, int32_t* __restrict__ out_k,
                                                          float* __restrict__ out_v, int32_t* __restrict__ bad) {
  // dynamic shared memory (scatter_smem_bytes(ROWS)): digit offsets,
  // per-warp digit counts of the chunk (16 bits each), row layout of the
  // tile, digit starts and, in the first pass, the staged chunk
  extern __shared__ __align__(16) unsigned char smem[];
  int64_t* sh_off = reinterpret_cast<int64_t*>(smem);
  int64_t* sh_gstart = sh_off + kRadix;
  unsigned short (*sh_wcnt)[kRadix] = reinterpret_cast<unsigned short (*)[kRadix]>(sh_gstart + kMaxTileRows);
  int* sh_start = reinterpret_cast<int*>(&sh_wcnt[kWarps][0]);
  int* sh_len = sh_start + kMaxTileRows + 1;
  int* sh_dstart = sh_len + kMaxTileRows;  // chunk-local start of each digit
  int* sh_wsum = sh_dstart + kRadix;       // kWarps
  int* stage_key = sh_wsum + kWarps;       // the chunk in sorted order
  int* stage_k = stage_key + kChunk;
  float* stage_v = reinterpret_cast<float*>(stage_k + kChunk);
  const int t = blockIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
    sh_off[d] = off[int64_t(d) * ntiles + t];
#pragma unroll
    for (int x = 0; x < kWarps; x++) sh_wcnt[x][d] = 0;
  }
  RowTile tile{};
  int64_t e0 = 0;
  int nent;
  if (ROWS) {
    load_row_tile(m, rows_per_tile, t, rp, order, sh_start, sh_gstart, sh_len, &tile, bad);
    nent = tile.nent;
  } else {
    e0 = int64_t(t) * kTileEntries;
    nent = int(nent_flat - e0 < kTileEntries ? nent_flat - e0 : kTileEntries);
    __syncthreads();
  }
  for (int c0 = 0; c0 < nent; c0 += kChunk) {
    int dig[kItems], rnk[kItems], kk[kItems];
    int kv[kItems];
    float vv[kItems];
    // load the lane's items first, so that their loads are in flight
    // together, then rank them within the warp in order
    {
      int row = -1;  // ROWS: row of this lane's previous item
#pragma unroll
      for (int it = 0; it < kItems; it++) {
        const int e = c0 + w * (kItems * 32) + it * 32 + lane;
        int c = 0, k = 0;
        float v = 0.f;
        if (e < nent) {
          int64_t q;
          if (ROWS) {
            if (row < 0)
              tile.locate(e, &row, &q);
            else
              tile.advance(e, &row, &q);
            k = int(tile.k0 + row);
          } else {
            q = e0 + e;
            k = __ldg(kin + q);
          }
          c = __ldg(key + q);
          v = __ldg(vin + q);
        }
        kk[it] = c;
        kv[it] = k;
        vv[it] = v;
      }
    }
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      const bool valid = c0 + w * (kItems * 32) + it * 32 + lane < nent;
      int c = kk[it];
      if (c < 0 || c >= n) c = 0;  // flagged by the histogram pass
      const int d = valid ? (c >> shift) & mask : -1;
      const unsigned peers = __match_any_sync(0xffffffffu, valid ? d : kRadix + lane);
      const int r = __popc(peers & lanemask_lt());
      int base = 0;
      if (valid) base = sh_wcnt[w][d];
      __syncwarp();
      if (valid && r == 0) sh_wcnt[w][d] = (unsigned short)(base + __popc(peers));
      __syncwarp();
      dig[it] = d;
      rnk[it] = base + r;
      kk[it] = c;
    }
    __syncthreads();
    // per digit (one per thread): exclusive prefix over the warps, chunk
    // total, and the digit's start in the chunk (exclusive scan of totals)
    static_assert(kRadix == kWarps * 32, "one digit per thread");
    const int dd = threadIdx.x;
    int tot = 0;
#pragma unroll
    for (int x = 0; x < kWarps; x++) {
      const int cnt = sh_wcnt[x][dd];
      sh_wcnt[x][dd] = (unsigned short)tot;
      tot += cnt;
    }
    int incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (!ROWS) {
      // second pass: the input is grouped by the previous digit, so the
      // lanes of a warp mostly share a digit and direct stores coalesce
      __syncthreads();
#pragma unroll
      for (int it = 0; it < kItems; it++) {
        const int d = dig[it];
        if (d >= 0) {
          const int64_t pos = sh_off[d] + sh_wcnt[w][d] + rnk[it];
          if (out_key) out_key[pos] = kk[it];
          out_k[pos] = kv[it];
          out_v[pos] = vv[it];
        }
      }
      __syncthreads();
      sh_off[dd] += tot;
#pragma unroll
      for (int x = 0; x < kWarps; x++) sh_wcnt[x][dd] = 0;
      __syncthreads();
      continue;
    }
    // first pass: neighbouring entries of a row carry neighbouring digits;
    // stage the chunk in sorted order so the stores coalesce
    if (lane == 31) sh_wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      const int v = sh_wsum[lane];
      int x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      sh_wsum[lane] = x - v;
    }
    __syncthreads();
    sh_dstart[dd] = sh_wsum[w] + incl - tot;
    __syncthreads();
    // stage the chunk in sorted order
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      const int d = dig[it];
      if (d >= 0) {
        const int slot = sh_dstart[d] + sh_wcnt[w][d] + rnk[it];
        stage_key[slot] = kk[it];
        stage_k[slot] = kv[it];
        stage_v[slot] = vv[it];
      }
    }
    __syncthreads();
    // write out: consecutive threads, consecutive positions of a digit
    const int cn = nent - c0 < kChunk ? nent - c0 : kChunk;
    for (int i = threadIdx.x; i < cn; i += blockDim.x) {
      const int c = stage_key[i];
      const int d = (c >> shift) & mask;
      const int64_t pos = sh_off[d] + (i - sh_dstart[d]);
      if (out_key) out_key[pos] = c;
      out_k[pos] = stage_k[i];
      out_v[pos] = stage_v[i];
    }
    __syncthreads();
    sh_off[dd] += tot;
#pragma unroll
    for (int x = 0; x < kWarps; x++) sh_wcnt[x][dd] = 0;
    __syncthreads();
  }
}

// dynamic shared memory of rs_scatter; the second pass does not stage
constexpr size_t scatter_smem_bytes(bool staged) {
  return sizeof(int64_t) * (kRadix + kMaxTileRows) + sizeof(unsigned short) * kWarps * kRadix +
         sizeof(int) * (2 * kMaxTileRows + 1 + kRadix + kWarps + (staged ? 3 * kChunk : 0));
}

}  // namespace

bool transpose_radix_plan(int64_t m, int64_t n, int64_t nnz, RadixPlan* p) {
  if (m <= 0 || n <= 0 || nnz <= 0 || n > (int64_t(1) << (2 * kRadixBits))) return false;
  int64_t rows = (kTileEntries * m) / nnz;
  rows = std::max<int64_t>(1, std::min<int64_t>(rows, kMaxTileRows));
  p->rows_per_tile = int(rows);
  p->ntiles_rows = (m + rows - 1) / rows;
  p->ntiles_flat = (nnz + kTileEntries - 1) / kTileEntries;
  // a tile of rows must hold fewer than 2^31 entries
  // the first digit is short (9 bits) where the second still covers the
  // rest: short digits give longer runs per digit in the first scatter
  p->passes = n <= kRadix ? 1 : 2;
  p->bits1 = (p->passes == 1 || n > (int64_t(1) << (2 * kRadixBits - 1))) ? kRadixBits : kRadixBits - 1;
  return p->ntiles_rows < INT32_MAX && p->ntiles_flat < INT32_MAX;
}

int64_t radix_hist_elems(const RadixPlan& p) {
  return int64_t(kRadix) * std::max(p.ntiles_rows, p.ntiles_flat);
}

cudaError_t launch_transpose_radix(const RadixPlan& p, int64_t m, int64_t n, int64_t nnz, const int64_t* rp,
                                   const int32_t* col, const float* val, const int32_t* order, int64_t* hist,
                                   int64_t* off, int64_t* scan_tmp, int32_t* colcnt, int64_t* colcnt64,
                                   int32_t* st_key, int32_t* st_k, float* st_v, int32_t* bad, int64_t* cp,
                                   int32_t* trow, float* tval, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(colcnt, 0, size_t(n) * sizeof(int32_t), s);
  const size_t sm = scatter_smem_bytes(true), sm2 = scatter_smem_bytes(false);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(rs_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(rs_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm2));
  if (e != cudaSuccess) return e;
  const int nt1 = int(p.ntiles_rows);
  const int64_t h1 = int64_t(kRadix) * nt1;
  const int m1 = (1 << p.bits1) - 1;
  // column counts in the last pass (see rs_hist)
  rs_hist<true><<<nt1, kWarps * 32, 0, s>>>(m, n, p.rows_per_tile, 0, rp, col, order, 0, m1, nt1, hist,
                                            p.passes == 1 ? colcnt : nullptr, bad);
  note_launches(1);
  if ((e = launch_scan_i64(hist, h1, off, scan_tmp, s)) != cudaSuccess) return e;
  if (p.passes == 1) {
    rs_scatter<true><<<nt1, kWarps * 32, sm, s>>>(m, n, p.rows_per_tile, 0, rp, col, nullptr, val, order, 0, m1, nt1,
                                                  off, nullptr, trow, tval, bad);
    note_launches(1);
  } else {
    rs_scatter<true><<<nt1, kWarps * 32, sm, s>>>(m, n, p.rows_per_tile, 0, rp, col, nullptr, val, order, 0, m1, nt1,
                                                  off, st_key, st_k, st_v, bad);
    note_launches(1);
    const int nt2 = int(p.ntiles_flat);
    const int64_t h2 = int64_t(kRadix) * nt2;
    rs_hist<false><<<nt2, kWarps * 32, 0, s>>>(m, n, 0, nnz, nullptr, st_key, nullptr, p.bits1, kRadix - 1, nt2,
                                               hist, colcnt, bad);
    note_launches(1);
    if ((e = launch_scan_i64(hist, h2, off, scan_tmp, s)) != cudaSuccess) return e;
    rs_scatter<false><<<nt2, kWarps * 32, sm2, s>>>(m, n, 0, nnz, nullptr, st_key, st_k, st_v, nullptr, p.bits1,
                                                   kRadix - 1, nt2, off, nullptr, trow, tval, bad);
    note_launches(1);
  }
  if ((e = launch_widen_i32(colcnt, n, colcnt64, s)) != cudaSuccess) return e;
  return launch_scan_i64(colcnt64, n, cp, scan_tmp, s);
}

}  // namespace raptr
