// Internal interface between the C ABI (api.cu) and the kernel translation
// units.  Host launch wrappers only; no device code here.
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "common.cuh"

namespace raptr {

// Records msg as this thread's last error (raptr_last_error) and returns st.
raptr_status set_error(raptr_status st, const std::string& msg);

// Process-wide count of kernels launched by this library (diagnostic).
void note_launches(long long k);
long long launches_so_far();

// Device allocations of the library (devmem.cu): blocks are parked for
// reuse when freed instead of going back to the driver;
// dev_free waits for the device like cudaFree.  dev_release returns the
// parked blocks of a device (-1: all) to the driver.
cudaError_t dev_alloc(void** p, size_t bytes);
void dev_free(void* p);
void dev_release(int device);
// Bytes the library may still allocate on `device`: the device's free
// memory plus the library's parked blocks, within RAPTR_DEVICE_MEMORY_LIMIT
// when that is set.
size_t dev_available(int device);
template <class T>
cudaError_t dev_malloc(T** p, size_t bytes) {
  void* q = nullptr;
  cudaError_t e = dev_alloc(&q, bytes);
  *p = static_cast<T*>(q);
  return e;
}

// Host-side phase trace, enabled by the environment variable RAPTR_TRACE=1:
// one line per event on stderr, prefixed with the milliseconds since the
// process's first trace line.  trace_ms() is a host clock in milliseconds.
bool trace_on();
void trace(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
double trace_ms();

// ---- system matrix rows (kernels_sm.cu) ----------------------------------

// Hash/slot capacity levels for the per-channel accumulation table; a row
// whose distinct voxels do not fit is re-run at the next level.
int sm_num_levels();
int sm_level_capacity(int level);   // entries per row slot
int sm_level_threads(int level);
int sm_pick_level(const DGeom& g, int nrays);

// Builds rows [row0, row0+nrows) of the list into staging slots (slot i at
// st_col/st_val + i*capacity).  row_nnz[i] = entries, or -1 if the table
// overflowed.  *d_flags |= 1 on overflow, |= 4 for a channel id out of range.
// With d_table_reasons (4 ints) the rows the dense kernel leaves to the hash
// table are counted by reason: no slab axis, windows over the slot limit,
// a ray outside the windows, a slot decoding outside the grid.  parts: 1 =
// the dense kernel only (rows it cannot take keep row_nnz = -2), 2 = the
// table kernel for those rows only, 3 = both; with d_rays every row takes
// the table kernel whatever parts says.
constexpr int kRowsDense = 1, kRowsTable = 2, kRowsAll = 3;
cudaError_t launch_sm_rows(int level, const DGeom& g, const float2* d_sincos, const int32_t* d_cnl, int64_t row0,
                           int64_t nrows, int nrays, uint32_t seed, const float* d_rays, int32_t* st_col,
                           float* st_val, int32_t* row_nnz, int32_t* d_flags, cudaStream_t s,
                           int32_t* d_table_reasons = nullptr, int parts = kRowsAll);

// Exclusive scan of row_nnz[0..n) into row_ptr[0..n] (int64) starting at
// *d_base; *d_base is advanced by the sum.  One block.
cudaError_t launch_rows_scan(const int32_t* row_nnz, int64_t n, int64_t* row_ptr, int64_t* d_base, cudaStream_t s);

cudaError_t launch_rows_scan_i64(const int64_t* counts, int64_t n, int64_t* row_ptr, int64_t* d_base, cudaStream_t s);

// Copies staged rows to their final CSR position; entries at or beyond
// `capacity` are not written.
cudaError_t launch_rows_gather(const int32_t* st_col, const float* st_val, int slot_cap, const int64_t* row_ptr,
                               int64_t nrows, int64_t capacity, int32_t* col, float* val, cudaStream_t s);

// Keep-zeros expansion of one row block: for every candidate of the row
// (written in order by the workqueue fill), look up its value in the
// zero-free staged row.
cudaError_t launch_expand_candidates(const int32_t* st_col, const float* st_val, int slot_cap, const int32_t* row_nnz,
                                     const int64_t* cand_ptr, int64_t nrows, int32_t* cand_vxl, float* out_val,
                                     cudaStream_t s);

cudaError_t launch_rays(const DGeom& g, const float2* d_sincos, const int32_t* d_cnl, int64_t n, int nrays,
                        uint32_t seed, float* d_rays, cudaStream_t s);

// ---- candidate search (kernels_sm.cu) --------------------------------------

// counts[i] = candidates of list entry li0+i; entry li0 starts at voxel
// start_vxl.  A channel id out of range counts 0 and sets *d_flags |= 4.
cudaError_t launch_wq_count(const DGeom& g, const float2* d_sincos, const int32_t* d_list, int64_t li0, int64_t n,
                            int64_t start_vxl, int64_t* d_counts, int32_t* d_flags, cudaStream_t s);
// Writes candidate k of list entry li0+i to position offsets[i]+k when below
// max_out (d_cnl_out may be null).
cudaError_t launch_wq_fill(const DGeom& g, const float2* d_sincos, const int32_t* d_list, int64_t li0, int64_t n,
                           int64_t start_vxl, const int64_t* d_offsets, int64_t max_out, int32_t* d_cnl_out,
                           int32_t* d_vxl_out, int32_t* d_flags, cudaStream_t s);

// ---- scans and small utilities (kernels_util.cu) ---------------------------

// Exclusive scan of int64 counts into offsets (n+1 entries, offsets[n] = total).
// temp must hold scan_temp_elems(n) int64.
int64_t scan_temp_elems(int64_t n);
cudaError_t launch_scan_i64(const int64_t* in, int64_t n, int64_t* out, int64_t* temp, cudaStream_t s);

cudaError_t launch_coo2csr(const int32_t* rows, int64_t nnz, int64_t m, int64_t* row_ptr, int64_t* temp,
                           cudaStream_t s);
cudaError_t launch_csr2ecsr(int64_t* ecsr, const int32_t* yrow, int64_t nnzr, const int64_t* csr, int64_t m,
                            cudaStream_t s);

// ---- SpMV and MLEM (kernels_mlem.cu) ---------------------------------------

cudaError_t launch_spmv(int op, int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val,
                        float alpha, const float* x, float beta, float* y, cudaStream_t s);
cudaError_t launch_divides(float* r, const float* a, const float* b, int64_t n, cudaStream_t s);
cudaError_t launch_divides_multiplies(float* r, const float* a, const float* b, const float* c, int64_t n,
                                      cudaStream_t s);
cudaError_t launch_scales(float* x, float alpha, int64_t n, cudaStream_t s);
cudaError_t launch_sum(const float* x, int64_t n, double* d_acc, cudaStream_t s);
cudaError_t launch_column_sums(int64_t m, const int64_t* rp, const int32_t* col, const float* val, double* s64,
                               cudaStream_t s);
// s64[j] = sum of column j through the transpose (warp per column, no atomics).
cudaError_t launch_column_sums_csc(int64_t n, const int64_t* cp, const float* tval, double* s64, cudaStream_t s);
// s32 = s64 / sum(s64) with the sum taken inside (one CTA, fixed order).
cudaError_t launch_sens_normalise_self(int64_t n, const double* s64, float* s32, cudaStream_t s);
cudaError_t launch_sum_f64(const double* x, int64_t n, double* d_acc, cudaStream_t s);

// c += A^T (y / (A x)); when d_ll is non-null, d_ll[0] += sum y*log(Ax),
// d_ll[1] += sum Ax (FP64).
cudaError_t launch_mlem_project(int64_t m, const int64_t* rp, const int32_t* col, const float* val, const float* y,
                                const float* x, float* c, double* d_ll, cudaStream_t s);
// x = x*c/(s + (s==0)); d_acc[0] += sum(x) (FP64).
// The projection of launch_mlem_project for rows in the build's staging
// slots (row i at st_col/st_val + i*cap, row_nnz[i] entries; rows with
// row_nnz < 0 skipped); with s64 non-null also s64[col] += val (FP64) for
// every built row.
cudaError_t launch_stage_project(int64_t nrows, const int32_t* st_col, const float* st_val, int cap,
                                 const int32_t* row_nnz, const float* y, const float* x, float* c, double* s64,
                                 cudaStream_t s);
cudaError_t launch_mlem_update(int64_t n, float* x, const float* c, const float* sens, double* d_acc, cudaStream_t s);
// x *= float(1/float(d_acc[0])); c = 0; d_acc[0] reset by the next project.
cudaError_t launch_mlem_normalise(int64_t n, float* x, float* c, double* d_acc, cudaStream_t s);
cudaError_t launch_mlem_normalise_from(int64_t n, float* x, const float* xx, double* d_acc, cudaStream_t s);
cudaError_t launch_zero_f64(double* p, int64_t n, cudaStream_t s);

// Transpose (CSC) of a CSR matrix: column counts (int32 atomics), widening to
// int64, and the fill through per-column cursors (initialised to col_ptr).
// ---- precision forms (kernels_precision.cu) --------------------------------

// FP16 copy of a matrix: rscale (m), hval (nnz, CSR order), htval (nnz,
// order of the transpose trow/tval, whose index is a position in `order`
// or the row when order is null), pscale (m, rscale by position).
cudaError_t launch_half_convert(int64_t m, int64_t nnz, const int64_t* rp, const float* val, const int32_t* trow,
                                const float* tval, const int32_t* order, float* rscale, uint16_t* hval,
                                uint16_t* htval, float* pscale, cudaStream_t s);
// FP64 column sums of the FP16 matrix through its transpose.
cudaError_t launch_sens_half(int64_t n, const int64_t* cp, const int32_t* trow, const uint16_t* htval,
                             const float* pscale, double* s64, cudaStream_t s);
// e[rank_i] = rscale_i * y_i / (A x)_i (0 where y_i == 0).
cudaError_t launch_mlem_forward_half(int64_t m, const int64_t* rp, const int32_t* col, const uint16_t* hval,
                                     const float* rscale, const float* y, const float* x, const int32_t* rank,
                                     float* e, double* d_ll, cudaStream_t s, unsigned long long* next = nullptr);
// Delta-coded FP16 runs (rows of the FP16 matrix or columns of its
// transpose): word = (h << 16) | index step, runs starting on quads of four
// words.  launch_pack_count writes the quads of each of the cnt runs of
// (ptr, idx) into quads[0..cnt) (*bad |= 1 on a descending index);
// launch_pack_fill writes the anchors and words of the runs, run r from
// word 4*qoff[r] (qoff: the exclusive scan of the quads).
cudaError_t launch_pack_count(int64_t cnt, const int64_t* ptr, const int32_t* idx, int64_t* quads, int32_t* bad,
                              cudaStream_t s);
cudaError_t launch_pack_fill(int64_t cnt, const int64_t* ptr, const int32_t* idx, const uint16_t* hv,
                             const int64_t* qoff, int32_t* anchor, uint32_t* words, cudaStream_t s);
// The FP16 passes over delta-coded runs (16-byte aligned words): as
// launch_mlem_forward_half / launch_mlem_back_half, with `next` required
// (an 8-byte counter, zero at launch).
cudaError_t launch_mlem_forward_packed(int64_t m, const int64_t* seg, const int32_t* anchor, const uint32_t* words,
                                       const float* rscale, const float* y, const float* x, const int32_t* rank,
                                       float* e, double* d_ll, unsigned long long* next, cudaStream_t s);
cudaError_t launch_mlem_back_packed(int64_t n, const int64_t* seg, const int32_t* anchor, const uint32_t* words,
                                    const float* e, const float* x, const float* sens, float* out, double* d_acc,
                                    bool update, unsigned long long* next, cudaStream_t s);
// c_j = sum h_kj e_k, compensated; with update and `next` as launch_mlem_back.
cudaError_t launch_mlem_back_half(int64_t n, const int64_t* cp, const int32_t* trow, const uint16_t* htval,
                                  const float* e, const float* x, const float* sens, float* out, double* d_acc,
                                  bool update, cudaStream_t s, unsigned long long* next = nullptr);
// One MLEM iteration with FP64 vectors (x, e, xx: n / m / n doubles, acc one
// double); s64 is the normalised sensitivity.
cudaError_t launch_mlem_f64_iteration(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val,
                                      const int64_t* cp, const int32_t* trow, const float* tval, const int32_t* rank,
                                      const float* y, const double* s64, double* x, double* e, double* xx,
                                      double* acc, double* d_ll, cudaStream_t s);

// ---- batched MLEM (kernels_batch.cu) ---------------------------------------

// K frames over one matrix (FP16 values with row scales when half, else
// FP32); X, Y frame-minor (n x K, m x K); E (m x K) and XX (n x K) scratch.
struct BatchArgs {
  int64_t m = 0, n = 0;
  int K = 0;
  bool half = false;
  const int64_t* rp = nullptr;
  const int32_t* col = nullptr;
  const void* val = nullptr;
  const float* rscale = nullptr;
  const int64_t* cp = nullptr;
  const int32_t* trow = nullptr;
  const void* tval = nullptr;
  const int32_t* rank = nullptr;
  const int32_t* col_order = nullptr;  // back-pass column order (may be null)
  const float* Y = nullptr;
  const float* S = nullptr;
  float* X = nullptr;
  float* E = nullptr;
  float* XX = nullptr;
  // Row blocks of the transpose's order for the back pass (may be null):
  // seg (n x (seg_blocks+1) int32, launch_block_seg) and the partial sums P
  // (n x the largest tile floats).
  const int32_t* seg = nullptr;
  int seg_blocks = 0;
  float* P = nullptr;
  // n x the largest tile floats (may be null): a tile narrower than the
  // batch gathers its images from a compact copy here
  float* Xt = nullptr;
};
// The row-block offsets of every column of a transpose (see BatchArgs.seg):
// seg[j*(B+1) + b] = offset in column j of its first entry with row >= b*m/B.
cudaError_t launch_block_seg(int64_t n, int64_t m, int B, const int64_t* cp, const int32_t* trow, int32_t* seg,
                             cudaStream_t s);
// K frames (a multiple of 4) in tiles of at most kt (4, 8, 16, 32 or 64).
bool batch_tile_supported(int K, int kt);
// The tile that starts at frame f0: kt while kt frames remain, else the
// largest power of two that fits.
int batch_tile_at(int K, int kt, int f0);
// One iteration for all K frames in tiles of at most kt frames (acc: K
// doubles, next: K/4 * max(1, seg_blocks) work counters, both scratch);
// ev_mid, when set, is recorded between the two passes.
cudaError_t launch_batch_iteration(const BatchArgs& a, int kt, double* acc, unsigned long long* next, cudaStream_t s,
                                   cudaEvent_t ev_mid);

// Back-projection order of a list of channels (kernels_util.cu): key per
// channel in [0, channel_order_keys(g)); mark counts keys (bad |= 1 on a
// repeated key or a channel out of range); with prefix = exclusive scan of
// mark, rank[r] = prefix[key(cnl[r])] and order[rank[r]] = r.
int64_t channel_order_keys(const DGeom& g);
cudaError_t launch_channel_order_mark(const DGeom& g, int64_t m, const int32_t* cnl, unsigned long long* mark,
                                      int32_t* bad, cudaStream_t s);
cudaError_t launch_channel_order_rank(const DGeom& g, int64_t m, const int32_t* cnl, const int64_t* prefix,
                                      int32_t* rank, int32_t* order, cudaStream_t s);

// Radix-sort CSR -> CSC (kernels_transpose.cu): the same result as the
// blocked transpose below, for n <= 2^20.  Buffers: hist and off
// radix_hist_elems(plan) (+1 for off) int64, scan_tmp
// scan_temp_elems(max(radix_hist_elems, n)) int64, colcnt n int32, colcnt64
// n int64, staging st_key / st_k / st_v nnz each (unused when n <= 1024),
// bad one int32 (|= 1 for an index out of range).
struct RadixPlan {
  int rows_per_tile = 0;
  int passes = 0;
  int bits1 = 0;  // bits of the first digit
  int64_t ntiles_rows = 0, ntiles_flat = 0;
};
bool transpose_radix_plan(int64_t m, int64_t n, int64_t nnz, RadixPlan* p);
int64_t radix_hist_elems(const RadixPlan& p);
cudaError_t launch_transpose_radix(const RadixPlan& p, int64_t m, int64_t n, int64_t nnz, const int64_t* rp,
                                   const int32_t* col, const float* val, const int32_t* order, int64_t* hist,
                                   int64_t* off, int64_t* scan_tmp, int32_t* colcnt, int64_t* colcnt64,
                                   int32_t* st_key, int32_t* st_k, float* st_v, int32_t* bad, int64_t* cp,
                                   int32_t* trow, float* tval, cudaStream_t s);

// Deterministic CSR -> CSC (rows ascending in the order `order`, or
// natural order when null, within each column).  cnt holds B*n int32,
// colcount n int64, scan_tmp scan_temp_elems(n) int64, bad one int32 that
// is set when an index is out of range.
int transpose_blocks(int64_t m, int64_t n);
cudaError_t launch_transpose_blocked(int64_t m, int64_t n, int B, const int64_t* rp, const int32_t* col,
                                     const float* val, const int32_t* order, bool positions, int32_t* cnt,
                                     int64_t* colcount, int64_t* scan_tmp, int32_t* bad, int64_t* cp, int32_t* trow,
                                     float* tval, cudaStream_t s);
// e_i = y_i / (A x)_i (0 for y_i == 0); optional FP64 log-likelihood sums.
// With `next` (an 8-byte counter, zero at launch) the warps draw rows from
// it, kRowChunk at a time.
cudaError_t launch_mlem_forward(int64_t m, const int64_t* rp, const int32_t* col, const float* val, const float* y,
                                const float* x, const int32_t* rank, float* e, double* d_ll, cudaStream_t s,
                                unsigned long long* next = nullptr);
// c_j = (A^T e)_j by columns; with update: out = x*c/(s+(s==0)), d_acc += sum.
// With `next` (an 8-byte counter, zero at launch) the warps draw columns
// from it instead of taking them by a grid stride.
cudaError_t launch_mlem_back(int64_t n, const int64_t* cp, const int32_t* trow, const float* tval, const float* e,
                             const float* x, const float* sens, float* out, double* d_acc, bool update,
                             cudaStream_t s, unsigned long long* next = nullptr);
cudaError_t launch_iota(int32_t* p, int64_t n, cudaStream_t s);
cudaError_t launch_fill(float* p, float v, int64_t n, cudaStream_t s);
cudaError_t launch_narrow_i64(const int64_t* in, int64_t n, int32_t* out, cudaStream_t s);
cudaError_t launch_widen_i32(const int32_t* in, int64_t n, int64_t* out, cudaStream_t s);

// MLEM with its workspace in a fixed device array (mlem_noalloc.cu).
raptr_status mlem_noalloc(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val,
                          const float* y, const float* s, float* x, int32_t n_iter, cudaStream_t st,
                          std::string* err);

}  // namespace raptr
