/*
 * raptr_b200 -- C ABI of the B200 (sm_100a) reconstruction hot path of raptr.
 *
 * Plain C types only: device buffers are raw pointers allocated by the caller
 * (cudaMalloc or any allocator), sizes are int64_t, a CUDA stream is passed
 * as `void *` (a cudaStream_t; NULL = the legacy default stream).  Every call
 * is stream-ordered unless documented otherwise, returns a raptr_status and
 * never aborts; raptr_last_error() describes the last failure of the calling
 * thread.
 *
 * Reference interfaces replaced (paths relative to the raptr source tree):
 *   raptr_workqueue        getWorkqueue            src/getWorkqueue.hpp:149-155, :207-212
 *   raptr_rays             RandRayGen              src/RayGenerators.hpp:36-67
 *   raptr_sm_build         systemMatrixCalculation src/wrappers.hpp:185-196
 *                          (kernel getSystemMatrix src/getSystemMatrixDeviceOnly.cu:357-384,
 *                           cooSort src/cooSort.hpp:75-99,
 *                           convertCoo2Csr src/cusparseWrapper.hpp:53-60,
 *                           convertCsr2Ecsr src/convertCsr2Ecsr.hpp:51-64)
 *   raptr_coo2csr          convertCoo2Csr          src/cusparseWrapper.hpp:53-60
 *   raptr_csr2ecsr         convertCsr2Ecsr         src/convertCsr2Ecsr.hpp:51-64
 *   raptr_spmv             CSRmv<float>            src/csrmv.hpp:61-66, :72-83
 *   raptr_divides          divides                 src/mlemOperations.hpp:44-54
 *   raptr_divides_multiplies dividesMultiplies     src/mlemOperations.hpp:88-104
 *   raptr_scales           scales                  src/mlemOperations.hpp:146-153
 *   raptr_sum              sum                     src/mlemOperations.hpp:163-169
 *   raptr_mlem             MLEM loop               src/tests/reco.cu:229-321
 *   raptr_mlem_stream      chunked MLEM loop       src/tests/reco.cu:226-275, src/wrappers.hpp:429-464
 *   raptr_reco_host        reco main flow          src/tests/reco.cu:53-352
 */
#ifndef RAPTR_B200_H
#define RAPTR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RAPTR_ABI_VERSION 6

typedef enum raptr_status {
  RAPTR_OK = 0,
  RAPTR_ERR_INVALID = 1,     /* bad argument (null pointer, size, geometry)        */
  RAPTR_ERR_CUDA = 2,        /* a CUDA runtime call failed                          */
  RAPTR_ERR_CAPACITY = 3,    /* caller buffer too small; required size returned     */
  RAPTR_ERR_OVERFLOW = 4,    /* an internal per-row table overflowed (after retry)  */
  RAPTR_ERR_NOMEM = 5,       /* device allocation failed                            */
  RAPTR_ERR_UNSUPPORTED = 6, /* feature not available for these arguments           */
  RAPTR_ERR_TIMEOUT = 7      /* a wait ended before the work finished               */
} raptr_status;

/* Scanner geometry.  Field meaning and units as in DefaultVoxelGrid
 * (src/VoxelGrid.hpp:151-176: grid origin, voxel pitch, voxel counts) and
 * DefaultMeasurementSetup (src/MeasurementSetup.hpp:181-220).  Voxel linear
 * id = ix*ny*nz + iy*nz + iz (src/VoxelGridLinIndex.hpp:74-80); channel
 * linear id = (((ida*n0z + id0z)*n0y + id0y)*n1z + id1z)*n1y + id1y
 * (src/MeasurementSetupLinIndex.hpp:82-91). */
typedef struct raptr_geom {
  float grid_o[3];
  float grid_d[3];
  int32_t grid_n[3];
  float pos0x, pos1x;
  int32_t na, n0z, n0y, n1z, n1y;
  float da, segx, segy, segz;
} raptr_geom;

/* A per-geometry device context: the per-angle sine/cosine table, the
 * device it lives on and reusable scratch.  Contexts are independent (no
 * global state), so geometries can be served side by side.  A context may
 * be used from one host thread at a time. */
typedef struct raptr_ctx raptr_ctx;

/* A system matrix held by the library in device memory (CSR, int64 row
 * pointers, int32 columns, float values). */
typedef struct raptr_matrix raptr_matrix;

int raptr_abi_version(void);
const char* raptr_last_error(void);
/* Number of kernels this library has launched in this process (kernels
 * replayed from a CUDA graph included). */
int64_t raptr_kernel_launches(void);

/* No counterpart in the reference (it frees its buffers with cudaFree).
 * Device blocks that the library frees (matrices, their transposes,
 * transpose staging, build scratch, counters) are kept for reuse by its
 * next allocations of a similar size, up to two thirds of each device's memory,
 * because freeing and reallocating tens of GB per reconstruction job costs
 * host time while the device idles.  Freeing still waits for the device's
 * work, as cudaFree does.  raptr_trim_memory returns the kept blocks of
 * `device` (-1: every device) to the driver, e.g. before the caller
 * allocates much device memory by other means; the library also does so by
 * itself when one of its allocations fails. */
raptr_status raptr_trim_memory(int device);

raptr_status raptr_ctx_create(const raptr_geom* geom, int device, raptr_ctx** out);
raptr_status raptr_ctx_destroy(raptr_ctx* ctx);
int64_t raptr_ctx_num_channels(const raptr_ctx* ctx);
int64_t raptr_ctx_num_voxels(const raptr_ctx* ctx);

/* ---- candidate search (getWorkqueue) ------------------------------------ */

/* Enclosing-cylinder candidates (channel, voxel) of the listed channels in
 * the reference's scan order (list-major, voxel-minor), starting at the
 * cursor (*list_id, *vxl_id) and returning at most max_out entries.  On
 * return the cursor points one voxel past the last entry returned (next list
 * entry at the end of the grid; (n_list, 0) when exhausted), as
 * getWorkqueueEntry leaves it (src/getWorkqueue.hpp:53-133).  d_cnl_out and
 * d_vxl_out hold max_out entries.  Synchronises the stream (the count and
 * cursor are host values). */
raptr_status raptr_workqueue(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int64_t* list_id,
                             int64_t* vxl_id, int64_t max_out, int32_t* d_cnl_out, int32_t* d_vxl_out,
                             int64_t* n_found, void* stream);

/* Number of candidates of each listed channel (d_counts: n_list int64). */
raptr_status raptr_candidate_counts(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int64_t* d_counts,
                                    void* stream);

/* ---- rays ------------------------------------------------------------------ */

/* Endpoints of rays [0, nrays) of each listed channel: d_rays holds
 * n_list*nrays*6 floats (x0,y0,z0,x1,y1,z1).  Uniforms come from
 * Philox4x32-10 with key (seed, channel) and counter (ray, 0|1, 0, 0); the
 * reference draws them from curand XORWOW instead (src/RayGenerators.hpp:44). */
raptr_status raptr_rays(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int32_t nrays, uint32_t seed,
                        float* d_rays, void* stream);

/* ---- system matrix --------------------------------------------------------- */

#define RAPTR_SM_KEEP_ZEROS 1 /* keep every candidate, also exact zeros (the reference's COO structure) */

/* Rows of the system matrix for the listed channels, row i <-> d_cnl_ids[i]
 * (the reference's ECSR row space).  Element (i, v) = mean over rays of the
 * intersection length of ray r with voxel v, for every voxel v that passes
 * the enclosing-cylinder test; exact zeros are dropped unless
 * RAPTR_SM_KEEP_ZEROS.  Columns ascend within a row.  Rays come from
 * d_rays (n_list*nrays*6 floats) when non-null, else from the Philox stream
 * of raptr_rays.
 *
 * Output goes to caller buffers: d_row_ptr (n_list+1 int64), d_col/d_val
 * (capacity entries).  If the matrix has more than `capacity` entries the
 * call returns RAPTR_ERR_CAPACITY with *nnz_out = the required count and
 * the row pointers filled (call again with a larger buffer).  Synchronises
 * the stream. */
raptr_status raptr_sm_build(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int32_t nrays, uint32_t seed,
                            const float* d_rays, int32_t flags, int64_t capacity, int64_t* d_row_ptr, int32_t* d_col,
                            float* d_val, int64_t* nnz_out, void* stream);

/* Same build into a matrix allocated and owned by the library (resident in
 * HBM until raptr_matrix_destroy). */
raptr_status raptr_sm_build_alloc(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int32_t nrays,
                                  uint32_t seed, const float* d_rays, int32_t flags, raptr_matrix** out,
                                  void* stream);
raptr_status raptr_matrix_info(const raptr_matrix* A, int64_t* m, int64_t* n, int64_t* nnz, int64_t** d_row_ptr,
                               int32_t** d_col, float** d_val);
raptr_status raptr_matrix_destroy(raptr_matrix* A);

/* Transpose (CSC) of the library matrix, built once and kept resident beside
 * the CSR (same values, grouped by voxel): back projection then gathers by
 * columns instead of scattering with atomics.  Synchronises the stream.
 * The columns list the rows in the matrix's back-projection order: channels
 * sorted by (angle, z0+z1, y0+y1, z0-z1, y0-y1), so that the channels
 * crossing one voxel are few dense runs of that order.  The CSC's row
 * index is then the position k in that order (row = order[k]; see
 * raptr_matrix_row_order) and a vector it is applied to is laid out the
 * same way (raptr_mlem_forward_ordered writes it so).  A matrix whose list
 * repeats a channel keeps the natural order (order and rank null, the row
 * index is the row).  Entries within a column are ascending in k, so
 * results do not depend on scheduling. */
raptr_status raptr_matrix_transpose(raptr_matrix* A, void* stream);
/* Pointers of the transpose (null until raptr_matrix_transpose). */
raptr_status raptr_matrix_csc_info(const raptr_matrix* A, int64_t** d_col_ptr, int32_t** d_row_idx, float** d_tval);
/* Back-projection order of the rows after raptr_matrix_transpose:
 * d_order[k] = row at position k, d_rank[row] = its position (m int32 each);
 * both null for the natural order. */
raptr_status raptr_matrix_row_order(const raptr_matrix* A, int32_t** d_order, int32_t** d_rank);

/* ---- sparse formats --------------------------------------------------------- */

/* CSC of an m x n CSR matrix into caller buffers: d_col_ptr (n+1 int64),
 * d_row_idx and d_tval (nnz each).  Within a column the rows are ascending
 * (the result does not depend on scheduling).  Replaces the transposed
 * cusparse csrmv of src/csrmv.hpp:61-66 as a stored CSC.  Synchronises the
 * stream; column indices outside [0, n) give RAPTR_ERR_INVALID. */
raptr_status raptr_csr_transpose(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                                 const float* d_val, int64_t* d_col_ptr, int32_t* d_row_idx, float* d_tval,
                                 void* stream);
/* The same with the rows taken in a caller order: d_order (m int32) is a
 * permutation of [0, m), row d_order[k] is the k-th; within each column the
 * entries are ascending in k and d_pos_idx holds k instead of the row.  No
 * counterpart in the reference.  Back projection through this CSC reads a
 * vector laid out in the same order (v_k = e[d_order[k]]); an order that
 * puts rows crossing the same voxels next to each other makes those reads
 * dense. */
raptr_status raptr_csr_transpose_ordered(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                                         const float* d_val, const int32_t* d_order, int64_t* d_col_ptr,
                                         int32_t* d_pos_idx, float* d_tval, void* stream);

/* Row pointers (m+1 int64) from sorted COO row indices (nnz int32). */
raptr_status raptr_coo2csr(const int32_t* d_rows, int64_t nnz, int64_t m, int64_t* d_row_ptr, void* stream);

/* ECSR row pointers: d_ecsr[i] = d_csr[d_yrow[i]], d_ecsr[nnzr] = d_csr[m]. */
raptr_status raptr_csr2ecsr(int64_t* d_ecsr, const int32_t* d_yrow, int64_t nnzr, const int64_t* d_csr, int64_t m,
                            void* stream);

/* Row pointers between the reference's int32 CSR (src/cusparseWrapper.hpp:53-60,
 * src/csrmv.hpp:61-66) and the int64 ones used here.  Narrowing checks the
 * last (largest) pointer and returns RAPTR_ERR_INVALID when it exceeds
 * INT32_MAX; it synchronises the stream for that check. */
raptr_status raptr_row_ptr_narrow(const int64_t* d_in, int64_t n, int32_t* d_out, void* stream);
raptr_status raptr_row_ptr_widen(const int32_t* d_in, int64_t n, int64_t* d_out, void* stream);

/* ---- SpMV ---------------------------------------------------------------- */

#define RAPTR_OP_N 0 /* y = alpha*A*x   + beta*y  (forward projection) */
#define RAPTR_OP_T 1 /* y = alpha*A^T*x + beta*y  (back projection)    */

/* The CSRmv contract (src/csrmv.hpp:31-66) on an m x n CSR matrix with
 * int64 row pointers.  beta == 0 does not read y. */
raptr_status raptr_spmv(int32_t op, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                        const float* d_val, float alpha, const float* d_x, float beta, float* d_y, void* stream);

/* ---- element-wise MLEM operations --------------------------------------- */

raptr_status raptr_divides(float* d_res, const float* d_dividend, const float* d_divisor, int64_t n, void* stream);
raptr_status raptr_divides_multiplies(float* d_res, const float* d_a, const float* d_b, const float* d_c, int64_t n,
                                      void* stream);
raptr_status raptr_scales(float* d_x, float alpha, int64_t n, void* stream);
/* Sum of d_x, accumulated in double; synchronises the stream. */
raptr_status raptr_sum(const float* d_x, int64_t n, double* sum_out, void* stream);

/* ---- sensitivity and MLEM ------------------------------------------------- */

/* Column sums of A in double (d_s64, n entries, overwritten) and, when
 * d_s32 is non-null, the same image normalised to sum 1 in float. */
raptr_status raptr_sensitivity(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                               const float* d_val, double* d_s64, float* d_s32, void* stream);
/* The same through the transpose (its column pointers and values): no
 * atomics, so the sums come out the same on every run; about six times
 * faster than the CSR form at 70^3 x 5.14M channels. */
raptr_status raptr_sensitivity_csc(int64_t n, const int64_t* d_col_ptr, const float* d_tval, double* d_s64,
                                   float* d_s32, void* stream);

typedef struct raptr_mlem_opts {
  int32_t use_graph;   /* capture the iteration loop in a CUDA graph            */
  double* h_loglik;    /* optional: per-iteration Poisson log-likelihood (FP64)  */
  float* h_kernel_ms;  /* optional: 2*n_iter device times (ms) of the two passes of
                          each iteration, from CUDA events on the stream; when
                          set the loop is launched without a graph             */
  const int32_t* d_row_rank; /* optional, with the transpose: the CSC's row
                          index is the position in an order, d_row_rank[row]
                          the row's position (raptr_matrix_row_order)         */
} raptr_mlem_opts;

/* n_iter MLEM iterations in the order of src/tests/reco.cu:230-303:
 * yt = A x; e = y / yt; c = A^T e; x = x*c/(s + (s==0)); x *= 1/sum(x).
 * Rows of A correspond to d_y; rows with y == 0 are not measured and are
 * skipped (the reference's matrix has no such rows).  d_s is the normalised
 * sensitivity.  d_x is updated in place.  With the transpose given
 * (d_col_ptr, d_row_idx, d_tval non-null) an iteration is two gather passes
 * (rows, then columns, with the ratio and the update fused into them);
 * without it, one pass over the rows that scatters the back projection with
 * atomics. */
raptr_status raptr_mlem(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                        const float* d_val, const int64_t* d_col_ptr, const int32_t* d_row_idx, const float* d_tval,
                        const float* d_y, const float* d_s, float* d_x, int32_t n_iter, const raptr_mlem_opts* opts,
                        void* stream);

/* The two halves of one MLEM iteration, for callers that combine partial
 * back projections across devices (row-sharded matrix):
 *   raptr_mlem_project: d_c += A^T (d_y / (A d_x)) over the rows of this
 *     shard (rows with y == 0 skipped); when d_ll is non-null, d_ll[0] +=
 *     sum y*log(Ax) and d_ll[1] += sum Ax in FP64;
 *   raptr_mlem_update: d_x = d_x*d_c/(d_s + (d_s==0)); d_x *= 1/sum(d_x);
 *     d_c = 0.  d_acc is one double of device scratch. */
raptr_status raptr_mlem_project(int64_t m, const int64_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                                const float* d_y, const float* d_x, float* d_c, double* d_ll, void* stream);
raptr_status raptr_mlem_update(int64_t n, float* d_x, float* d_c, const float* d_s, double* d_acc, void* stream);
/* The same halves on the row/column pair:
 *   raptr_mlem_forward: d_e = d_y / (A d_x) over the rows of this shard
 *     (0 where y == 0), optional FP64 log-likelihood sums into d_ll[0..1];
 *   raptr_mlem_back: d_c = A^T d_e by columns (this shard's partial sums). */
raptr_status raptr_mlem_forward(int64_t m, const int64_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                                const float* d_y, const float* d_x, float* d_e, double* d_ll, void* stream);
raptr_status raptr_mlem_back(int64_t n, const int64_t* d_col_ptr, const int32_t* d_row_idx, const float* d_tval,
                             const float* d_e, float* d_c, void* stream);
/* raptr_mlem_forward storing e_i at d_e[d_row_rank[i]], the layout that
 * raptr_mlem_back reads through a transpose in that order. */
raptr_status raptr_mlem_forward_ordered(int64_t m, const int64_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                                        const float* d_y, const float* d_x, const int32_t* d_row_rank, float* d_e,
                                        double* d_ll, void* stream);

/* ---- precision forms ------------------------------------------------------
 * No counterpart in the reference (FP32 throughout, src/tests/reco.cu).
 *
 * FP16 system matrix: a_ij ~= rscale_i * h_ij with h IEEE binary16 (as
 * uint16_t bits) and rscale_i = max_j |a_ij| * 2^-15, so h <= 32768.  The
 * matrix keeps h in CSR order (d_hval) and in the order of its transpose
 * (d_htval), and the row scales by row (d_rscale) and by position of the
 * transpose (d_pscale).  Requires raptr_matrix_transpose; synchronises. */
raptr_status raptr_matrix_half(raptr_matrix* A, void* stream);
raptr_status raptr_matrix_half_info(const raptr_matrix* A, uint16_t** d_hval, float** d_rscale, uint16_t** d_htval,
                                    float** d_pscale);
/* Frees the FP32 values of the CSR and its transpose once the FP16 form
 * exists (the FP16 iterations need only indices and binary16 values);
 * raptr_matrix_info / raptr_matrix_csc_info then return null values. */
raptr_status raptr_matrix_drop_f32(raptr_matrix* A);
/* Device bytes held by the matrix (all its forms). */
raptr_status raptr_matrix_bytes(const raptr_matrix* A, int64_t* bytes);
/* FP64 column sums of the FP16 matrix (through its transpose), and the same
 * normalised to sum 1 in float when d_s32 is non-null. */
raptr_status raptr_sensitivity_half(int64_t n, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                                    const uint16_t* d_htval, const float* d_pscale, double* d_s64, float* d_s32,
                                    void* stream);
/* raptr_mlem with the FP16 matrix: FP32 vectors and accumulation, the back
 * projection's compensated; the transpose is required (opts->d_row_rank as
 * for raptr_mlem).  Per entry 6 matrix bytes per pass instead of 8. */
raptr_status raptr_mlem_half(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                             const uint16_t* d_hval, const float* d_rscale, const int64_t* d_col_ptr,
                             const int32_t* d_row_idx, const uint16_t* d_htval, const float* d_y, const float* d_s,
                             float* d_x, int32_t n_iter, const raptr_mlem_opts* opts, void* stream);
/* Delta-coded FP16 runs, 4 bytes per entry instead of 6: each of the count
 * runs of (d_ptr, d_idx, d_hv) -- the rows of a CSR with its binary16
 * values, or the columns of its transpose -- as 32-bit words (h << 16) | d,
 * d the run's index step from the previous word (from the run's anchor,
 * its first index, for the first word).  A step above 65535 takes extra
 * words of step 65535 and value 0 before the entry's word.  Run r holds
 * the words [4*d_seg[r], 4*d_seg[r+1]) (offsets in quads of four words; a
 * run's last quad is padded with words 0); d_anchor[r] is its first index
 * (0 for an empty run).  Indices must ascend within a run.
 * Two phases: with d_words null, fills d_seg (count + 1 int64) and
 * *h_words (the words needed); then, with d_words (16-byte aligned,
 * words_cap >= *h_words) and d_anchor (count int32), the runs.
 * Synchronises. */
raptr_status raptr_pack_half(int64_t count, const int64_t* d_ptr, const int32_t* d_idx, const uint16_t* d_hv,
                             int64_t* d_seg, int32_t* d_anchor, uint32_t* d_words, int64_t words_cap,
                             int64_t* h_words, void* stream);
/* The matrix's FP16 form delta-coded (raptr_pack_half of its CSR and of its
 * transpose, kept with the matrix); requires raptr_matrix_half.  Synchronises. */
raptr_status raptr_matrix_packed(raptr_matrix* A, void* stream);
raptr_status raptr_matrix_packed_info(const raptr_matrix* A, int64_t** d_seg, int32_t** d_anchor,
                                      uint32_t** d_words, int64_t** d_tseg, int32_t** d_tanchor,
                                      uint32_t** d_twords);
/* raptr_mlem_half over the delta-coded runs: rows (d_seg, d_anchor,
 * d_words) with the row scales d_rscale, columns of the transpose (d_tseg,
 * d_tanchor, d_twords) in the order opts->d_row_rank gives (as for
 * raptr_mlem_half).  The same values and accumulation as raptr_mlem_half;
 * per entry 4 matrix bytes per pass instead of 6. */
raptr_status raptr_mlem_packed(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_seg, const int32_t* d_anchor,
                               const uint32_t* d_words, const float* d_rscale, const int64_t* d_tseg,
                               const int32_t* d_tanchor, const uint32_t* d_twords, const float* d_y,
                               const float* d_s, float* d_x, int32_t n_iter, const raptr_mlem_opts* opts,
                               void* stream);
/* The same iteration with FP64 vectors and accumulation over the FP32
 * matrix (the reference for the FP32 and FP16 images): d_s64 is the
 * normalised sensitivity, d_x64 the image (updated in place); h_loglik,
 * when non-null, receives n_iter log-likelihoods.  Synchronises. */
raptr_status raptr_mlem_f64(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                            const float* d_val, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                            const float* d_tval, const int32_t* d_row_rank, const float* d_y, const double* d_s64,
                            double* d_x64, int32_t n_iter, double* h_loglik, void* stream);

/* ---- batched frames -------------------------------------------------------
 * No counterpart in the reference (one measurement per run).  n_frames
 * reconstructions that share one system matrix, iterated together: d_y
 * (m x n_frames) and d_x (n x n_frames) are frame-minor (y[i*n_frames + f]),
 * d_s is the one normalised sensitivity; each frame's image is normalised
 * to sum 1 after every iteration.  The matrix is FP32 (value_type 0: d_val /
 * d_tval float) or the FP16 form (value_type 1: d_val = hval, d_tval =
 * htval, d_rscale the row scales).  The transpose is required and d_row_rank
 * follows it (raptr_matrix_row_order, may be null for the natural order).  When one
 * frame tile's ratios exceed ~96 MB, the back pass runs over groups of row
 * blocks of the transpose so that the ratios it gathers stay in L2.
 * n_frames must be a multiple of 4.  Each pass handles up to frame_tile
 * frames per sweep of the matrix (4, 8, 16, 32 or 64; 0 = 32): tiles of
 * frame_tile frames while that many remain, then the largest power of two
 * that fits (40 frames at 32: 32 + 8).  d_x and d_y must be 16-byte
 * aligned.
 * opts: use_graph captures the n_iter iterations in a CUDA graph;
 * h_kernel_ms receives per iteration the forward and back-pass times. */
raptr_status raptr_mlem_batch(raptr_ctx* ctx, int64_t m, int64_t n, int32_t n_frames, int32_t value_type,
                              const int64_t* d_row_ptr, const int32_t* d_col, const void* d_val,
                              const float* d_rscale, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                              const void* d_tval, const int32_t* d_row_rank, const float* d_y, const float* d_s,
                              float* d_x, int32_t n_iter, int32_t frame_tile, const raptr_mlem_opts* opts,
                              void* stream);
/* Picks the frame tile by timing one iteration per candidate on a copy of
 * d_x (left unchanged): *best_tile, and h_ms[5] (when non-null) the times
 * for tiles 4, 8, 16, 32, 64 (n_frames a multiple of 4). */
raptr_status raptr_mlem_batch_autotune(raptr_ctx* ctx, int64_t m, int64_t n, int32_t n_frames, int32_t value_type,
                                       const int64_t* d_row_ptr, const int32_t* d_col, const void* d_val,
                                       const float* d_rscale, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                                       const void* d_tval, const int32_t* d_row_rank, const float* d_y,
                                       const float* d_s, const float* d_x, int32_t* best_tile, float* h_ms,
                                       void* stream);

/* ---- MLEM with rows rebuilt in every iteration ------------------------------
 * Replaces the reference's chunked reconstruction (src/tests/reco.cu:226-275:
 * per iteration and per chunk of LIMM measured rows, getSystemMatrix ->
 * cooSort -> coo2csr -> forward CSRmv -> divides -> transposed CSRmv; chunk
 * sizes src/wrappers.hpp:429-464), which bounds memory by rebuilding the
 * matrix chunk by chunk, for problems whose system matrix does not fit the
 * device.  The rows of the listed channels are built in chunks; after the
 * first iteration the leading rows that fit resident_bytes (CSR at 8 bytes
 * per entry plus 8 per row) stay resident, and the other rows are rebuilt,
 * forward-projected and back-projected (scattered) in every iteration
 * straight from the build's staging, never stored.  d_y: counts of the
 * listed channels (rows with y == 0 are not projected).  d_s: the
 * normalised sensitivity, or null to compute it in the first iteration
 * (FP64 column sums of every listed row, normalised to sum 1); d_s_out
 * (optional, num_voxels floats) receives the one used.  d_x (num_voxels)
 * is updated in place.  Besides resident_bytes the call uses about 1 GiB of
 * row staging and a few image-sized vectors; resident_bytes = 0 rebuilds
 * every row in every iteration, as the reference does.  Synchronises. */
typedef struct raptr_stream_stats {
  int64_t resident_rows;    /* leading rows kept after the first iteration  */
  int64_t resident_entries; /* their entries                                 */
  int64_t streamed_rows;    /* rows rebuilt in every iteration               */
  int32_t level;            /* row table level the rows were built at        */
  double first_iter_ms;     /* first iteration: every row built              */
  double iter_ms;           /* mean of the later iterations                  */
} raptr_stream_stats;
raptr_status raptr_mlem_stream(raptr_ctx* ctx, const int32_t* d_cnl, int64_t n_list, int32_t nrays, uint32_t seed,
                               const float* d_y, const float* d_s, float* d_s_out, float* d_x, int32_t n_iter,
                               int64_t resident_bytes, raptr_stream_stats* stats, void* stream);

/* MLEM iterations that allocate no device memory.  No counterpart in the
 * reference (which allocates its buffers itself).  For callers that cannot
 * allocate where they reconstruct -- e.g. a server that reserves its whole
 * HBM budget up front, or a pipeline that cannot take the synchronisation a
 * cudaMalloc/cudaFree brings.  Same iteration as raptr_mlem without a
 * transpose (one pass over the rows, back projection scattered with
 * atomics); the caller passes the matrix, y, s and x (updated in place).
 * The workspace is a fixed device array inside the library, sized for at
 * most 1,048,576 voxels (4 MiB, held on every GPU that loads the library
 * until exit); larger n is rejected with RAPTR_ERR_INVALID, and so are null
 * d_col / d_val when m > 0.  Runs on the current device; the first call on
 * a device looks up the array's device address, so make that first call
 * before any stream capture.  That address is kept for the life of the
 * process: do not use the library across a cudaDeviceReset.  All calls on
 * a device share the array: each call clears what must start at zero, and
 * calls that overlap on the GPU race on it. */
raptr_status raptr_mlem_noalloc(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                                const float* d_val, const float* d_y, const float* d_s, float* d_x, int32_t n_iter,
                                void* stream);

/* ---- serving ----------------------------------------------------------------
 * No counterpart in the reference (one reconstruction per process run).
 * A server runs MLEM reconstructions of mixed geometry on one GPU as they
 * are submitted: a worker thread keeps one system matrix per (geometry,
 * rays, seed) resident -- FP16 form with its transpose, built on the first
 * request, evicted least recently used when the HBM budget needs room --
 * and iterates all admitted requests of a geometry together (batched
 * frames, one CUDA stream per geometry so that geometries overlap on the
 * device).  Requests join and leave between iterations; each keeps its own
 * iteration count.  A request waits in the queue while its matrix and
 * state do not fit the budget (and fails with RAPTR_ERR_NOMEM when they
 * never can).  Each result equals the batched FP16 iteration of that
 * request alone, up to summation order. */
typedef struct raptr_server raptr_server;
typedef struct raptr_server_opts {
  int64_t hbm_budget_bytes; /* resident matrices + request state; leave room for
                               a build's transient memory (~24 bytes/entry)   */
  int32_t max_frames;       /* requests per geometry batch, 1..64              */
  int32_t keep_fp32;        /* keep the FP32 values of cached matrices         */
} raptr_server_opts;
typedef struct raptr_request_stats {
  double queue_ms;   /* submit -> admitted                                    */
  double run_ms;     /* admitted -> result on the host                        */
  double total_ms;   /* submit -> result on the host                          */
  int32_t iterations;
  int32_t frames_max; /* largest batch the request ran in                     */
  int32_t cold_build; /* 1 when its admission built the matrix                */
} raptr_request_stats;
typedef struct raptr_server_stats {
  int64_t submitted, completed, iterations, batch_steps, builds, evictions;
  int64_t resident_matrices, resident_bytes, queued, running;
} raptr_server_stats;
raptr_status raptr_server_create(int32_t device, const raptr_server_opts* opts, raptr_server** out);
/* Stops the worker (running and queued requests fail) and frees the device
 * memory. */
raptr_status raptr_server_destroy(raptr_server* s);
/* Queues a reconstruction: h_y holds the counts of all channels of the
 * geometry (channel id order, copied), n_iter MLEM iterations from a
 * uniform image. */
raptr_status raptr_server_submit(raptr_server* s, const raptr_geom* geom, int32_t nrays, uint32_t seed,
                                 const float* h_y, int32_t n_iter, int64_t* request_id);
/* Waits (timeout_ms < 0: without limit) for a request, copies its image
 * (voxels of the geometry) to h_x when non-null and forgets the request.
 * RAPTR_ERR_TIMEOUT leaves it pending. */
raptr_status raptr_server_wait(raptr_server* s, int64_t request_id, float* h_x, int32_t timeout_ms,
                               raptr_request_stats* stats);
raptr_status raptr_server_get_stats(raptr_server* s, raptr_server_stats* out);

/* ---- end-to-end ------------------------------------------------------------ */

typedef struct raptr_reco_stats {
  double build_ms;      /* system matrix build (all channels)            */
  double sens_ms;       /* sensitivity, normalisation, start image       */
  double iter_ms;       /* all MLEM iterations                           */
  double total_ms;      /* device time from the first copy to the image  */
  int64_t nnz;          /* entries of the matrix (resident ones if streamed) */
  int64_t h2d_bytes;    /* bytes copied host -> device                   */
  int64_t d2h_bytes;    /* bytes copied device -> host                   */
  double transpose_ms;  /* transpose in back-projection order            */
  double inputs_ms;     /* allocations and copy of the counts            */
  double output_ms;     /* copy of the image to the host                 */
  double setup_ms;      /* host time creating the context and stream     */
  double release_ms;    /* host time returning the device memory         */
  double wall_ms;       /* host time of the whole call                   */
  int64_t streamed_rows;/* rows rebuilt in every iteration (0: resident) */
} raptr_reco_stats;

/* The reco executable's flow from host buffers (src/tests/reco.cu:53-352):
 * measured counts h_y over all channels of the geometry (dense, num_channels
 * floats, zero = not measured), nrays rays per channel, n_iter iterations
 * from h_x0 (num_voxels floats; null = uniform image normalised to sum 1),
 * result in h_x (num_voxels floats).  The sensitivity is computed from the
 * matrix of all channels (h_sens null) or taken from h_sens (num_voxels).
 * The matrix and its transpose are built once and kept resident for all
 * iterations; when they do not fit the device (an allocation fails), the
 * call goes on as raptr_mlem_stream with the rows that fit kept resident
 * and the others rebuilt in every iteration (stats->streamed_rows). */
raptr_status raptr_reco_host(const raptr_geom* geom, int device, const float* h_y, int32_t nrays, uint32_t seed,
                             int32_t n_iter, const float* h_sens, const float* h_x0, float* h_x,
                             raptr_reco_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* RAPTR_B200_H */
