// The C ABI of raptr_b200 (include/raptr_b200.h): contexts, the chunked
// system-matrix build, the candidate search, SpMV/MLEM entry points and the
// end-to-end reconstruction from host buffers.
//
// Host code in this file computes the per-angle sine/cosine table with the
// C library's sinf/cosf on the float expression of
// src/MeasurementSetupTrafo2CartCoord.hpp:110-111; it is compiled with
// -ffp-contract=off so the expression is evaluated as written.
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdlib>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "internal.h"

using namespace raptr;

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------

namespace {

thread_local std::string g_last_error;

raptr_status fail(raptr_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

}  // namespace

namespace raptr {

double trace_ms() {
  using clk = std::chrono::steady_clock;
  static const clk::time_point t0 = clk::now();
  return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

bool trace_on() {
  static const bool on = [] {
    const char* v = std::getenv("RAPTR_TRACE");
    return v && *v && std::strcmp(v, "0") != 0;
  }();
  return on;
}

void trace(const char* fmt, ...) {
  if (!trace_on()) return;
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "[raptr %10.1f ms] %s\n", trace_ms(), buf);
}

}  // namespace raptr

namespace {

raptr_status cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky launch error for the next call
  return fail(e == cudaErrorMemoryAllocation ? RAPTR_ERR_NOMEM : RAPTR_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define RCU(call)                                  \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

#define RCHECK(expr)                              \
  do {                                            \
    raptr_status _s = (expr);                     \
    if (_s != RAPTR_OK) return _s;                \
  } while (0)

// Makes `dev` current for the scope and restores the caller's device.
struct DeviceScope {
  int prev = -1;
  bool ok = true;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceScope() {
    int cur;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Per-angle (sin, cos) as the reference evaluates them:
// sinf(T(M_PI)*ida*da/T(180.0)) with T = float, left to right.
void sincos_table(const raptr_geom& g, std::vector<float2>& out) {
  out.resize(size_t(g.na));
  for (int a = 0; a < g.na; a++) {
    float arg = float(M_PI) * float(a);
    arg = arg * g.da;
    arg = arg / 180.0f;
    out[size_t(a)] = make_float2(sinf(arg), cosf(arg));
  }
}

raptr_status validate_geom(const raptr_geom* g) {
  if (!g) return fail(RAPTR_ERR_INVALID, "geometry is null");
  for (int d = 0; d < 3; d++) {
    if (g->grid_n[d] <= 0) return fail(RAPTR_ERR_INVALID, "grid_n must be positive");
    if (!(g->grid_d[d] > 0.f) || !std::isfinite(g->grid_d[d])) return fail(RAPTR_ERR_INVALID, "grid_d must be positive");
    if (!std::isfinite(g->grid_o[d])) return fail(RAPTR_ERR_INVALID, "grid_o must be finite");
  }
  if (g->grid_n[1] > 1024) return fail(RAPTR_ERR_UNSUPPORTED, "grid_n[1] above 1024 is not supported");
  double nvox = double(g->grid_n[0]) * g->grid_n[1] * g->grid_n[2];
  if (nvox >= 2147483647.0) return fail(RAPTR_ERR_UNSUPPORTED, "more than 2^31-1 voxels");
  if (g->na <= 0 || g->n0z <= 0 || g->n0y <= 0 || g->n1z <= 0 || g->n1y <= 0)
    return fail(RAPTR_ERR_INVALID, "detector counts must be positive");
  double ncnl = double(g->na) * g->n0z * g->n0y * g->n1z * g->n1y;
  if (ncnl >= 2147483647.0) return fail(RAPTR_ERR_UNSUPPORTED, "more than 2^31-1 channels");
  if (!(g->segx > 0.f) || !(g->segy > 0.f) || !(g->segz > 0.f)) return fail(RAPTR_ERR_INVALID, "segment edges must be positive");
  if (!std::isfinite(g->pos0x) || !std::isfinite(g->pos1x) || !std::isfinite(g->da))
    return fail(RAPTR_ERR_INVALID, "setup positions and angle step must be finite");
  return RAPTR_OK;
}

}  // namespace

namespace raptr {
raptr_status set_error(raptr_status st, const std::string& msg) { return fail(st, msg); }
}  // namespace raptr

// ---------------------------------------------------------------------------
// Context and matrix objects
// ---------------------------------------------------------------------------

namespace raptr {
// The batched back pass in row-block groups (BatchArgs.seg): blocks of the
// transpose's row order, and the ratio bytes of one frame tile above which
// the grouping is used.
constexpr int kBatchRowBlocks = 16;
constexpr double kBatchBlockingBytes = 96.0 * (1 << 20);
}  // namespace raptr

struct raptr_ctx {
  raptr_geom geom;
  DGeom dg;
  int device = 0;
  float2* d_sincos = nullptr;
  // Growable device scratch, carved per call.
  unsigned char* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  // Small fixed device scratch.
  int64_t* d_i64 = nullptr;   // 64 entries
  int32_t* d_flags = nullptr; // 16 entries
  // Page-locked host words that asynchronous reads of flags and totals land
  // in (allocated on first use).
  int64_t* h_pin = nullptr;   // 16 entries
  double* d_f64 = nullptr;    // 64 entries
  // Voxels in compact (y, z) tubes along x: the column order of the
  // batched back pass, built on first use.
  int32_t* d_col_order = nullptr;
  // Row-block offsets of the columns of a transpose (see BatchArgs.seg),
  // computed for every batched call (a transpose's arrays can be freed and
  // their memory reused by another, so nothing is cached by address).
  int32_t* d_bseg = nullptr;
  int64_t bseg_n = -1;

  cudaError_t block_seg(const int64_t* cp, const int32_t* trow, int64_t m, int64_t n, cudaStream_t s,
                        const int32_t** out) {
    if (bseg_n < n) {
      dev_free(d_bseg);
      d_bseg = nullptr;
      bseg_n = -1;
      cudaError_t e = dev_malloc(&d_bseg, size_t(n) * (kBatchRowBlocks + 1) * sizeof(int32_t));
      if (e != cudaSuccess) return e;
      bseg_n = n;
    }
    cudaError_t e = launch_block_seg(n, m, kBatchRowBlocks, cp, trow, d_bseg, s);
    if (e != cudaSuccess) return e;
    *out = d_bseg;
    return cudaSuccess;
  }

  cudaError_t col_order(const int32_t** out) {
    if (!d_col_order) {
      const int nx = dg.n[0], ny = dg.n[1], nz = dg.n[2];
      // about one wave of warps (148 SMs x 64) per tube
      int tb = int(std::lround(std::sqrt(9472.0 / std::max(nx, 1))));
      tb = std::max(1, std::min(tb, std::max(ny, nz)));
      std::vector<int32_t> h;
      h.reserve(size_t(nx) * ny * nz);
      for (int ty = 0; ty < ny; ty += tb)
        for (int tz = 0; tz < nz; tz += tb)
          for (int x = 0; x < nx; x++)
            for (int y = ty; y < std::min(ny, ty + tb); y++)
              for (int z = tz; z < std::min(nz, tz + tb); z++) h.push_back(int32_t((int64_t(x) * ny + y) * nz + z));
      cudaError_t e = dev_malloc(&d_col_order, h.size() * sizeof(int32_t));
      if (e == cudaSuccess) e = cudaMemcpy(d_col_order, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        dev_free(d_col_order);
        d_col_order = nullptr;
        return e;
      }
    }
    *out = d_col_order;
    return cudaSuccess;
  }

  raptr_status ensure_scratch(size_t bytes) {
    if (bytes <= scratch_bytes) return RAPTR_OK;
    if (d_scratch) dev_free(d_scratch);
    d_scratch = nullptr;
    scratch_bytes = 0;
    size_t want = std::max(bytes, size_t(64) << 20);
    RCU(dev_malloc(&d_scratch, want));
    scratch_bytes = want;
    return RAPTR_OK;
  }
};

struct raptr_matrix {
  int device = 0;
  int64_t m = 0, n = 0, nnz = 0, cap = 0;
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  float* val = nullptr;
  // transpose (CSC), built on request
  int64_t* cp = nullptr;
  int32_t* trow = nullptr;
  float* tval = nullptr;
  // channel of each row (matrices built by the library) and the geometry
  // they belong to: the transpose is then built in the back-projection order
  // of the channels, trow holding positions in that order
  int32_t* cnl = nullptr;
  DGeom geom{};
  int32_t* rank = nullptr;   // row -> position
  int32_t* order = nullptr;  // position -> row
  // FP16 form, built on request: a_ij ~= rscale_i * h_ij
  float* rscale = nullptr;
  float* pscale = nullptr;   // rscale by position of the transpose
  uint16_t* hval = nullptr;  // CSR order
  uint16_t* htval = nullptr; // transpose order
  // the FP16 form delta-coded (raptr_pack_half of the CSR and of the
  // transpose), built on request
  int64_t* pseg = nullptr;
  int32_t* panchor = nullptr;
  uint32_t* pword = nullptr;
  int64_t* tseg = nullptr;
  int32_t* tanchor = nullptr;
  uint32_t* tword = nullptr;
  int64_t pwords = 0, twords = 0;
};

namespace {

// Bump allocator over the context scratch.
struct Carve {
  unsigned char* base;
  size_t off = 0;
  explicit Carve(unsigned char* b) : base(b) {}
  template <typename T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += n * sizeof(T);
    return p;
  }
  static size_t need(std::initializer_list<size_t> bytes) {
    size_t t = 0;
    for (size_t b : bytes) t += ((b + 255) & ~size_t(255)) + 256;
    return t;
  }
};

constexpr size_t kStagingBudget = size_t(1) << 30;  // bytes of row staging per chunk

// Output of a build: caller buffers (fixed capacity) or a library matrix
// that grows.
struct BuildOut {
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  float* val = nullptr;
  int64_t cap = 0;
  raptr_matrix* grow = nullptr;  // non-null: grow this matrix on demand
  int64_t n_list = 0;
};

raptr_status ensure_capacity(BuildOut& o, int64_t need, int64_t rows_done, cudaStream_t s) {
  if (need <= o.cap || !o.grow) return RAPTR_OK;
  double per_row = rows_done > 0 ? double(need) / double(rows_done) : 0.0;
  // rows of a list differ in length (by projection angle, say): an estimate
  // from its first quarter gets more headroom, so that the output is not
  // regrown (a copy of everything so far) near the end
  const double headroom = rows_done * 4 < o.n_list ? 1.3 : 1.05;
  int64_t projected = int64_t(per_row * double(o.n_list) * headroom) + 1024;
  int64_t ncap = std::max(need + (need >> 3), projected);
  const double t0 = trace_on() ? trace_ms() : 0.0;
  int32_t* ncol = nullptr;
  float* nval = nullptr;
  RCU(dev_malloc(&ncol, size_t(ncap) * sizeof(int32_t)));
  cudaError_t e = dev_malloc(&nval, size_t(ncap) * sizeof(float));
  if (e != cudaSuccess) {
    dev_free(ncol);
    return cuda_fail(e, "cudaMalloc(matrix values)");
  }
  int64_t keep = std::min(o.cap, need);
  if (o.col && keep > 0) {
    RCU(cudaMemcpyAsync(ncol, o.col, size_t(keep) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    RCU(cudaMemcpyAsync(nval, o.val, size_t(keep) * sizeof(float), cudaMemcpyDeviceToDevice, s));
  }
  RCU(cudaStreamSynchronize(s));
  if (o.col) dev_free(o.col);
  if (o.val) dev_free(o.val);
  o.col = ncol;
  o.val = nval;
  o.cap = ncap;
  o.grow->col = ncol;
  o.grow->val = nval;
  o.grow->cap = ncap;
  if (trace_on())
    trace("build output grown to %lld entries (kept %lld): %.2f ms", (long long)ncap, (long long)keep, trace_ms() - t0);
  return RAPTR_OK;
}

struct Builder {
  raptr_ctx* ctx;
  const int32_t* d_cnl;
  int64_t n_list;
  int nrays;
  uint32_t seed;
  const float* d_rays;
  bool keep_zeros;
  cudaStream_t s;
  BuildOut& out;
  int64_t total = 0;       // entries placed so far (host mirror of d_base)
  int64_t rows_done = 0;

  // Builds rows [row0, row0+nrows) at `level` as a pipeline of chunks: the
  // row kernel of chunk i+1 runs while chunk i is placed (scan, capacity,
  // gather) on a placement stream, from a second staging buffer, so the
  // device does not idle while the host reads a chunk's flags and entry
  // count.  Even chunks run on the caller's stream and odd ones on a second
  // row stream, so that a chunk's CTAs fill the SMs as the previous chunk's
  // last ones retire (one stream would leave its last wave draining alone);
  // a chunk waits for the placement of the chunk two before it, which used
  // its buffer.  A chunk whose table overflowed drains the pipeline, is
  // rebuilt at the next level by rows(), and the pipeline restarts after it.
  raptr_status rows_pipelined(int level, int64_t row0, int64_t nrows) {
    const int H = sm_level_capacity(level);
    int64_t per = std::max<int64_t>(1, int64_t(kStagingBudget / (size_t(H) * 8)));
    per = std::min<int64_t>(per, 65536);
    if (!ctx->h_pin) RCU(cudaMallocHost(&ctx->h_pin, 16 * sizeof(int64_t)));
    // words 0-1: the dense kernel's flags, 2-3: the table kernel's (per buffer)
    volatile int32_t* h_flags = reinterpret_cast<volatile int32_t*>(ctx->h_pin);
    volatile int64_t* h_total = ctx->h_pin + 2;
    cudaStream_t P = nullptr, S2 = nullptr;
    cudaEvent_t ev_k[2] = {nullptr, nullptr}, ev_g[2] = {nullptr, nullptr}, ev_j = nullptr;
    auto release = [&]() {
      for (auto e : ev_k) if (e) cudaEventDestroy(e);
      for (auto e : ev_g) if (e) cudaEventDestroy(e);
      if (ev_j) cudaEventDestroy(ev_j);
      if (P) cudaStreamDestroy(P);
      if (S2) cudaStreamDestroy(S2);
    };
    struct Guard {
      std::function<void()> f;
      ~Guard() { f(); }
    } guard{release};
    RCU(cudaStreamCreateWithFlags(&P, cudaStreamNonBlocking));
    RCU(cudaStreamCreateWithFlags(&S2, cudaStreamNonBlocking));
    for (int b = 0; b < 2; b++) {
      RCU(cudaEventCreateWithFlags(&ev_k[b], cudaEventDisableTiming));
      RCU(cudaEventCreateWithFlags(&ev_g[b], cudaEventDisableTiming));
    }
    RCU(cudaEventCreateWithFlags(&ev_j, cudaEventDisableTiming));
    auto drain = [&]() -> cudaError_t {
      cudaError_t e = cudaStreamSynchronize(s);
      cudaError_t e2 = cudaStreamSynchronize(S2);
      cudaError_t e3 = cudaStreamSynchronize(P);
      return e != cudaSuccess ? e : (e2 != cudaSuccess ? e2 : e3);
    };
    const int64_t end = row0 + nrows;
    int64_t r0 = row0;
    while (r0 < end) {
      const int64_t n = (end - r0 + per - 1) / per;  // chunks from r0 on
      size_t need = Carve::need({size_t(per) * H * sizeof(int32_t), size_t(per) * H * sizeof(float),
                                 size_t(per) * sizeof(int32_t), size_t(per) * H * sizeof(int32_t),
                                 size_t(per) * H * sizeof(float), size_t(per) * sizeof(int32_t)});
      RCHECK(ctx->ensure_scratch(need));
      Carve cv(ctx->d_scratch);
      int32_t* st_col[2];
      float* st_val[2];
      int32_t* row_nnz[2];
      for (int b = 0; b < 2; b++) {
        st_col[b] = cv.take<int32_t>(size_t(per) * H);
        st_val[b] = cv.take<float>(size_t(per) * H);
        row_nnz[b] = cv.take<int32_t>(size_t(per));
      }
      // placement and the second row stream start after the caller's
      // earlier work
      RCU(cudaEventRecord(ev_j, s));
      RCU(cudaStreamWaitEvent(P, ev_j, 0));
      RCU(cudaStreamWaitEvent(S2, ev_j, 0));
      auto launch = [&](int64_t i) -> cudaError_t {
        const int b = int(i & 1);
        cudaStream_t q = b ? S2 : s;  // buffer b's chunks, in order, on one stream
        const int64_t r = r0 + i * per, k = std::min(per, end - r);
        cudaError_t e = cudaSuccess;
        if (i >= 2) e = cudaStreamWaitEvent(q, ev_g[b], 0);  // chunk i-2 has left this buffer
        if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_flags + b, 0, sizeof(int32_t), q);
        if (e == cudaSuccess)
          e = launch_sm_rows(level, ctx->dg, ctx->d_sincos, d_cnl, r, k, nrays, seed, d_rays, st_col[b], st_val[b],
                             row_nnz[b], ctx->d_flags + b, q, ctx->d_flags + 4, d_rays ? kRowsAll : kRowsDense);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(const_cast<int32_t*>(h_flags) + b, ctx->d_flags + b, sizeof(int32_t),
                              cudaMemcpyDeviceToHost, q);
        if (e == cudaSuccess) e = cudaEventRecord(ev_k[b], q);
        return e;
      };
      cudaError_t e = launch(0);
      if (e != cudaSuccess) {
        drain();
        return cuda_fail(e, "system-matrix rows");
      }
      int64_t next_r0 = end;
      for (int64_t i = 0; i < n; i++) {
        const int b = int(i & 1);
        const int64_t r = r0 + i * per, k = std::min(per, end - r);
        const double t0 = trace_on() ? trace_ms() : 0.0;
        if (i + 1 < n) e = launch(i + 1);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev_k[b]);
        if (e != cudaSuccess) {
          drain();
          return cuda_fail(e, "system-matrix rows");
        }
        const int32_t flags = h_flags[b];
        if (flags & 6) {
          RCU(drain());
          if (flags & 4) return fail(RAPTR_ERR_INVALID, "a channel id is outside [0, number of channels)");
          return fail(RAPTR_ERR_OVERFLOW, "ray walk did not terminate (internal error)");
        }
        if (flags & 1) {
          RCU(drain());
          if (level + 1 >= sm_num_levels())
            return fail(RAPTR_ERR_OVERFLOW, "a row has more distinct voxels than the largest per-row table holds");
          RCHECK(rows(level + 1, r, k));
          next_r0 = r + k;
          break;
        }
        e = cudaStreamWaitEvent(P, ev_k[b], 0);
        if (!d_rays) {
          // The rows the dense kernel left to the hash table, on the
          // placement stream: a row or two per chunk, which would otherwise
          // hold up the next chunk's dense rows on the caller's stream.
          if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_flags + 2 + b, 0, sizeof(int32_t), P);
          if (e == cudaSuccess)
            e = launch_sm_rows(level, ctx->dg, ctx->d_sincos, d_cnl, r, k, nrays, seed, nullptr, st_col[b],
                               st_val[b], row_nnz[b], ctx->d_flags + 2 + b, P, nullptr, kRowsTable);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(const_cast<int32_t*>(h_flags) + 2 + b, ctx->d_flags + 2 + b, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, P);
          if (e == cudaSuccess) e = cudaStreamSynchronize(P);
          if (e != cudaSuccess) {
            drain();
            return cuda_fail(e, "system-matrix rows (table)");
          }
          const int32_t tflags = h_flags[2 + b];
          if (tflags & 6) {
            RCU(drain());
            if (tflags & 4) return fail(RAPTR_ERR_INVALID, "a channel id is outside [0, number of channels)");
            return fail(RAPTR_ERR_OVERFLOW, "ray walk did not terminate (internal error)");
          }
          if (tflags & 1) {
            RCU(drain());
            if (level + 1 >= sm_num_levels())
              return fail(RAPTR_ERR_OVERFLOW, "a row has more distinct voxels than the largest per-row table holds");
            RCHECK(rows(level + 1, r, k));
            next_r0 = r + k;
            break;
          }
        }
        if (e == cudaSuccess) e = launch_rows_scan(row_nnz[b], k, out.rp + r, ctx->d_i64, P);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(const_cast<int64_t*>(h_total), ctx->d_i64, sizeof(int64_t), cudaMemcpyDeviceToHost, P);
        if (e == cudaSuccess) e = cudaStreamSynchronize(P);
        if (e != cudaSuccess) {
          drain();
          return cuda_fail(e, "system-matrix placement");
        }
        const int64_t new_total = *h_total;
        rows_done += k;
        if (trace_on())
          trace("build rows %lld+%lld level %d: rows and placement %.2f ms, %lld entries", (long long)r,
                (long long)k, level, trace_ms() - t0, (long long)new_total);
        raptr_status st = ensure_capacity(out, new_total, rows_done, P);
        if (st != RAPTR_OK) {
          drain();
          return st;
        }
        e = launch_rows_gather(st_col[b], st_val[b], H, out.rp + r, k, out.cap, out.col, out.val, P);
        if (e == cudaSuccess) e = cudaEventRecord(ev_g[b], P);
        if (e != cudaSuccess) {
          drain();
          return cuda_fail(e, "system-matrix placement");
        }
        total = new_total;
      }
      // the caller's stream continues after the placement
      RCU(cudaEventRecord(ev_j, P));
      RCU(cudaStreamWaitEvent(s, ev_j, 0));
      if (next_r0 < end) RCU(drain());  // buffers are re-carved after rows() used the scratch
      r0 = next_r0;
    }
    return RAPTR_OK;
  }

  // Builds rows [row0, row0+nrows) at `level`, retrying at higher levels on
  // table overflow, and places them.
  raptr_status rows(int level, int64_t row0, int64_t nrows) {
    const int H = sm_level_capacity(level);
    int64_t per = std::max<int64_t>(1, int64_t(kStagingBudget / (size_t(H) * 8)));
    per = std::min<int64_t>(per, 65536);
    for (int64_t r = row0; r < row0 + nrows; r += per) {
      const int64_t k = std::min(per, row0 + nrows - r);
      size_t need = Carve::need({size_t(k) * H * sizeof(int32_t), size_t(k) * H * sizeof(float),
                                 size_t(k) * sizeof(int32_t), size_t(k) * sizeof(int64_t),
                                 size_t(scan_temp_elems(k)) * sizeof(int64_t)});
      RCHECK(ctx->ensure_scratch(need));
      Carve cv(ctx->d_scratch);
      int32_t* st_col = cv.take<int32_t>(size_t(k) * H);
      float* st_val = cv.take<float>(size_t(k) * H);
      int32_t* row_nnz = cv.take<int32_t>(size_t(k));
      int64_t* cand = cv.take<int64_t>(size_t(k));
      (void)cand;
      const double t0 = trace_on() ? trace_ms() : 0.0;
      RCU(cudaMemsetAsync(ctx->d_flags, 0, sizeof(int32_t), s));
      RCU(launch_sm_rows(level, ctx->dg, ctx->d_sincos, d_cnl, r, k, nrays, seed, d_rays, st_col, st_val, row_nnz,
                         ctx->d_flags, s, ctx->d_flags + 4));
      int32_t flags = 0;
      RCU(cudaMemcpyAsync(&flags, ctx->d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      RCU(cudaStreamSynchronize(s));
      if (flags & 4) return fail(RAPTR_ERR_INVALID, "a channel id is outside [0, number of channels)");
      if (flags & 2) return fail(RAPTR_ERR_OVERFLOW, "ray walk did not terminate (internal error)");
      if (flags & 1) {
        if (level + 1 < sm_num_levels()) {
          RCHECK(rows(level + 1, r, k));
          continue;
        }
        return fail(RAPTR_ERR_OVERFLOW, "a row has more distinct voxels than the largest per-row table holds");
      }
      if (!keep_zeros) {
        RCU(launch_rows_scan(row_nnz, k, out.rp + r, ctx->d_i64, s));
      } else {
        int64_t* counts = cand;
        RCU(launch_wq_count(ctx->dg, ctx->d_sincos, d_cnl, r, k, 0, counts, ctx->d_flags, s));
        RCU(launch_rows_scan_i64(counts, k, out.rp + r, ctx->d_i64, s));
      }
      int64_t new_total = 0;
      RCU(cudaMemcpyAsync(&new_total, ctx->d_i64, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      RCU(cudaStreamSynchronize(s));
      rows_done += k;
      if (trace_on())
        trace("build rows %lld+%lld level %d: rows and placement %.2f ms, %lld entries", (long long)r, (long long)k,
              level, trace_ms() - t0, (long long)new_total);
      RCHECK(ensure_capacity(out, new_total, rows_done, s));
      if (!keep_zeros) {
        RCU(launch_rows_gather(st_col, st_val, H, out.rp + r, k, out.cap, out.col, out.val, s));
      } else if (new_total <= out.cap) {
        RCU(launch_wq_fill(ctx->dg, ctx->d_sincos, d_cnl, r, k, 0, out.rp + r, out.cap, nullptr, out.col, ctx->d_flags,
                           s));
        RCU(launch_expand_candidates(st_col, st_val, H, row_nnz, out.rp + r, k, out.col, out.val, s));
      }
      total = new_total;
    }
    return RAPTR_OK;
  }
};

raptr_status run_build(raptr_ctx* ctx, const int32_t* d_cnl, int64_t n_list, int nrays, uint32_t seed,
                       const float* d_rays, int32_t flags, BuildOut& out, int64_t* nnz_out, cudaStream_t s) {
  if (n_list < 0) return fail(RAPTR_ERR_INVALID, "n_list must be non-negative");
  if (n_list > 0 && !d_cnl) return fail(RAPTR_ERR_INVALID, "channel list is null");
  if (nrays <= 0) return fail(RAPTR_ERR_INVALID, "nrays must be positive");
  if (!out.rp) return fail(RAPTR_ERR_INVALID, "row pointer buffer is null");
  RCU(cudaMemsetAsync(ctx->d_i64, 0, sizeof(int64_t), s));
  RCU(cudaMemsetAsync(out.rp, 0, sizeof(int64_t), s));
  RCU(cudaMemsetAsync(ctx->d_flags + 4, 0, 4 * sizeof(int32_t), s));  // rows left to the table, by reason
  out.n_list = n_list;
  Builder b{ctx, d_cnl, n_list, nrays, seed, d_rays, (flags & RAPTR_SM_KEEP_ZEROS) != 0, s, out};
  if (n_list > 0) {
    const int level = sm_pick_level(ctx->dg, nrays);
    if (b.keep_zeros)
      RCHECK(b.rows(level, 0, n_list));
    else
      RCHECK(b.rows_pipelined(level, 0, n_list));
  }
  RCU(cudaStreamSynchronize(s));
  *nnz_out = b.total;
  if (trace_on()) {
    int32_t why[4] = {0, 0, 0, 0};
    RCU(cudaMemcpy(why, ctx->d_flags + 4, sizeof(why), cudaMemcpyDeviceToHost));
    trace("build: %lld rows, rows built with the hash table: %d without a slab axis, %d with windows over the "
          "slot limit, %d with a ray outside its windows, %d with a slot outside the grid",
          (long long)n_list, why[0], why[1], why[2], why[3]);
  }
  if (b.total > out.cap && !out.grow) {
    return fail(RAPTR_ERR_CAPACITY, "matrix has " + std::to_string(b.total) + " entries, buffer holds " +
                                        std::to_string(out.cap));
  }
  return RAPTR_OK;
}

}  // namespace

extern "C" {

int raptr_abi_version(void) { return RAPTR_ABI_VERSION; }

raptr_status raptr_trim_memory(int device) {
  dev_release(device < 0 ? -1 : device);
  return RAPTR_OK;
}

const char* raptr_last_error(void) { return g_last_error.c_str(); }

int64_t raptr_kernel_launches(void) { return launches_so_far(); }

raptr_status raptr_ctx_create(const raptr_geom* geom, int device, raptr_ctx** out) {
  if (!out) return fail(RAPTR_ERR_INVALID, "out is null");
  *out = nullptr;
  RCHECK(validate_geom(geom));
  DeviceScope ds(device);
  if (!ds.ok) return fail(RAPTR_ERR_CUDA, "cannot select device " + std::to_string(device));
  raptr_ctx* c = new raptr_ctx;
  c->geom = *geom;
  c->dg = to_dgeom(*geom);
  c->device = device;
  std::vector<float2> tab;
  sincos_table(*geom, tab);
  cudaError_t e = dev_malloc(&c->d_sincos, tab.size() * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemcpy(c->d_sincos, tab.data(), tab.size() * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = dev_malloc(&c->d_i64, 64 * sizeof(int64_t));
  if (e == cudaSuccess) e = dev_malloc(&c->d_flags, 16 * sizeof(int32_t));
  if (e == cudaSuccess) e = dev_malloc(&c->d_f64, 64 * sizeof(double));
  if (e != cudaSuccess) {
    raptr_ctx_destroy(c);
    return cuda_fail(e, "context allocation");
  }
  *out = c;
  return RAPTR_OK;
}

raptr_status raptr_ctx_destroy(raptr_ctx* ctx) {
  if (!ctx) return RAPTR_OK;
  DeviceScope ds(ctx->device);
  dev_free(ctx->d_sincos);
  dev_free(ctx->d_scratch);
  dev_free(ctx->d_i64);
  dev_free(ctx->d_flags);
  dev_free(ctx->d_f64);
  dev_free(ctx->d_col_order);
  dev_free(ctx->d_bseg);
  cudaFreeHost(ctx->h_pin);
  delete ctx;
  return RAPTR_OK;
}

int64_t raptr_ctx_num_channels(const raptr_ctx* ctx) {
  if (!ctx) return 0;
  const raptr_geom& g = ctx->geom;
  return int64_t(g.na) * g.n0z * g.n0y * g.n1z * g.n1y;
}

int64_t raptr_ctx_num_voxels(const raptr_ctx* ctx) {
  if (!ctx) return 0;
  return int64_t(ctx->geom.grid_n[0]) * ctx->geom.grid_n[1] * ctx->geom.grid_n[2];
}

// ---- candidate search -------------------------------------------------------

raptr_status raptr_candidate_counts(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int64_t* d_counts,
                                    void* stream) {
  if (!ctx || (n_list > 0 && (!d_cnl_ids || !d_counts))) return fail(RAPTR_ERR_INVALID, "null argument");
  DeviceScope ds(ctx->device);
  RCU(launch_wq_count(ctx->dg, ctx->d_sincos, d_cnl_ids, 0, n_list, 0, d_counts, nullptr, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_workqueue(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int64_t* list_id,
                             int64_t* vxl_id, int64_t max_out, int32_t* d_cnl_out, int32_t* d_vxl_out,
                             int64_t* n_found, void* stream) {
  if (!ctx || !list_id || !vxl_id || !n_found) return fail(RAPTR_ERR_INVALID, "null argument");
  *n_found = 0;
  if (max_out <= 0) return RAPTR_OK;
  if (!d_cnl_out || !d_vxl_out || (n_list > 0 && !d_cnl_ids)) return fail(RAPTR_ERR_INVALID, "null buffer");
  const int64_t nvox = raptr_ctx_num_voxels(ctx);
  if (*list_id < 0 || *vxl_id < 0 || *vxl_id >= nvox)
    return fail(RAPTR_ERR_INVALID, "cursor out of range");  // the reference exits here (src/getWorkqueue.hpp:108-111)
  DeviceScope ds(ctx->device);
  cudaStream_t s = as_stream(stream);
  const int64_t kBatch = 16384;
  int64_t li = *list_id, vi = *vxl_id, found = 0;
  std::vector<int64_t> h_off;
  while (li < n_list && found < max_out) {
    const int64_t B = std::min(kBatch, n_list - li);
    RCHECK(ctx->ensure_scratch(Carve::need({size_t(B) * 8, size_t(B + 1) * 8, size_t(scan_temp_elems(B)) * 8})));
    Carve cv(ctx->d_scratch);
    int64_t* counts = cv.take<int64_t>(size_t(B));
    int64_t* offs = cv.take<int64_t>(size_t(B + 1));
    int64_t* tmp = cv.take<int64_t>(size_t(scan_temp_elems(B)));
    RCU(cudaMemsetAsync(ctx->d_flags, 0, sizeof(int32_t), s));
    RCU(launch_wq_count(ctx->dg, ctx->d_sincos, d_cnl_ids, li, B, vi, counts, ctx->d_flags, s));
    RCU(launch_scan_i64(counts, B, offs, tmp, s));
    const int64_t remaining = max_out - found;
    RCU(launch_wq_fill(ctx->dg, ctx->d_sincos, d_cnl_ids, li, B, vi, offs, remaining, d_cnl_out + found,
                       d_vxl_out + found, nullptr, s));
    h_off.resize(size_t(B + 1));
    int32_t flags = 0;
    RCU(cudaMemcpyAsync(h_off.data(), offs, size_t(B + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RCU(cudaMemcpyAsync(&flags, ctx->d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCU(cudaStreamSynchronize(s));
    if (flags & 4) return fail(RAPTR_ERR_INVALID, "a channel id is outside [0, number of channels)");
    const int64_t total = h_off[size_t(B)];
    if (total >= remaining) {
      // The last entry returned is entry `remaining-1` of this batch.
      int64_t j = int64_t(std::upper_bound(h_off.begin(), h_off.end(), remaining - 1) - h_off.begin()) - 1;
      int32_t last_v = 0;
      RCU(cudaMemcpy(&last_v, d_vxl_out + found + remaining - 1, sizeof(int32_t), cudaMemcpyDeviceToHost));
      found = max_out;
      if (last_v < nvox - 1) {
        *list_id = li + j;
        *vxl_id = last_v + 1;
      } else {
        *list_id = li + j + 1;
        *vxl_id = 0;
      }
      *n_found = found;
      return RAPTR_OK;
    }
    found += total;
    li += B;
    vi = 0;
  }
  *list_id = n_list;
  *vxl_id = 0;
  *n_found = found;
  return RAPTR_OK;
}

// ---- rays -----------------------------------------------------------------------

raptr_status raptr_rays(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int32_t nrays, uint32_t seed,
                        float* d_rays, void* stream) {
  if (!ctx || nrays <= 0 || (n_list > 0 && (!d_cnl_ids || !d_rays))) return fail(RAPTR_ERR_INVALID, "bad argument");
  DeviceScope ds(ctx->device);
  RCU(launch_rays(ctx->dg, ctx->d_sincos, d_cnl_ids, n_list, nrays, seed, d_rays, as_stream(stream)));
  return RAPTR_OK;
}

// ---- system matrix ----------------------------------------------------------------

raptr_status raptr_sm_build(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int32_t nrays, uint32_t seed,
                            const float* d_rays, int32_t flags, int64_t capacity, int64_t* d_row_ptr, int32_t* d_col,
                            float* d_val, int64_t* nnz_out, void* stream) {
  if (!ctx || !nnz_out) return fail(RAPTR_ERR_INVALID, "null argument");
  if (capacity < 0 || (capacity > 0 && (!d_col || !d_val))) return fail(RAPTR_ERR_INVALID, "bad output buffers");
  DeviceScope ds(ctx->device);
  BuildOut out;
  out.rp = d_row_ptr;
  out.col = d_col;
  out.val = d_val;
  out.cap = capacity;
  return run_build(ctx, d_cnl_ids, n_list, nrays, seed, d_rays, flags, out, nnz_out, as_stream(stream));
}

raptr_status raptr_sm_build_alloc(raptr_ctx* ctx, const int32_t* d_cnl_ids, int64_t n_list, int32_t nrays,
                                  uint32_t seed, const float* d_rays, int32_t flags, raptr_matrix** out_m,
                                  void* stream) {
  if (!ctx || !out_m) return fail(RAPTR_ERR_INVALID, "null argument");
  *out_m = nullptr;
  DeviceScope ds(ctx->device);
  raptr_matrix* A = new raptr_matrix;
  A->device = ctx->device;
  A->m = n_list;
  A->n = raptr_ctx_num_voxels(ctx);
  cudaError_t e = dev_malloc(&A->rp, size_t(n_list + 1) * sizeof(int64_t));
  if (e != cudaSuccess) {
    delete A;
    return cuda_fail(e, "cudaMalloc(row pointers)");
  }
  BuildOut out;
  out.rp = A->rp;
  out.grow = A;
  int64_t nnz = 0;
  raptr_status st = run_build(ctx, d_cnl_ids, n_list, nrays, seed, d_rays, flags, out, &nnz, as_stream(stream));
  if (st != RAPTR_OK) {
    raptr_matrix_destroy(A);
    return st;
  }
  A->nnz = nnz;
  A->geom = ctx->dg;
  if (n_list > 0) {
    cudaError_t ec = dev_malloc(&A->cnl, size_t(n_list) * sizeof(int32_t));
    if (ec == cudaSuccess)
      ec = cudaMemcpyAsync(A->cnl, d_cnl_ids, size_t(n_list) * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                           as_stream(stream));
    if (ec != cudaSuccess) {
      raptr_matrix_destroy(A);
      return cuda_fail(ec, "cudaMalloc(channel list)");
    }
  }
  *out_m = A;
  return RAPTR_OK;
}

raptr_status raptr_matrix_info(const raptr_matrix* A, int64_t* m, int64_t* n, int64_t* nnz, int64_t** d_row_ptr,
                               int32_t** d_col, float** d_val) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (m) *m = A->m;
  if (n) *n = A->n;
  if (nnz) *nnz = A->nnz;
  if (d_row_ptr) *d_row_ptr = A->rp;
  if (d_col) *d_col = A->col;
  if (d_val) *d_val = A->val;
  return RAPTR_OK;
}

raptr_status raptr_matrix_destroy(raptr_matrix* A) {
  if (!A) return RAPTR_OK;
  DeviceScope ds(A->device);
  const double t0 = trace_on() ? trace_ms() : 0.0;
  dev_free(A->rp);
  dev_free(A->col);
  dev_free(A->val);
  dev_free(A->cp);
  dev_free(A->trow);
  dev_free(A->tval);
  dev_free(A->cnl);
  dev_free(A->rank);
  dev_free(A->order);
  dev_free(A->rscale);
  dev_free(A->pscale);
  dev_free(A->hval);
  dev_free(A->htval);
  dev_free(A->pseg);
  dev_free(A->panchor);
  dev_free(A->pword);
  dev_free(A->tseg);
  dev_free(A->tanchor);
  dev_free(A->tword);
  if (trace_on()) trace("matrix released: %.2f ms", trace_ms() - t0);
  delete A;
  return RAPTR_OK;
}

namespace {

raptr_status transpose_impl(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                            const int32_t* d_order, int64_t* d_col_ptr, int32_t* d_row_idx, float* d_tval,
                            cudaStream_t s) {
  if (m < 0 || n <= 0 || m > INT32_MAX || n > INT32_MAX || !d_row_ptr || !d_col_ptr)
    return fail(RAPTR_ERR_INVALID, "bad argument");
  int64_t nnz = 0;
  RCU(cudaMemcpyAsync(&nnz, d_row_ptr + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  RCU(cudaStreamSynchronize(s));
  if (nnz > 0 && (!d_col || !d_val || !d_row_idx || !d_tval)) return fail(RAPTR_ERR_INVALID, "null buffer");
  // radix sort by column when it applies and its staging (12 bytes per
  // entry) fits; else the blocked transpose (4 bytes per column and block)
  RadixPlan plan;
  if (nnz > 0 && transpose_radix_plan(m, n, nnz, &plan)) {
    const int64_t nh = radix_hist_elems(plan);
    int64_t *hist = nullptr, *off = nullptr, *tmp = nullptr, *cc64 = nullptr;
    int32_t *cc = nullptr, *bad = nullptr, *st_key = nullptr, *st_k = nullptr;
    float* st_v = nullptr;
    // plain allocations: the stream-ordered pool grows slowly at these
    // sizes (the staging is tens of GB at full size)
    const double t0 = trace_on() ? trace_ms() : 0.0;
    cudaError_t e = dev_malloc(&hist, size_t(nh) * sizeof(int64_t));
    if (e == cudaSuccess) e = dev_malloc(&off, size_t(nh + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = dev_malloc(&tmp, size_t(scan_temp_elems(std::max(nh, n))) * sizeof(int64_t));
    if (e == cudaSuccess) e = dev_malloc(&cc, size_t(n) * sizeof(int32_t));
    if (e == cudaSuccess) e = dev_malloc(&cc64, size_t(n) * sizeof(int64_t));
    if (e == cudaSuccess) e = dev_malloc(&bad, sizeof(int32_t));
    bool staged = true;
    if (e == cudaSuccess && plan.passes > 1) {
      if (dev_malloc(&st_key, size_t(nnz) * sizeof(int32_t)) != cudaSuccess ||
          dev_malloc(&st_k, size_t(nnz) * sizeof(int32_t)) != cudaSuccess ||
          dev_malloc(&st_v, size_t(nnz) * sizeof(float)) != cudaSuccess) {
        (void)cudaGetLastError();  // does not fit: the blocked transpose needs less
        staged = false;
      }
    }
    int32_t h_bad = 0;
    const double t1 = trace_on() ? trace_ms() : 0.0;
    if (e == cudaSuccess && staged) {
      e = cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
      if (e == cudaSuccess)
        e = launch_transpose_radix(plan, m, n, nnz, d_row_ptr, d_col, d_val, d_order, hist, off, tmp, cc, cc64,
                                   st_key, st_k, st_v, bad, d_col_ptr, d_row_idx, d_tval, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaStreamSynchronize(s);
    const double t2 = trace_on() ? trace_ms() : 0.0;
    dev_free(hist);
    dev_free(off);
    dev_free(tmp);
    dev_free(cc);
    dev_free(cc64);
    dev_free(bad);
    dev_free(st_key);
    dev_free(st_k);
    dev_free(st_v);
    if (trace_on())
      trace("transpose radix (%d passes, %s): allocations %.2f ms, sort %.2f ms, release %.2f ms, total %.2f ms",
            plan.passes, staged ? "staged" : "staging does not fit", t1 - t0, t2 - t1, trace_ms() - t2,
            trace_ms() - t0);
    if (e != cudaSuccess) return cuda_fail(e, "raptr_csr_transpose");
    if (h_bad) return fail(RAPTR_ERR_INVALID, "column index or row order entry out of range");
    if (staged) return RAPTR_OK;
  }
  const int B = transpose_blocks(m, n);
  int32_t *cnt = nullptr, *bad = nullptr;
  int64_t *colcount = nullptr, *tmp = nullptr;
  cudaError_t e = cudaMallocAsync(&cnt, size_t(B) * size_t(n) * sizeof(int32_t), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&colcount, size_t(n) * sizeof(int64_t), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&tmp, size_t(scan_temp_elems(n)) * sizeof(int64_t), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&bad, sizeof(int32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
  if (e == cudaSuccess)
    e = launch_transpose_blocked(m, n, B, d_row_ptr, d_col, d_val, d_order, d_order != nullptr, cnt, colcount, tmp,
                                 bad, d_col_ptr, d_row_idx, d_tval, s);
  int32_t h_bad = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (cnt) cudaFreeAsync(cnt, s);
  if (colcount) cudaFreeAsync(colcount, s);
  if (tmp) cudaFreeAsync(tmp, s);
  if (bad) cudaFreeAsync(bad, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "raptr_csr_transpose");
  if (h_bad) return fail(RAPTR_ERR_INVALID, "column index or row order entry out of range");
  return RAPTR_OK;
}

}  // namespace

raptr_status raptr_csr_transpose(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                                 const float* d_val, int64_t* d_col_ptr, int32_t* d_row_idx, float* d_tval,
                                 void* stream) {
  return transpose_impl(m, n, d_row_ptr, d_col, d_val, nullptr, d_col_ptr, d_row_idx, d_tval, as_stream(stream));
}

raptr_status raptr_csr_transpose_ordered(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                                         const float* d_val, const int32_t* d_order, int64_t* d_col_ptr,
                                         int32_t* d_pos_idx, float* d_tval, void* stream) {
  if (m > 0 && !d_order) return fail(RAPTR_ERR_INVALID, "order is null");
  return transpose_impl(m, n, d_row_ptr, d_col, d_val, d_order, d_col_ptr, d_pos_idx, d_tval, as_stream(stream));
}

namespace {

// Back-projection order of the rows of a library-built matrix (its
// channels): fills A->rank / A->order and sets *have.  Leaves the natural
// order (*have false) when the rows repeat a channel or the key space is
// too large to mark.
cudaError_t matrix_row_order(raptr_matrix* A, cudaStream_t s, bool* have) {
  *have = false;
  if (!A->cnl || A->m <= 0) return cudaSuccess;
  const int64_t K = channel_order_keys(A->geom);
  if (K <= 0 || K > (int64_t(1) << 28)) return cudaSuccess;
  unsigned long long* mark = nullptr;
  int64_t *prefix = nullptr, *tmp = nullptr;
  int32_t* bad = nullptr;
  const double t0 = trace_on() ? trace_ms() : 0.0;
  // plain allocations: the stream-ordered pool grows slowly at this size
  cudaError_t e = dev_malloc(&mark, size_t(K) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = dev_malloc(&prefix, size_t(K + 1) * sizeof(int64_t));
  if (e == cudaSuccess) e = dev_malloc(&tmp, size_t(scan_temp_elems(K)) * sizeof(int64_t));
  if (e == cudaSuccess) e = dev_malloc(&bad, sizeof(int32_t));
  const double t1 = trace_on() ? trace_ms() : 0.0;
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
  if (e == cudaSuccess) e = launch_channel_order_mark(A->geom, A->m, A->cnl, mark, bad, s);
  if (e == cudaSuccess) e = launch_scan_i64(reinterpret_cast<const int64_t*>(mark), K, prefix, tmp, s);
  int32_t h_bad = 1;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && !h_bad) {
    e = dev_malloc(&A->rank, size_t(A->m) * sizeof(int32_t));
    if (e == cudaSuccess) e = dev_malloc(&A->order, size_t(A->m) * sizeof(int32_t));
    if (e == cudaSuccess) e = launch_channel_order_rank(A->geom, A->m, A->cnl, prefix, A->rank, A->order, s);
    if (e == cudaSuccess) {
      *have = true;
    } else {
      dev_free(A->rank);
      dev_free(A->order);
      A->rank = A->order = nullptr;
    }
  }
  const double t2 = trace_on() ? trace_ms() : 0.0;
  dev_free(mark);
  dev_free(prefix);
  dev_free(tmp);
  dev_free(bad);
  if (trace_on())
    trace("row order: allocations %.2f ms, keys and ranks %.2f ms, release %.2f ms", t1 - t0, t2 - t1,
          trace_ms() - t2);
  return e;
}

}  // namespace

raptr_status raptr_matrix_transpose(raptr_matrix* A, void* stream) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (A->cp) return RAPTR_OK;
  DeviceScope ds(A->device);
  cudaStream_t s = as_stream(stream);
  bool ordered = false;
  const double t0 = trace_on() ? trace_ms() : 0.0;
  RCU(matrix_row_order(A, s, &ordered));
  const double t1 = trace_on() ? trace_ms() : 0.0;
  cudaError_t e = dev_malloc(&A->cp, size_t(A->n + 1) * sizeof(int64_t));
  if (e == cudaSuccess) e = dev_malloc(&A->trow, size_t(std::max<int64_t>(A->nnz, 1)) * sizeof(int32_t));
  if (e == cudaSuccess) e = dev_malloc(&A->tval, size_t(std::max<int64_t>(A->nnz, 1)) * sizeof(float));
  if (trace_on()) trace("transpose: row order %.2f ms, CSC allocations %.2f ms", t1 - t0, trace_ms() - t1);
  raptr_status st = RAPTR_OK;
  if (e != cudaSuccess)
    st = cuda_fail(e, "cudaMalloc(transpose)");
  else
    st = transpose_impl(A->m, A->n, A->rp, A->col, A->val, ordered ? A->order : nullptr, A->cp, A->trow, A->tval, s);
  if (st != RAPTR_OK) {
    dev_free(A->cp);
    dev_free(A->trow);
    dev_free(A->tval);
    dev_free(A->rank);
    dev_free(A->order);
    A->cp = nullptr;
    A->trow = nullptr;
    A->tval = nullptr;
    A->rank = A->order = nullptr;
  }
  return st;
}

raptr_status raptr_matrix_row_order(const raptr_matrix* A, int32_t** d_order, int32_t** d_rank) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (d_order) *d_order = A->order;
  if (d_rank) *d_rank = A->rank;
  return RAPTR_OK;
}

raptr_status raptr_matrix_csc_info(const raptr_matrix* A, int64_t** d_col_ptr, int32_t** d_row_idx, float** d_tval) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (d_col_ptr) *d_col_ptr = A->cp;
  if (d_row_idx) *d_row_idx = A->trow;
  if (d_tval) *d_tval = A->tval;
  return RAPTR_OK;
}

// ---- sparse formats ---------------------------------------------------------------

raptr_status raptr_coo2csr(const int32_t* d_rows, int64_t nnz, int64_t m, int64_t* d_row_ptr, void* stream) {
  if (m < 0 || nnz < 0 || !d_row_ptr || (nnz > 0 && !d_rows)) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_coo2csr(d_rows, nnz, m, d_row_ptr, nullptr, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_csr2ecsr(int64_t* d_ecsr, const int32_t* d_yrow, int64_t nnzr, const int64_t* d_csr, int64_t m,
                            void* stream) {
  if (nnzr < 0 || m < 0 || !d_ecsr || !d_csr || (nnzr > 0 && !d_yrow)) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_csr2ecsr(d_ecsr, d_yrow, nnzr, d_csr, m, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_row_ptr_narrow(const int64_t* d_in, int64_t n, int32_t* d_out, void* stream) {
  if (n < 0 || (n > 0 && (!d_in || !d_out))) return fail(RAPTR_ERR_INVALID, "bad argument");
  if (n == 0) return RAPTR_OK;
  cudaStream_t s = as_stream(stream);
  int64_t last = 0;
  RCU(cudaMemcpyAsync(&last, d_in + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  RCU(cudaStreamSynchronize(s));
  if (last > int64_t(INT32_MAX) || last < 0)
    return fail(RAPTR_ERR_INVALID, "row pointer " + std::to_string(last) + " does not fit in int32");
  RCU(launch_narrow_i64(d_in, n, d_out, s));
  return RAPTR_OK;
}

raptr_status raptr_row_ptr_widen(const int32_t* d_in, int64_t n, int64_t* d_out, void* stream) {
  if (n < 0 || (n > 0 && (!d_in || !d_out))) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_widen_i32(d_in, n, d_out, as_stream(stream)));
  return RAPTR_OK;
}

// ---- SpMV -----------------------------------------------------------------------------

raptr_status raptr_spmv(int32_t op, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                        const float* d_val, float alpha, const float* d_x, float beta, float* d_y, void* stream) {
  if (op != RAPTR_OP_N && op != RAPTR_OP_T) return fail(RAPTR_ERR_INVALID, "op must be RAPTR_OP_N or RAPTR_OP_T");
  if (m < 0 || n < 0 || !d_row_ptr || !d_x || !d_y) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_spmv(op, m, n, d_row_ptr, d_col, d_val, alpha, d_x, beta, d_y, as_stream(stream)));
  return RAPTR_OK;
}

// ---- element-wise ---------------------------------------------------------------------

raptr_status raptr_divides(float* d_res, const float* d_dividend, const float* d_divisor, int64_t n, void* stream) {
  if (n < 0 || (n > 0 && (!d_res || !d_dividend || !d_divisor))) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_divides(d_res, d_dividend, d_divisor, n, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_divides_multiplies(float* d_res, const float* d_a, const float* d_b, const float* d_c, int64_t n,
                                      void* stream) {
  if (n < 0 || (n > 0 && (!d_res || !d_a || !d_b || !d_c))) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_divides_multiplies(d_res, d_a, d_b, d_c, n, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_scales(float* d_x, float alpha, int64_t n, void* stream) {
  if (n < 0 || (n > 0 && !d_x)) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_scales(d_x, alpha, n, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_sum(const float* d_x, int64_t n, double* sum_out, void* stream) {
  if (n < 0 || !sum_out || (n > 0 && !d_x)) return fail(RAPTR_ERR_INVALID, "bad argument");
  cudaStream_t s = as_stream(stream);
  double* acc = nullptr;
  RCU(cudaMallocAsync(&acc, sizeof(double), s));
  cudaError_t e = launch_sum(d_x, n, acc, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sum_out, acc, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(acc, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "raptr_sum");
  return RAPTR_OK;
}

// ---- sensitivity and MLEM -------------------------------------------------------------

raptr_status raptr_sensitivity_csc(int64_t n, const int64_t* d_col_ptr, const float* d_tval, double* d_s64,
                                   float* d_s32, void* stream) {
  if (n <= 0 || !d_col_ptr || !d_s64) return fail(RAPTR_ERR_INVALID, "bad argument");
  cudaStream_t s = as_stream(stream);
  RCU(launch_column_sums_csc(n, d_col_ptr, d_tval, d_s64, s));
  if (d_s32) RCU(launch_sens_normalise_self(n, d_s64, d_s32, s));
  return RAPTR_OK;
}

raptr_status raptr_sensitivity(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                               const float* d_val, double* d_s64, float* d_s32, void* stream) {
  if (m < 0 || n <= 0 || !d_row_ptr || !d_s64) return fail(RAPTR_ERR_INVALID, "bad argument");
  cudaStream_t s = as_stream(stream);
  RCU(cudaMemsetAsync(d_s64, 0, size_t(n) * sizeof(double), s));
  RCU(launch_column_sums(m, d_row_ptr, d_col, d_val, d_s64, s));
  // no device scratch for the sum: a stream-ordered allocation here took
  // from microseconds to hundreds of milliseconds of host time
  if (d_s32) RCU(launch_sens_normalise_self(n, d_s64, d_s32, s));
  return RAPTR_OK;
}

raptr_status raptr_mlem_project(int64_t m, const int64_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                                const float* d_y, const float* d_x, float* d_c, double* d_ll, void* stream) {
  if (m < 0 || !d_row_ptr || !d_y || !d_x || !d_c) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_mlem_project(m, d_row_ptr, d_col, d_val, d_y, d_x, d_c, d_ll, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_mlem_update(int64_t n, float* d_x, float* d_c, const float* d_s, double* d_acc, void* stream) {
  if (n <= 0 || !d_x || !d_c || !d_s || !d_acc) return fail(RAPTR_ERR_INVALID, "bad argument");
  cudaStream_t s = as_stream(stream);
  RCU(cudaMemsetAsync(d_acc, 0, sizeof(double), s));
  RCU(launch_mlem_update(n, d_x, d_c, d_s, d_acc, s));
  RCU(launch_mlem_normalise(n, d_x, d_c, d_acc, s));
  return RAPTR_OK;
}

raptr_status raptr_mlem_forward(int64_t m, const int64_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                                const float* d_y, const float* d_x, float* d_e, double* d_ll, void* stream) {
  if (m < 0 || !d_row_ptr || !d_y || !d_x || !d_e) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_mlem_forward(m, d_row_ptr, d_col, d_val, d_y, d_x, nullptr, d_e, d_ll, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_mlem_forward_ordered(int64_t m, const int64_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                                        const float* d_y, const float* d_x, const int32_t* d_row_rank, float* d_e,
                                        double* d_ll, void* stream) {
  if (m < 0 || !d_row_ptr || !d_y || !d_x || !d_e || (m > 0 && !d_row_rank))
    return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_mlem_forward(m, d_row_ptr, d_col, d_val, d_y, d_x, d_row_rank, d_e, d_ll, as_stream(stream)));
  return RAPTR_OK;
}

raptr_status raptr_mlem_back(int64_t n, const int64_t* d_col_ptr, const int32_t* d_row_idx, const float* d_tval,
                             const float* d_e, float* d_c, void* stream) {
  if (n <= 0 || !d_col_ptr || !d_e || !d_c) return fail(RAPTR_ERR_INVALID, "bad argument");
  RCU(launch_mlem_back(n, d_col_ptr, d_row_idx, d_tval, d_e, nullptr, nullptr, d_c, nullptr, false,
                       as_stream(stream)));
  return RAPTR_OK;
}

namespace {

// Arrays of one MLEM form: FP16 when htval is set (with hval, rscale and
// the transpose), FP32 gather when the transpose is given, else FP32
// scatter over the rows.
struct MlemArrays {
  const int64_t* rp = nullptr;
  const int32_t* col = nullptr;
  const float* val = nullptr;
  const uint16_t* hval = nullptr;
  const float* rscale = nullptr;
  const int64_t* cp = nullptr;
  const int32_t* trow = nullptr;
  const float* tval = nullptr;
  const uint16_t* htval = nullptr;
  // delta-coded FP16 runs (with rscale): rows and transpose columns
  const int64_t* pseg = nullptr;
  const int32_t* panchor = nullptr;
  const uint32_t* pword = nullptr;
  const int64_t* tseg = nullptr;
  const int32_t* tanchor = nullptr;
  const uint32_t* tword = nullptr;
};

raptr_status mlem_impl(raptr_ctx* ctx, int64_t m, int64_t n, const MlemArrays& A, const float* d_y, const float* d_s,
                       float* d_x, int32_t n_iter, const raptr_mlem_opts* opts, cudaStream_t s) {
  const int64_t* d_row_ptr = A.rp;
  const int32_t* d_col = A.col;
  const float* d_val = A.val;
  const int64_t* d_col_ptr = A.cp;
  const int32_t* d_row_idx = A.trow;
  const float* d_tval = A.tval;
  const bool packed = A.pword != nullptr;
  const bool half = A.htval != nullptr;
  if (n_iter == 0) return RAPTR_OK;
  DeviceScope ds(ctx->device);
  const bool want_ll = opts && opts->h_loglik;
  const bool want_times = opts && opts->h_kernel_ms;
  const bool use_graph = opts && opts->use_graph && !want_times;
  const bool csc = d_col_ptr != nullptr || packed;
  const int32_t* rank = opts ? opts->d_row_rank : nullptr;
  std::vector<cudaEvent_t> evs;
  if (want_times) {
    evs.resize(size_t(3 * n_iter));
    for (auto& ev : evs) RCU(cudaEventCreate(&ev));
  }
  RCHECK(ctx->ensure_scratch(Carve::need({size_t(n) * sizeof(float), size_t(csc ? m : 1) * sizeof(float),
                                          size_t(2 * n_iter + 4) * sizeof(double)})));
  Carve cv(ctx->d_scratch);
  float* c = cv.take<float>(size_t(n));  // correction (scatter path) or x before normalisation
  float* e = cv.take<float>(size_t(csc ? m : 1));
  double* acc = cv.take<double>(size_t(2 * n_iter + 4));
  // acc[0]: the image sum; acc[1], acc[2]: the counters the forward and
  // back passes draw rows and columns from (all three cleared in every
  // iteration); from acc[4]: log-likelihood sums
  auto* next_row = reinterpret_cast<unsigned long long*>(acc + 1);
  auto* next_col = reinterpret_cast<unsigned long long*>(acc + 2);
  double* ll = acc + 4;
  RCU(cudaMemsetAsync(c, 0, size_t(n) * sizeof(float), s));
  RCU(cudaMemsetAsync(acc, 0, size_t(2 * n_iter + 4) * sizeof(double), s));

  auto enqueue = [&](cudaStream_t q) -> cudaError_t {
    for (int32_t it = 0; it < n_iter; it++) {
      double* lli = want_ll ? ll + 2 * it : nullptr;
      cudaError_t err = cudaMemsetAsync(acc, 0, 3 * sizeof(double), q);
      if (want_times && err == cudaSuccess) err = cudaEventRecord(evs[size_t(3 * it)], q);
      if (csc) {
        if (err == cudaSuccess)
          err = packed ? launch_mlem_forward_packed(m, A.pseg, A.panchor, A.pword, A.rscale, d_y, d_x, rank, e, lli,
                                                    next_row, q)
                : half ? launch_mlem_forward_half(m, d_row_ptr, d_col, A.hval, A.rscale, d_y, d_x, rank, e, lli, q,
                                                  next_row)
                       : launch_mlem_forward(m, d_row_ptr, d_col, d_val, d_y, d_x, rank, e, lli, q, next_row);
        if (want_times && err == cudaSuccess) err = cudaEventRecord(evs[size_t(3 * it + 1)], q);
        if (err == cudaSuccess)
          err = packed ? launch_mlem_back_packed(n, A.tseg, A.tanchor, A.tword, e, d_x, d_s, c, acc, true, next_col, q)
                : half ? launch_mlem_back_half(n, d_col_ptr, d_row_idx, A.htval, e, d_x, d_s, c, acc, true, q,
                                               next_col)
                       : launch_mlem_back(n, d_col_ptr, d_row_idx, d_tval, e, d_x, d_s, c, acc, true, q, next_col);
        if (want_times && err == cudaSuccess) err = cudaEventRecord(evs[size_t(3 * it + 2)], q);
        if (err == cudaSuccess) err = launch_mlem_normalise_from(n, d_x, c, acc, q);
      } else {
        if (err == cudaSuccess) err = launch_mlem_project(m, d_row_ptr, d_col, d_val, d_y, d_x, c, lli, q);
        if (want_times && err == cudaSuccess) err = cudaEventRecord(evs[size_t(3 * it + 1)], q);
        if (err == cudaSuccess) err = launch_mlem_update(n, d_x, c, d_s, acc, q);
        if (want_times && err == cudaSuccess) err = cudaEventRecord(evs[size_t(3 * it + 2)], q);
        if (err == cudaSuccess) err = launch_mlem_normalise(n, d_x, c, acc, q);
      }
      if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
  };

  if (!use_graph) {
    RCU(enqueue(s));
  } else {
    const double tg0 = trace_on() ? trace_ms() : 0.0;
    cudaStream_t cap;
    RCU(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ev, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cap, ev, 0);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t e1 = enqueue(cap);
      cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
      e = (e1 != cudaSuccess) ? e1 : e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    const double tg1 = trace_on() ? trace_ms() : 0.0;
    if (trace_on()) trace("mlem: %d iterations captured and instantiated in %.2f ms", int(n_iter), tg1 - tg0);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, cap);
    // the launches were counted when they were captured; the graph runs
    // each of them once
    if (e == cudaSuccess) e = cudaEventRecord(ev, cap);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cap);
    const double tg2 = trace_on() ? trace_ms() : 0.0;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventDestroy(ev);
    cudaStreamDestroy(cap);
    if (trace_on()) trace("mlem: graph ran in %.2f ms, released in %.2f ms", tg2 - tg1, trace_ms() - tg2);
    if (e != cudaSuccess) return cuda_fail(e, "MLEM graph");
  }
  if (want_times) {
    RCU(cudaStreamSynchronize(s));
    for (int32_t it = 0; it < n_iter; it++) {
      float a = 0.f, b = 0.f;
      RCU(cudaEventElapsedTime(&a, evs[size_t(3 * it)], evs[size_t(3 * it + 1)]));
      RCU(cudaEventElapsedTime(&b, evs[size_t(3 * it + 1)], evs[size_t(3 * it + 2)]));
      opts->h_kernel_ms[2 * it] = a;
      opts->h_kernel_ms[2 * it + 1] = b;
    }
    for (auto& ev : evs) cudaEventDestroy(ev);
  }
  if (want_ll) {
    std::vector<double> h(size_t(2 * n_iter));
    RCU(cudaMemcpyAsync(h.data(), ll, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    double ysum = 0.0;
    RCU(launch_sum(d_y, m, acc + 1, s));
    RCU(cudaMemcpyAsync(&ysum, acc + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    RCU(cudaStreamSynchronize(s));
    // Poisson log-likelihood (without the log y! term) at the best global
    // scale of A x: sum y log(k Ax) - k sum Ax with k = sum y / sum Ax.
    for (int32_t it = 0; it < n_iter; it++) {
      double s1 = h[size_t(2 * it)], s2 = h[size_t(2 * it + 1)];
      opts->h_loglik[it] = s1 + ysum * std::log(ysum / s2) - ysum;
    }
  }
  return RAPTR_OK;
}

}  // namespace

raptr_status raptr_mlem(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                        const float* d_val, const int64_t* d_col_ptr, const int32_t* d_row_idx, const float* d_tval,
                        const float* d_y, const float* d_s, float* d_x, int32_t n_iter, const raptr_mlem_opts* opts,
                        void* stream) {
  if (!ctx || m < 0 || n <= 0 || n_iter < 0 || !d_row_ptr || !d_y || !d_s || !d_x)
    return fail(RAPTR_ERR_INVALID, "bad argument");
  MlemArrays A;
  A.rp = d_row_ptr;
  A.col = d_col;
  A.val = d_val;
  A.cp = d_col_ptr;
  A.trow = d_row_idx;
  A.tval = d_tval;
  return mlem_impl(ctx, m, n, A, d_y, d_s, d_x, n_iter, opts, as_stream(stream));
}

raptr_status raptr_mlem_half(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                             const uint16_t* d_hval, const float* d_rscale, const int64_t* d_col_ptr,
                             const int32_t* d_row_idx, const uint16_t* d_htval, const float* d_y, const float* d_s,
                             float* d_x, int32_t n_iter, const raptr_mlem_opts* opts, void* stream) {
  if (!ctx || m < 0 || n <= 0 || n_iter < 0 || !d_row_ptr || !d_y || !d_s || !d_x || !d_col_ptr || !d_htval ||
      (m > 0 && (!d_hval || !d_rscale)))
    return fail(RAPTR_ERR_INVALID, "bad argument");
  MlemArrays A;
  A.rp = d_row_ptr;
  A.col = d_col;
  A.hval = d_hval;
  A.rscale = d_rscale;
  A.cp = d_col_ptr;
  A.trow = d_row_idx;
  A.htval = d_htval;
  return mlem_impl(ctx, m, n, A, d_y, d_s, d_x, n_iter, opts, as_stream(stream));
}

raptr_status raptr_mlem_packed(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_seg, const int32_t* d_anchor,
                               const uint32_t* d_words, const float* d_rscale, const int64_t* d_tseg,
                               const int32_t* d_tanchor, const uint32_t* d_twords, const float* d_y,
                               const float* d_s, float* d_x, int32_t n_iter, const raptr_mlem_opts* opts,
                               void* stream) {
  if (!ctx || m < 0 || n <= 0 || n_iter < 0 || !d_y || !d_s || !d_x || !d_tseg || !d_tanchor || !d_twords ||
      (m > 0 && (!d_seg || !d_anchor || !d_words || !d_rscale)))
    return fail(RAPTR_ERR_INVALID, "bad argument");
  if (((reinterpret_cast<uintptr_t>(d_words) | reinterpret_cast<uintptr_t>(d_twords)) & 15u) != 0)
    return fail(RAPTR_ERR_INVALID, "the words of the delta-coded runs must be 16-byte aligned");
  MlemArrays A;
  A.rscale = d_rscale;
  A.pseg = d_seg;
  A.panchor = d_anchor;
  A.pword = d_words;
  A.tseg = d_tseg;
  A.tanchor = d_tanchor;
  A.tword = d_twords;
  return mlem_impl(ctx, m, n, A, d_y, d_s, d_x, n_iter, opts, as_stream(stream));
}

raptr_status raptr_mlem_f64(raptr_ctx* ctx, int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                            const float* d_val, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                            const float* d_tval, const int32_t* d_row_rank, const float* d_y, const double* d_s64,
                            double* d_x64, int32_t n_iter, double* h_loglik, void* stream) {
  if (!ctx || m < 0 || n <= 0 || n_iter < 0 || !d_row_ptr || !d_col_ptr || !d_y || !d_s64 || !d_x64)
    return fail(RAPTR_ERR_INVALID, "bad argument");
  if (n_iter == 0) return RAPTR_OK;
  DeviceScope ds(ctx->device);
  cudaStream_t s = as_stream(stream);
  double *e = nullptr, *xx = nullptr, *acc = nullptr;
  cudaError_t err = cudaMallocAsync(&e, size_t(std::max<int64_t>(m, 1)) * sizeof(double), s);
  if (err == cudaSuccess) err = cudaMallocAsync(&xx, size_t(n) * sizeof(double), s);
  if (err == cudaSuccess) err = cudaMallocAsync(&acc, size_t(2 * n_iter + 2) * sizeof(double), s);
  if (err == cudaSuccess) err = cudaMemsetAsync(acc, 0, size_t(2 * n_iter + 2) * sizeof(double), s);
  for (int32_t it = 0; it < n_iter && err == cudaSuccess; it++)
    err = launch_mlem_f64_iteration(m, n, d_row_ptr, d_col, d_val, d_col_ptr, d_row_idx, d_tval, d_row_rank, d_y,
                                    d_s64, d_x64, e, xx, acc, h_loglik ? acc + 2 + 2 * it : nullptr, s);
  std::vector<double> h(size_t(2 * n_iter));
  double ysum = 0.0;
  if (err == cudaSuccess && h_loglik) {
    err = cudaMemcpyAsync(h.data(), acc + 2, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = launch_sum(d_y, m, acc + 1, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&ysum, acc + 1, sizeof(double), cudaMemcpyDeviceToHost, s);
  }
  if (e) cudaFreeAsync(e, s);
  if (xx) cudaFreeAsync(xx, s);
  if (acc) cudaFreeAsync(acc, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cuda_fail(err, "raptr_mlem_f64");
  if (h_loglik)
    for (int32_t it = 0; it < n_iter; it++)
      h_loglik[it] = h[size_t(2 * it)] + ysum * std::log(ysum / h[size_t(2 * it + 1)]) - ysum;
  return RAPTR_OK;
}

raptr_status raptr_matrix_half(raptr_matrix* A, void* stream) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (!A->cp) return fail(RAPTR_ERR_INVALID, "the FP16 form needs the transpose: call raptr_matrix_transpose first");
  if (A->hval) return RAPTR_OK;
  DeviceScope ds(A->device);
  cudaStream_t s = as_stream(stream);
  const size_t mm = size_t(std::max<int64_t>(A->m, 1)), nz = size_t(std::max<int64_t>(A->nnz, 1));
  cudaError_t e = dev_malloc(&A->rscale, mm * sizeof(float));
  if (e == cudaSuccess) e = dev_malloc(&A->pscale, mm * sizeof(float));
  if (e == cudaSuccess) e = dev_malloc(&A->hval, nz * sizeof(uint16_t));
  if (e == cudaSuccess) e = dev_malloc(&A->htval, nz * sizeof(uint16_t));
  if (e == cudaSuccess)
    e = launch_half_convert(A->m, A->nnz, A->rp, A->val, A->trow, A->tval, A->order, A->rscale, A->hval, A->htval,
                            A->pscale, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    dev_free(A->rscale);
    dev_free(A->pscale);
    dev_free(A->hval);
    dev_free(A->htval);
    A->rscale = A->pscale = nullptr;
    A->hval = A->htval = nullptr;
    return cuda_fail(e, "raptr_matrix_half");
  }
  return RAPTR_OK;
}

raptr_status raptr_matrix_half_info(const raptr_matrix* A, uint16_t** d_hval, float** d_rscale, uint16_t** d_htval,
                                    float** d_pscale) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (d_hval) *d_hval = A->hval;
  if (d_rscale) *d_rscale = A->rscale;
  if (d_htval) *d_htval = A->htval;
  if (d_pscale) *d_pscale = A->pscale;
  return RAPTR_OK;
}

raptr_status raptr_pack_half(int64_t count, const int64_t* d_ptr, const int32_t* d_idx, const uint16_t* d_hv,
                             int64_t* d_seg, int32_t* d_anchor, uint32_t* d_words, int64_t words_cap,
                             int64_t* h_words, void* stream) {
  if (count < 0 || !d_ptr || !d_seg || !h_words) return fail(RAPTR_ERR_INVALID, "bad argument");
  if (d_words && (!d_anchor || !d_idx || !d_hv)) return fail(RAPTR_ERR_INVALID, "bad argument");
  if ((reinterpret_cast<uintptr_t>(d_words) & 15u) != 0) return fail(RAPTR_ERR_INVALID, "d_words is not 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  int64_t *quads = nullptr, *tmp = nullptr;
  int32_t* bad = nullptr;
  int32_t h_bad = 0;
  int64_t h_quads = 0;
  cudaError_t e = cudaMallocAsync(&quads, size_t(std::max<int64_t>(count, 1)) * sizeof(int64_t), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&tmp, size_t(scan_temp_elems(count)) * sizeof(int64_t), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&bad, sizeof(int32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
  if (e == cudaSuccess) e = launch_pack_count(count, d_ptr, d_idx, quads, bad, s);
  if (e == cudaSuccess) e = launch_scan_i64(quads, count, d_seg, tmp, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_quads, d_seg + count, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  const bool fill = e == cudaSuccess && !h_bad && d_words && h_quads * 4 <= words_cap;
  if (fill) e = launch_pack_fill(count, d_ptr, d_idx, d_hv, d_seg, d_anchor, d_words, s);
  if (fill && e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(quads, s);
  cudaFreeAsync(tmp, s);
  cudaFreeAsync(bad, s);
  if (e != cudaSuccess) return cuda_fail(e, "raptr_pack_half");
  if (h_bad) return fail(RAPTR_ERR_INVALID, "indices descend within a run");
  *h_words = h_quads * 4;
  if (d_words && h_quads * 4 > words_cap) return fail(RAPTR_ERR_INVALID, "words_cap is below the words needed");
  return RAPTR_OK;
}

raptr_status raptr_matrix_packed(raptr_matrix* A, void* stream) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (!A->hval) return fail(RAPTR_ERR_INVALID, "the delta-coded form needs the FP16 form: call raptr_matrix_half first");
  if (A->pword) return RAPTR_OK;
  DeviceScope ds(A->device);
  raptr_status st = RAPTR_OK;
  auto pack = [&](int64_t count, const int64_t* ptr, const int32_t* idx, const uint16_t* hv, int64_t** seg,
                  int32_t** anc, uint32_t** words, int64_t* nwords) {
    if (st != RAPTR_OK) return;
    cudaError_t e = dev_malloc(seg, size_t(count + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = dev_malloc(anc, size_t(std::max<int64_t>(count, 1)) * sizeof(int32_t));
    if (e != cudaSuccess) {
      st = cuda_fail(e, "raptr_matrix_packed");
      return;
    }
    st = raptr_pack_half(count, ptr, idx, hv, *seg, *anc, nullptr, 0, nwords, stream);
    if (st != RAPTR_OK) return;
    e = dev_malloc(words, size_t(std::max<int64_t>(*nwords, 4)) * sizeof(uint32_t));
    if (e != cudaSuccess) {
      st = cuda_fail(e, "raptr_matrix_packed");
      return;
    }
    st = raptr_pack_half(count, ptr, idx, hv, *seg, *anc, *words, *nwords, nwords, stream);
  };
  pack(A->m, A->rp, A->col, A->hval, &A->pseg, &A->panchor, &A->pword, &A->pwords);
  pack(A->n, A->cp, A->trow, A->htval, &A->tseg, &A->tanchor, &A->tword, &A->twords);
  if (st != RAPTR_OK) {
    const std::string msg = g_last_error;
    dev_free(A->pseg);
    dev_free(A->panchor);
    dev_free(A->pword);
    dev_free(A->tseg);
    dev_free(A->tanchor);
    dev_free(A->tword);
    A->pseg = A->tseg = nullptr;
    A->panchor = A->tanchor = nullptr;
    A->pword = A->tword = nullptr;
    A->pwords = A->twords = 0;
    return fail(st, msg);
  }
  return RAPTR_OK;
}

raptr_status raptr_matrix_packed_info(const raptr_matrix* A, int64_t** d_seg, int32_t** d_anchor,
                                      uint32_t** d_words, int64_t** d_tseg, int32_t** d_tanchor,
                                      uint32_t** d_twords) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (d_seg) *d_seg = A->pseg;
  if (d_anchor) *d_anchor = A->panchor;
  if (d_words) *d_words = A->pword;
  if (d_tseg) *d_tseg = A->tseg;
  if (d_tanchor) *d_tanchor = A->tanchor;
  if (d_twords) *d_twords = A->tword;
  return RAPTR_OK;
}

raptr_status raptr_matrix_drop_f32(raptr_matrix* A) {
  if (!A) return fail(RAPTR_ERR_INVALID, "matrix is null");
  if (!A->hval) return fail(RAPTR_ERR_INVALID, "the FP32 values are the only ones: call raptr_matrix_half first");
  DeviceScope ds(A->device);
  dev_free(A->val);
  dev_free(A->tval);
  A->val = nullptr;
  A->tval = nullptr;
  return RAPTR_OK;
}

raptr_status raptr_matrix_bytes(const raptr_matrix* A, int64_t* bytes) {
  if (!A || !bytes) return fail(RAPTR_ERR_INVALID, "bad argument");
  const int64_t m = A->m, n = A->n, z = A->nnz;
  int64_t b = (m + 1) * 8 + (A->col ? z * 4 : 0) + (A->val ? z * 4 : 0);
  if (A->cp) b += (n + 1) * 8 + (A->trow ? z * 4 : 0) + (A->tval ? z * 4 : 0);
  if (A->cnl) b += m * 4;
  if (A->rank) b += m * 8;
  if (A->hval) b += z * 4 + m * 8;
  if (A->pword) b += (A->pwords + A->twords) * 4 + (m + 1) * 8 + m * 4 + (n + 1) * 8 + n * 4;
  *bytes = b;
  return RAPTR_OK;
}

raptr_status raptr_sensitivity_half(int64_t n, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                                    const uint16_t* d_htval, const float* d_pscale, double* d_s64, float* d_s32,
                                    void* stream) {
  if (n <= 0 || !d_col_ptr || !d_s64) return fail(RAPTR_ERR_INVALID, "bad argument");
  cudaStream_t s = as_stream(stream);
  RCU(launch_sens_half(n, d_col_ptr, d_row_idx, d_htval, d_pscale, d_s64, s));
  if (d_s32) RCU(launch_sens_normalise_self(n, d_s64, d_s32, s));
  return RAPTR_OK;
}

// ---- batched MLEM ----------------------------------------------------------

namespace {

raptr_status batch_args(raptr_ctx* ctx, int64_t m, int64_t n, int32_t K, int32_t value_type, const int64_t* d_row_ptr,
                        const int32_t* d_col, const void* d_val, const float* d_rscale, const int64_t* d_col_ptr,
                        const int32_t* d_row_idx, const void* d_tval, const int32_t* d_row_rank, const float* d_y,
                        const float* d_s, float* d_x, BatchArgs* a) {
  if (!ctx || m < 0 || n <= 0 || K <= 0 || K > 4096 || (value_type != 0 && value_type != 1) || !d_row_ptr ||
      !d_col_ptr || !d_y || !d_s || !d_x || (m > 0 && (!d_val || !d_tval)) || (value_type == 1 && m > 0 && !d_rscale))
    return fail(RAPTR_ERR_INVALID, "bad argument");
  // the passes gather four frames at a time (16-byte loads of the images
  // and measurements)
  if ((reinterpret_cast<uintptr_t>(d_x) & 15u) != 0 || (reinterpret_cast<uintptr_t>(d_y) & 15u) != 0)
    return fail(RAPTR_ERR_INVALID, "the images and measurements must be 16-byte aligned");
  a->m = m;
  a->n = n;
  a->K = K;
  a->half = value_type == 1;
  a->rp = d_row_ptr;
  a->col = d_col;
  a->val = d_val;
  a->rscale = d_rscale;
  a->cp = d_col_ptr;
  a->trow = d_row_idx;
  a->tval = d_tval;
  a->rank = d_row_rank;
  a->Y = d_y;
  a->S = d_s;
  a->X = d_x;
  return RAPTR_OK;
}

int default_frame_tile(int K) { return batch_tile_supported(K, 32) ? 32 : 0; }

}  // namespace

raptr_status raptr_mlem_batch(raptr_ctx* ctx, int64_t m, int64_t n, int32_t n_frames, int32_t value_type,
                              const int64_t* d_row_ptr, const int32_t* d_col, const void* d_val,
                              const float* d_rscale, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                              const void* d_tval, const int32_t* d_row_rank, const float* d_y, const float* d_s,
                              float* d_x, int32_t n_iter, int32_t frame_tile, const raptr_mlem_opts* opts,
                              void* stream) {
  BatchArgs a;
  RCHECK(batch_args(ctx, m, n, n_frames, value_type, d_row_ptr, d_col, d_val, d_rscale, d_col_ptr, d_row_idx, d_tval,
                    d_row_rank, d_y, d_s, d_x, &a));
  if (n_iter < 0) return fail(RAPTR_ERR_INVALID, "bad argument");
  const int kt = frame_tile > 0 ? frame_tile : default_frame_tile(n_frames);
  if (!batch_tile_supported(n_frames, kt))
    return fail(RAPTR_ERR_INVALID, "the number of frames must be a multiple of 4 and the frame tile 4, 8, 16, 32 or 64");
  if (n_iter == 0) return RAPTR_OK;
  DeviceScope ds(ctx->device);
  cudaStream_t s = as_stream(stream);
  const bool want_times = opts && opts->h_kernel_ms;
  const bool use_graph = opts && opts->use_graph && !want_times;
  RCHECK(ctx->ensure_scratch(Carve::need({size_t(std::max<int64_t>(m, 1)) * n_frames * sizeof(float),
                                          size_t(n) * n_frames * sizeof(float), size_t(n_frames) * sizeof(double),
                                          size_t(n_frames) * sizeof(unsigned long long) * kBatchRowBlocks,
                                          size_t(n) * std::min(kt, int(n_frames)) * sizeof(float),
                                          size_t(n) * batch_tile_at(n_frames, kt, 0) * sizeof(float)})));
  Carve cv(ctx->d_scratch);
  // the tube order of the back pass applies when the columns are the
  // context's voxels
  if (n == int64_t(ctx->dg.n[0]) * ctx->dg.n[1] * ctx->dg.n[2]) RCU(ctx->col_order(&a.col_order));
  a.E = cv.take<float>(size_t(std::max<int64_t>(m, 1)) * n_frames);
  a.XX = cv.take<float>(size_t(n) * n_frames);
  double* acc = cv.take<double>(size_t(n_frames));
  unsigned long long* next = cv.take<unsigned long long>(size_t(n_frames) * kBatchRowBlocks);
  // the compact images of a tile narrower than the batch (the first tile
  // is the widest: 12 frames at kt = 64 run as 8 + 4)
  const int widest = batch_tile_at(n_frames, kt, 0);
  if (widest < n_frames) a.Xt = cv.take<float>(size_t(n) * widest);
  // the back pass in row-block groups when one tile's ratios exceed L2
  if (m > 0 && double(m) * std::min(kt, int(n_frames)) * sizeof(float) > kBatchBlockingBytes) {
    RCU(ctx->block_seg(d_col_ptr, d_row_idx, m, n, s, &a.seg));
    a.seg_blocks = kBatchRowBlocks;
    a.P = cv.take<float>(size_t(n) * std::min(kt, int(n_frames)));
  }
  std::vector<cudaEvent_t> evs;
  if (want_times) {
    evs.resize(size_t(3 * n_iter));
    for (auto& ev : evs) RCU(cudaEventCreate(&ev));
  }
  auto enqueue = [&](cudaStream_t q) -> cudaError_t {
    for (int32_t it = 0; it < n_iter; it++) {
      cudaError_t err = cudaSuccess;
      if (want_times) err = cudaEventRecord(evs[size_t(3 * it)], q);
      if (err == cudaSuccess) err = launch_batch_iteration(a, kt, acc, next, q, want_times ? evs[size_t(3 * it + 1)] : nullptr);
      if (want_times && err == cudaSuccess) err = cudaEventRecord(evs[size_t(3 * it + 2)], q);
      if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
  };
  if (!use_graph) {
    RCU(enqueue(s));
  } else {
    cudaStream_t cap;
    RCU(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ev, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cap, ev, 0);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t e1 = enqueue(cap);
      cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
      e = (e1 != cudaSuccess) ? e1 : e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, cap);
    if (e == cudaSuccess) e = cudaEventRecord(ev, cap);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cap);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventDestroy(ev);
    cudaStreamDestroy(cap);
    if (e != cudaSuccess) return cuda_fail(e, "batched MLEM graph");
  }
  if (want_times) {
    RCU(cudaStreamSynchronize(s));
    for (int32_t it = 0; it < n_iter; it++) {
      float t0 = 0.f, t1 = 0.f;
      RCU(cudaEventElapsedTime(&t0, evs[size_t(3 * it)], evs[size_t(3 * it + 1)]));
      RCU(cudaEventElapsedTime(&t1, evs[size_t(3 * it + 1)], evs[size_t(3 * it + 2)]));
      opts->h_kernel_ms[2 * it] = t0;
      opts->h_kernel_ms[2 * it + 1] = t1;
    }
    for (auto& ev : evs) cudaEventDestroy(ev);
  }
  return RAPTR_OK;
}

raptr_status raptr_mlem_batch_autotune(raptr_ctx* ctx, int64_t m, int64_t n, int32_t n_frames, int32_t value_type,
                                       const int64_t* d_row_ptr, const int32_t* d_col, const void* d_val,
                                       const float* d_rscale, const int64_t* d_col_ptr, const int32_t* d_row_idx,
                                       const void* d_tval, const int32_t* d_row_rank, const float* d_y,
                                       const float* d_s, const float* d_x, int32_t* best_tile, float* h_ms,
                                       void* stream) {
  if (!best_tile) return fail(RAPTR_ERR_INVALID, "bad argument");
  DeviceScope ds(ctx ? ctx->device : 0);
  cudaStream_t s = as_stream(stream);
  // time one iteration per candidate tile on a copy of the images
  float* xc = nullptr;
  RCU(cudaMallocAsync(&xc, size_t(n) * n_frames * sizeof(float), s));
  const int tiles[5] = {4, 8, 16, 32, 64};
  float best = 0.f;
  *best_tile = 0;
  raptr_status st = RAPTR_OK;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int i = 0; i < 5 && st == RAPTR_OK; i++) {
    const int kt = tiles[i];
    if (h_ms) h_ms[i] = -1.f;
    if (!batch_tile_supported(n_frames, kt)) continue;
    float ms = 0.f;
    for (int rep = 0; rep < 3 && st == RAPTR_OK; rep++) {  // first is a warm-up
      cudaMemcpyAsync(xc, d_x, size_t(n) * n_frames * sizeof(float), cudaMemcpyDeviceToDevice, s);
      cudaEventRecord(e0, s);
      st = raptr_mlem_batch(ctx, m, n, n_frames, value_type, d_row_ptr, d_col, d_val, d_rscale, d_col_ptr, d_row_idx,
                            d_tval, d_row_rank, d_y, d_s, xc, 1, kt, nullptr, stream);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms += t / 2;
    }
    if (h_ms) h_ms[i] = ms;
    if (st == RAPTR_OK && (*best_tile == 0 || ms < best)) {
      best = ms;
      *best_tile = kt;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(xc, s);
  cudaStreamSynchronize(s);
  if (st != RAPTR_OK) return st;
  if (*best_tile == 0) return fail(RAPTR_ERR_INVALID, "no frame tile divides the number of frames");
  return RAPTR_OK;
}

raptr_status raptr_mlem_stream(raptr_ctx* ctx, const int32_t* d_cnl, int64_t n_list, int32_t nrays, uint32_t seed,
                               const float* d_y, const float* d_s, float* d_s_out, float* d_x, int32_t n_iter,
                               int64_t resident_bytes, raptr_stream_stats* stats, void* stream) {
  if (!ctx || n_list < 0 || (n_list > 0 && (!d_cnl || !d_y)) || nrays <= 0 || n_iter < 0 || !d_x ||
      resident_bytes < 0)
    return fail(RAPTR_ERR_INVALID, "bad argument");
  if (stats) *stats = raptr_stream_stats{};
  if (n_iter == 0) return RAPTR_OK;
  DeviceScope ds(ctx->device);
  cudaStream_t s = as_stream(stream);
  const int64_t N = raptr_ctx_num_voxels(ctx);
  // resident CSR of the leading rows: row pointers for every row, entries
  // up to what resident_bytes leaves after them
  const int64_t rp_bytes = (n_list + 1) * int64_t(sizeof(int64_t));
  const int64_t cap = resident_bytes > rp_bytes ? (resident_bytes - rp_bytes) / 8 : 0;
  int64_t* rp = nullptr;
  int32_t* rcol = nullptr;
  float* rval = nullptr;
  float *c = nullptr, *s32 = nullptr;
  double* s64 = nullptr;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  struct Owned {
    std::function<void()> f;
    ~Owned() { f(); }
  } owned{[&] {
    dev_free(rp);
    dev_free(rcol);
    dev_free(rval);
    dev_free(c);
    dev_free(s32);
    dev_free(s64);
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }};
  for (auto& e : ev) RCU(cudaEventCreate(&e));
  if (cap > 0) {
    RCU(dev_malloc(&rp, size_t(rp_bytes)));
    RCU(dev_malloc(&rcol, size_t(cap) * sizeof(int32_t)));
    RCU(dev_malloc(&rval, size_t(cap) * sizeof(float)));
  }
  RCU(dev_malloc(&c, size_t(N) * sizeof(float)));
  if (!d_s) {
    RCU(dev_malloc(&s64, size_t(N) * sizeof(double)));
    RCU(dev_malloc(&s32, size_t(N) * sizeof(float)));
  }
  const float* s_use = d_s ? d_s : s32;
  double* acc = ctx->d_f64;  // [0]: image sum, [1]: sensitivity sum
  int level = sm_pick_level(ctx->dg, nrays);
  int64_t n_res = 0, n_ent = 0;
  volatile int64_t* h_words = nullptr;
  if (!ctx->h_pin) RCU(cudaMallocHost(&ctx->h_pin, 16 * sizeof(int64_t)));
  h_words = ctx->h_pin;
  volatile int32_t* h_flags = reinterpret_cast<volatile int32_t*>(const_cast<int64_t*>(h_words + 4));

  // Builds rows [from, n_list) chunk by chunk and projects them from the
  // staging; in the first iteration also keeps the leading chunks that fit
  // the resident CSR.
  auto sweep = [&](bool first, int64_t from) -> raptr_status {
    const int H = sm_level_capacity(level);
    int64_t per = std::max<int64_t>(1, int64_t(kStagingBudget / (size_t(H) * 8)));
    per = std::min<int64_t>(per, 65536);
    // fewer rows per chunk when the device (or the library's memory limit)
    // has less room than the usual staging
    const size_t room = dev_available(ctx->device) + ctx->scratch_bytes;
    per = std::max<int64_t>(1, std::min<int64_t>(per, int64_t(double(room) * 0.8 / (double(H) * 8 + 8))));
    RCHECK(ctx->ensure_scratch(Carve::need({size_t(per) * H * sizeof(int32_t), size_t(per) * H * sizeof(float),
                                            size_t(per) * sizeof(int32_t)})));
    Carve cv(ctx->d_scratch);
    int32_t* st_col = cv.take<int32_t>(size_t(per) * H);
    float* st_val = cv.take<float>(size_t(per) * H);
    int32_t* row_nnz = cv.take<int32_t>(size_t(per));
    bool open = first && cap > 0;
    for (int64_t r = from; r < n_list; r += per) {
      const int64_t k = std::min(per, n_list - r);
      RCU(launch_sm_rows(level, ctx->dg, ctx->d_sincos, d_cnl, r, k, nrays, seed, nullptr, st_col, st_val, row_nnz,
                         ctx->d_flags, s));
      RCU(launch_stage_project(k, st_col, st_val, H, row_nnz, d_y + r, d_x, c, first ? s64 : nullptr, s));
      if (!open) continue;
      RCU(launch_rows_scan(row_nnz, k, rp + r, ctx->d_i64, s));
      RCU(cudaMemcpyAsync(const_cast<int64_t*>(h_words), ctx->d_i64, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      RCU(cudaMemcpyAsync(const_cast<int32_t*>(h_flags), ctx->d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      RCU(cudaStreamSynchronize(s));
      const int64_t total = h_words[0];
      if (*h_flags != 0) {
        open = false;  // redone a level up anyway
        continue;
      }
      int64_t keep = k, kept_entries = total;
      if (total > cap) {
        // the chunk's leading rows that still fit; the rest of it and every
        // later chunk are rebuilt in every iteration
        std::vector<int64_t> h_rp(size_t(k) + 1);
        RCU(cudaMemcpy(h_rp.data(), rp + r, h_rp.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
        keep = int64_t(std::upper_bound(h_rp.begin(), h_rp.end(), cap) - h_rp.begin()) - 1;
        kept_entries = h_rp[size_t(keep)];
        open = false;
      }
      if (keep > 0) RCU(launch_rows_gather(st_col, st_val, H, rp + r, keep, cap, rcol, rval, s));
      n_res = r + keep;
      n_ent = kept_entries;
    }
    return RAPTR_OK;
  };

  for (int32_t it = 0; it < n_iter; it++) {
    const bool first = it == 0;
    if (first) RCU(cudaEventRecord(ev[0], s));
    RCU(cudaMemsetAsync(ctx->d_flags, 0, sizeof(int32_t), s));
    if (first) {
      n_res = n_ent = 0;
      RCU(cudaMemsetAsync(c, 0, size_t(N) * sizeof(float), s));
      RCU(cudaMemsetAsync(ctx->d_i64, 0, sizeof(int64_t), s));
      if (s64) RCU(cudaMemsetAsync(s64, 0, size_t(N) * sizeof(double), s));
    } else if (n_res > 0) {
      RCU(launch_mlem_project(n_res, rp, rcol, rval, d_y, d_x, c, nullptr, s));
    }
    RCHECK(sweep(first, first ? 0 : n_res));
    RCU(cudaMemcpyAsync(const_cast<int32_t*>(h_flags), ctx->d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCU(cudaStreamSynchronize(s));
    const int32_t flags = *h_flags;
    if (flags & 4) return fail(RAPTR_ERR_INVALID, "a channel id is outside [0, number of channels)");
    if (flags & 2) return fail(RAPTR_ERR_OVERFLOW, "ray walk did not terminate (internal error)");
    if (flags & 1) {
      // a row has more distinct voxels than the level's table: redo the
      // first iteration (nothing of it has been applied) a level up
      if (!first || level + 1 >= sm_num_levels())
        return fail(RAPTR_ERR_OVERFLOW, "a row has more distinct voxels than the largest per-row table holds");
      level++;
      it = -1;
      continue;
    }
    if (first && s64) RCU(launch_sens_normalise_self(N, s64, s32, s));
    if (first && d_s_out) RCU(cudaMemcpyAsync(d_s_out, s_use, size_t(N) * sizeof(float), cudaMemcpyDeviceToDevice, s));
    RCU(cudaMemsetAsync(acc, 0, sizeof(double), s));
    RCU(launch_mlem_update(N, d_x, c, s_use, acc, s));
    RCU(launch_mlem_normalise(N, d_x, c, acc, s));  // also clears c for the next iteration
    if (first) RCU(cudaEventRecord(ev[1], s));
  }
  RCU(cudaEventRecord(ev[2], s));
  RCU(cudaStreamSynchronize(s));
  if (stats) {
    float t01 = 0.f, t12 = 0.f;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    stats->resident_rows = n_res;
    stats->resident_entries = n_ent;
    stats->streamed_rows = n_list - n_res;
    stats->level = level;
    stats->first_iter_ms = t01;
    stats->iter_ms = n_iter > 1 ? t12 / double(n_iter - 1) : 0.0;
  }
  return RAPTR_OK;
}

raptr_status raptr_mlem_noalloc(int64_t m, int64_t n, const int64_t* d_row_ptr, const int32_t* d_col,
                                const float* d_val, const float* d_y, const float* d_s, float* d_x, int32_t n_iter,
                                void* stream) {
  std::string err;
  raptr_status st = mlem_noalloc(m, n, d_row_ptr, d_col, d_val, d_y, d_s, d_x, n_iter, as_stream(stream), &err);
  if (st != RAPTR_OK) return fail(st, err);
  return RAPTR_OK;
}

// ---- end-to-end -----------------------------------------------------------------------

raptr_status raptr_reco_host(const raptr_geom* geom, int device, const float* h_y, int32_t nrays, uint32_t seed,
                             int32_t n_iter, const float* h_sens, const float* h_x0, float* h_x,
                             raptr_reco_stats* stats) {
  if (!h_y || !h_x || nrays <= 0 || n_iter < 0) return fail(RAPTR_ERR_INVALID, "bad argument");
  const double t_call = trace_ms();
  trace("reco_host: start");
  raptr_ctx* ctx = nullptr;
  RCHECK(raptr_ctx_create(geom, device, &ctx));
  DeviceScope ds(device);
  const int64_t M = raptr_ctx_num_channels(ctx), N = raptr_ctx_num_voxels(ctx);
  cudaStream_t s;
  RCU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  // events: 0 start, 1 inputs on the device, 2 matrix built, 3 transpose
  // built, 4 sensitivity and start image ready, 5 iterations done, 6 image
  // on the host
  cudaEvent_t ev[7];
  for (auto& e : ev) cudaEventCreate(&e);
  const double t_setup = trace_ms();
  raptr_matrix* A = nullptr;
  float *d_y = nullptr, *d_x = nullptr, *d_s = nullptr;
  int32_t* d_list = nullptr;
  double* d_s64 = nullptr;
  raptr_status st = RAPTR_OK;
  auto cleanup = [&]() {
    raptr_matrix_destroy(A);
    dev_free(d_y);
    dev_free(d_x);
    dev_free(d_s);
    dev_free(d_list);
    dev_free(d_s64);
    for (auto& e : ev) cudaEventDestroy(e);
    cudaStreamDestroy(s);
    raptr_ctx_destroy(ctx);
  };
#define RSTEP(expr)                                         \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) {                                \
      st = cuda_fail(_e, #expr);                            \
      cleanup();                                            \
      return st;                                            \
    }                                                       \
  } while (0)
#define RSTATUS()                                           \
  do {                                                      \
    if (st != RAPTR_OK) {                                   \
      std::string msg = g_last_error;                       \
      cleanup();                                            \
      return fail(st, msg);                                 \
    }                                                       \
  } while (0)
  RSTEP(cudaEventRecord(ev[0], s));
  RSTEP(dev_malloc(&d_y, size_t(M) * sizeof(float)));
  RSTEP(dev_malloc(&d_x, size_t(N) * sizeof(float)));
  RSTEP(dev_malloc(&d_s, size_t(N) * sizeof(float)));
  RSTEP(dev_malloc(&d_list, size_t(M) * sizeof(int32_t)));
  RSTEP(cudaMemcpyAsync(d_y, h_y, size_t(M) * sizeof(float), cudaMemcpyHostToDevice, s));
  int64_t h2d = M * int64_t(sizeof(float));
  RSTEP(launch_iota(d_list, M, s));
  RSTEP(cudaEventRecord(ev[1], s));
  trace("reco_host: inputs on the device");
  st = raptr_sm_build_alloc(ctx, d_list, M, nrays, seed, nullptr, 0, &A, s);
  trace("reco_host: matrix built");
  RSTEP(cudaEventRecord(ev[2], s));
  if (st == RAPTR_OK) st = raptr_matrix_transpose(A, s);
  trace("reco_host: transpose built");
  RSTEP(cudaEventRecord(ev[3], s));
  // A matrix and transpose that do not fit the device: rebuild rows in every
  // iteration instead (raptr_mlem_stream), keeping as many as fit.
  const bool streamed = st == RAPTR_ERR_NOMEM;
  if (streamed) {
    raptr_matrix_destroy(A);
    A = nullptr;
    dev_release(device);
    trace("reco_host: the matrix does not fit: rows are rebuilt in every iteration");
  } else {
    RSTATUS();
  }
  if (!h_sens) {
    if (!streamed) {
      RSTEP(dev_malloc(&d_s64, size_t(N) * sizeof(double)));
      st = raptr_sensitivity_csc(N, A->cp, A->tval, d_s64, d_s, s);
      RSTATUS();
    }
  } else {
    RSTEP(cudaMemcpyAsync(d_s, h_sens, size_t(N) * sizeof(float), cudaMemcpyHostToDevice, s));
    h2d += N * int64_t(sizeof(float));
    // s /= sum(s) as src/tests/reco.cu:202-204
    RSTEP(launch_sum(d_s, N, ctx->d_f64, s));
    double sum = 0.0;
    RSTEP(cudaMemcpyAsync(&sum, ctx->d_f64, sizeof(double), cudaMemcpyDeviceToHost, s));
    RSTEP(cudaStreamSynchronize(s));
    RSTEP(launch_scales(d_s, float(1. / float(sum)), N, s));
  }
  if (h_x0) {
    RSTEP(cudaMemcpyAsync(d_x, h_x0, size_t(N) * sizeof(float), cudaMemcpyHostToDevice, s));
    h2d += N * int64_t(sizeof(float));
  } else {
    // Uniform image normalised to sum 1 (src/tests/reco.cu:145-158),
    // filled on the device
    RSTEP(launch_fill(d_x, float(1. / float(N)), N, s));
  }
  RSTEP(cudaEventRecord(ev[4], s));
  trace("reco_host: sensitivity");
  raptr_stream_stats sst{};
  if (streamed) {
    // what the library may still allocate, less the row staging (up to
    // 1 GiB, less when the room is small) and the working vectors
    const int64_t avail = int64_t(dev_available(device));
    const int64_t reserve = std::min<int64_t>(int64_t(1) << 30, avail / 2) + N * 24 + (int64_t(64) << 20);
    const int64_t resident = std::max<int64_t>(0, (avail - reserve) * 9 / 10);
    st = raptr_mlem_stream(ctx, d_list, M, nrays, seed, d_y, h_sens ? d_s : nullptr, nullptr, d_x, n_iter, resident,
                           &sst, s);
  } else {
    raptr_mlem_opts o{1, nullptr, nullptr, A->rank};
    st = raptr_mlem(ctx, A->m, N, A->rp, A->col, A->val, A->cp, A->trow, A->tval, d_y, d_s, d_x, n_iter, &o, s);
  }
  trace("reco_host: iterations enqueued");
  RSTATUS();
  RSTEP(cudaEventRecord(ev[5], s));
  RSTEP(cudaMemcpyAsync(h_x, d_x, size_t(N) * sizeof(float), cudaMemcpyDeviceToHost, s));
  RSTEP(cudaEventRecord(ev[6], s));
  RSTEP(cudaStreamSynchronize(s));
  const double t_image = trace_ms();
  const int64_t nnz = A ? A->nnz : sst.resident_entries;
  float t[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int i = 0; i < 6; i++) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
#undef RSTEP
#undef RSTATUS
  trace("reco_host: image on the host");
  cleanup();
  trace("reco_host: device memory released");
  if (stats) {
    stats->build_ms = t[1];
    stats->sens_ms = t[3];
    stats->iter_ms = t[4];
    stats->total_ms = t[0] + t[1] + t[2] + t[3] + t[4] + t[5];
    stats->nnz = nnz;
    stats->h2d_bytes = h2d;
    stats->d2h_bytes = N * int64_t(sizeof(float));
    stats->transpose_ms = t[2];
    stats->inputs_ms = t[0];
    stats->output_ms = t[5];
    stats->setup_ms = t_setup - t_call;
    stats->release_ms = trace_ms() - t_image;
    stats->wall_ms = trace_ms() - t_call;
    stats->streamed_rows = streamed ? sst.streamed_rows : 0;
  }
  return RAPTR_OK;
}

}  // extern "C"
