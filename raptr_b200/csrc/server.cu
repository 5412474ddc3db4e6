// Serving loop: MLEM reconstructions of mixed geometry submitted at any
// time, run with continuous batching on one GPU.
//
// A worker thread owns the device work.  Each (geometry, rays, seed) gets a
// cached system matrix (FP16 form with its transpose, FP32 values dropped
// once converted), kept resident in least-recently-used order within an
// HBM byte budget.  Requests of one geometry that are admitted form one
// batch: their images and measurements live interleaved on the device
// (frame-minor, raptr_mlem_batch layout) and every scheduler step runs one
// MLEM iteration of every batch, each batch on its own stream so that the
// geometries' kernels overlap.  Requests join a batch and leave it between
// iterations (the batch is re-laid out then), each with its own iteration
// count; a finished image is copied to the host and the request's device
// memory is returned.  Admission is by memory: a request waits while its
// matrix plus the batch state would exceed the budget after evicting idle
// matrices.  Each geometry's batch advances as soon as its previous
// iteration ends (end events are polled), so a small geometry is not held
// to the pace of a large one.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/raptr_b200.h"
#include "internal.h"
#include "lru_budget.h"

namespace raptr {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// out[r*knew + s] = old[r*kold + src[s]], or init where src[s] < 0.
__global__ void frames_relayout_kernel(int64_t rows, int kold, const float* __restrict__ old_, int knew,
                                       const int* __restrict__ src, float init, float* __restrict__ out) {
  const int64_t total = rows * knew;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = i / knew;
    const int s = int(i - r * knew);
    const int so = src[s];
    out[i] = so >= 0 ? old_[r * kold + so] : init;
  }
}

// out[r*k + s] = vecs[s][r].
__global__ void frames_from_vectors_kernel(int64_t rows, int k, const float* const* __restrict__ vecs,
                                           float* __restrict__ out) {
  const int64_t total = rows * k;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = i / k;
    out[i] = vecs[i - r * k][r];
  }
}

__global__ void frame_extract_kernel(int64_t rows, int k, int s, const float* __restrict__ X,
                                     float* __restrict__ out) {
  for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += int64_t(gridDim.x) * blockDim.x)
    out[r] = X[r * k + s];
}

// Makes `device` current for the scope.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int device) {
    cudaGetDevice(&prev);
    cudaSetDevice(device);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

unsigned grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  return unsigned(std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8)));
}

std::string key_of(const raptr_geom& g, int32_t nrays, uint32_t seed) {
  std::string k(reinterpret_cast<const char*>(&g), sizeof(g));
  k.append(reinterpret_cast<const char*>(&nrays), sizeof(nrays));
  k.append(reinterpret_cast<const char*>(&seed), sizeof(seed));
  return k;
}

int64_t channels_of(const raptr_geom& g) {
  return int64_t(g.na) * g.n0z * g.n0y * g.n1z * g.n1y;
}

int64_t voxels_of(const raptr_geom& g) {
  return int64_t(g.grid_n[0]) * g.grid_n[1] * g.grid_n[2];
}

struct Request {
  int64_t id = 0;
  std::string key;
  raptr_geom g{};
  int32_t nrays = 0, n_iter = 0, done = 0;
  uint32_t seed = 0;
  std::vector<float> y_host;
  std::vector<float> x_host;
  float* y_dev = nullptr;
  int slot = -1;  // column in the batch's interleaved arrays
  int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
  raptr_status status = RAPTR_OK;
  std::string error;
  Clock::time_point t_submit, t_admit, t_done;
  int frames_max = 0;
  bool cold = false;
};

struct Entry {
  std::string key;
  raptr_geom g{};
  int32_t nrays = 0;
  uint32_t seed = 0;
  raptr_ctx* ctx = nullptr;
  raptr_matrix* A = nullptr;
  int64_t m = 0, n = 0, matrix_bytes = 0;
  int64_t* rp = nullptr;
  int32_t* col = nullptr;
  uint16_t* hval = nullptr;
  float* rscale = nullptr;
  int64_t* cp = nullptr;
  int32_t* trow = nullptr;
  uint16_t* htval = nullptr;
  int32_t* rank = nullptr;
  float* s = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<Request*> active;
  bool dirty = true;
  // the iteration on the device: its end event and the requests in it
  cudaEvent_t done_ev = nullptr;
  bool in_flight = false;
  raptr_status launch_status = RAPTR_OK;
  std::string launch_error;
  std::vector<Request*> members;
  // The batch's interleaved arrays, allocated for kcap frames and reused
  // while the batch changes (grown, never shrunk): images in two buffers
  // (a relayout reads one and writes the other), measurements in one (they
  // are rebuilt from the requests' own vectors), and the small index
  // arrays of a relayout, staged through page-locked host memory.
  float* Xbuf[2] = {nullptr, nullptr};
  int xcur = 0;
  float* Y = nullptr;
  float* tmp = nullptr;  // one image, for a finished request's copy to the host
  int* d_src = nullptr;
  const float** d_ys = nullptr;
  int* h_src = nullptr;
  const float** h_ys = nullptr;
  int K = 0, kcap = 0;
  float* X() const { return Xbuf[xcur]; }
  int64_t batch_bytes() const { return int64_t(kcap) * (2 * n + m) * int64_t(sizeof(float)); }
};

}  // namespace
}  // namespace raptr

struct raptr_server {
  int device = 0;
  raptr_server_opts opts{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::thread worker;
  int64_t next_id = 1;
  std::map<int64_t, std::unique_ptr<raptr::Request>> requests;
  std::deque<raptr::Request*> queue;
  std::map<std::string, std::unique_ptr<raptr::Entry>> entries;
  raptr::LruBudget<std::string> cache{0};
  int64_t state_bytes = 0;  // measurement vectors of running requests
  // the requests' measurement vectors come from this pool, which keeps
  // freed memory for the next request (the default pool hands it back to
  // the driver at each synchronisation, and mapping it again cost up to
  // hundreds of milliseconds of the scheduler's time); trimmed when a
  // matrix is dropped
  cudaMemPool_t pool = nullptr;
  raptr_server_stats st{};

  void loop();
  bool admit(std::unique_lock<std::mutex>& lk);
  raptr_status build(raptr::Entry* e, std::string* err);
  void drop(raptr::Entry* e);
  cudaError_t relayout(raptr::Entry* e);
  void fail_request(raptr::Request* r, raptr_status s, const std::string& msg) {
    r->state = 3;
    r->status = s;
    r->error = msg;
    r->t_done = raptr::Clock::now();
  }
};

namespace raptr {
namespace {

// Bytes a matrix is expected to take before it is built: the known size
// when it was built before, else ~750 entries per channel at 12 bytes
// (indices of the CSR and its transpose plus FP16 values of both).
int64_t estimate_bytes(const raptr_geom& g) { return channels_of(g) * 750 * 12 + voxels_of(g) * 16; }

}  // namespace
}  // namespace raptr

using namespace raptr;

raptr_status raptr_server::build(Entry* e, std::string* err) {
  DeviceScope ds(device);
  raptr_status st_ = raptr_ctx_create(&e->g, device, &e->ctx);
  if (st_ != RAPTR_OK) {
    *err = raptr_last_error();
    return st_;
  }
  // small geometries first when the device is shared: their iterations
  // are short, so they should not queue behind a large batch's blocks
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  cudaStreamCreateWithPriority(&e->stream, cudaStreamNonBlocking, channels_of(e->g) < (int64_t(1) << 20) ? hi : lo);
  cudaEventCreateWithFlags(&e->done_ev, cudaEventDisableTiming);
  int32_t* lst = nullptr;
  const int64_t nch = channels_of(e->g);
  cudaError_t ce = cudaMalloc(&lst, size_t(nch) * sizeof(int32_t));
  if (ce == cudaSuccess) ce = launch_iota(lst, nch, e->stream);
  if (ce != cudaSuccess) {
    cudaFree(lst);
    *err = cudaGetErrorString(ce);
    return RAPTR_ERR_CUDA;
  }
  st_ = raptr_sm_build_alloc(e->ctx, lst, nch, e->nrays, e->seed, nullptr, 0, &e->A, e->stream);
  cudaStreamSynchronize(e->stream);
  cudaFree(lst);
  if (st_ == RAPTR_OK) st_ = raptr_matrix_transpose(e->A, e->stream);
  if (st_ == RAPTR_OK) st_ = raptr_matrix_half(e->A, e->stream);
  if (st_ == RAPTR_OK && opts.keep_fp32 == 0) st_ = raptr_matrix_drop_f32(e->A);
  if (st_ != RAPTR_OK) {
    *err = raptr_last_error();
    return st_;
  }
  int64_t nnz = 0;
  float* val = nullptr;
  raptr_matrix_info(e->A, &e->m, &e->n, &nnz, &e->rp, &e->col, &val);
  float* tv = nullptr;
  raptr_matrix_csc_info(e->A, &e->cp, &e->trow, &tv);
  float* ps = nullptr;
  raptr_matrix_half_info(e->A, &e->hval, &e->rscale, &e->htval, &ps);
  int32_t* order = nullptr;
  raptr_matrix_row_order(e->A, &order, &e->rank);
  double* s64 = nullptr;
  ce = cudaMalloc(&s64, size_t(e->n) * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->s, size_t(e->n) * sizeof(float));
  if (ce != cudaSuccess) {
    cudaFree(s64);
    *err = cudaGetErrorString(ce);
    return RAPTR_ERR_NOMEM;
  }
  st_ = raptr_sensitivity_half(e->n, e->cp, e->trow, e->htval, ps, s64, e->s, e->stream);
  cudaStreamSynchronize(e->stream);
  cudaFree(s64);
  if (st_ != RAPTR_OK) {
    *err = raptr_last_error();
    return st_;
  }
  raptr_matrix_bytes(e->A, &e->matrix_bytes);
  e->matrix_bytes += e->n * int64_t(sizeof(float));
  this->st.builds++;
  return RAPTR_OK;
}

void raptr_server::drop(Entry* e) {
  DeviceScope ds(device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (pool) cudaMemPoolTrimTo(pool, 0);
  cudaFree(e->Xbuf[0]);
  cudaFree(e->Xbuf[1]);
  cudaFree(e->Y);
  cudaFree(e->tmp);
  cudaFree(e->d_src);
  cudaFree(e->d_ys);
  cudaFreeHost(e->h_src);
  cudaFreeHost(e->h_ys);
  e->Xbuf[0] = e->Xbuf[1] = e->tmp = nullptr;
  e->d_src = nullptr;
  e->d_ys = nullptr;
  e->h_src = nullptr;
  e->h_ys = nullptr;
  e->kcap = e->K = 0;
  cudaFree(e->s);
  if (e->A) raptr_matrix_destroy(e->A);
  if (e->ctx) raptr_ctx_destroy(e->ctx);
  if (e->stream) cudaStreamDestroy(e->stream);
  if (e->done_ev) cudaEventDestroy(e->done_ev);
  e->done_ev = nullptr;
  e->Y = e->s = nullptr;
  e->A = nullptr;
  e->ctx = nullptr;
  e->stream = nullptr;
}

// Lays the batch out again for its current requests: K = the smallest
// multiple of 4 that holds them (the batch kernels run any such K in tiles
// of at most 64 frames, so at most 3 slots are padding, which repeat slot
// 0).  The arrays are reused; only a batch that outgrows them allocates
// (the next power of two of frames, up to max_frames), so requests joining
// and leaving do not allocate or synchronise.
cudaError_t raptr_server::relayout(Entry* e) {
  const int cnt = int(e->active.size());
  const int K = std::max(4, (cnt + 3) & ~3);
  cudaError_t ce = cudaSuccess;
  if (!e->h_src) {
    ce = cudaMallocHost(&e->h_src, 64 * sizeof(int));
    if (ce == cudaSuccess) ce = cudaMallocHost(&e->h_ys, 64 * sizeof(float*));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->d_src, 64 * sizeof(int));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->d_ys, 64 * sizeof(float*));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->tmp, size_t(e->n) * sizeof(float));
    if (ce != cudaSuccess) return ce;
  }
  for (int s = 0; s < K; s++) {
    Request* r = e->active[size_t(s < cnt ? s : 0)];
    e->h_src[s] = (r->slot >= 0 && e->X()) ? r->slot : -1;
    e->h_ys[s] = r->y_dev;
  }
  float* from = e->X();
  float* to = e->Xbuf[1 - e->xcur];
  float* old_other = nullptr;
  float* old_cur = nullptr;
  if (K > e->kcap) {
    int kc = 4;
    while (kc < K) kc <<= 1;
    kc = std::min(kc, std::max(K, int(opts.max_frames + 3) & ~3));
    float *x0 = nullptr, *x1 = nullptr, *y = nullptr;
    ce = cudaMalloc(&x0, size_t(e->n) * kc * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMalloc(&x1, size_t(e->n) * kc * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMalloc(&y, size_t(std::max<int64_t>(e->m, 1)) * kc * sizeof(float));
    if (ce != cudaSuccess) {
      cudaFree(x0);
      cudaFree(x1);
      cudaFree(y);
      return ce;
    }
    old_cur = e->Xbuf[e->xcur];
    old_other = e->Xbuf[1 - e->xcur];
    cudaFree(e->Y);  // rebuilt from the requests' vectors below
    e->Xbuf[1 - e->xcur] = x0;
    e->Xbuf[e->xcur] = x1;
    e->Y = y;
    e->kcap = kc;
    to = x0;
  }
  ce = cudaMemcpyAsync(e->d_src, e->h_src, size_t(K) * sizeof(int), cudaMemcpyHostToDevice, e->stream);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(e->d_ys, e->h_ys, size_t(K) * sizeof(float*), cudaMemcpyHostToDevice, e->stream);
  if (ce == cudaSuccess) {
    frames_relayout_kernel<<<grid_of(e->n * K), 256, 0, e->stream>>>(e->n, e->K, from, K, e->d_src,
                                                                     float(1.0 / double(e->n)), to);
    frames_from_vectors_kernel<<<grid_of(e->m * K), 256, 0, e->stream>>>(e->m, K, e->d_ys, e->Y);
    note_launches(2);
    ce = cudaGetLastError();
  }
  if (old_cur || old_other) {
    // the relayout above read the old image buffer: free it after that
    cudaStreamSynchronize(e->stream);
    cudaFree(old_cur);
    cudaFree(old_other);
  }
  if (ce != cudaSuccess) return ce;
  e->xcur = (to == e->Xbuf[0]) ? 0 : 1;
  e->K = K;
  for (int s = 0; s < cnt; s++) {
    e->active[size_t(s)]->slot = s;
    e->active[size_t(s)]->frames_max = std::max(e->active[size_t(s)]->frames_max, cnt);
  }
  e->dirty = false;
  return cudaSuccess;
}

// Admits queued requests in order while memory allows; builds matrices
// (without the lock).  Returns whether anything changed.
bool raptr_server::admit(std::unique_lock<std::mutex>& lk) {
  bool changed = false;
  for (auto it = queue.begin(); it != queue.end();) {
    Request* r = *it;
    auto ei = entries.find(r->key);
    Entry* e = ei == entries.end() ? nullptr : ei->second.get();
    if (e && int(e->active.size()) >= opts.max_frames) {
      ++it;
      continue;
    }
    const int64_t state_need = voxels_of(r->g) * 4 + channels_of(r->g) * 4 * 3;  // y + batch growth
    if (!e) {
      const int64_t est = cache.contains(r->key) ? cache.bytes(r->key) : estimate_bytes(r->g);
      bool running = false;
      for (auto& kv : entries) running = running || !kv.second->active.empty();
      std::vector<std::string> victims;
      const Admission adm = decide_admission(cache, est + state_bytes + state_need, running, &victims);
      // wait for running work to finish; fail (evicting nothing) when the
      // request cannot fit even with nothing else resident
      if (adm == Admission::kWait) break;
      if (adm == Admission::kFail) {
        fail_request(r, RAPTR_ERR_NOMEM, "the matrix does not fit the HBM budget");
        it = queue.erase(it);
        cv_done.notify_all();
        changed = true;
        continue;
      }
      for (auto& v : victims) {
        auto vi = entries.find(v);
        if (vi != entries.end()) {
          drop(vi->second.get());
          entries.erase(vi);
          st.evictions++;
        }
        cache.erase(v);
      }
      auto ne = std::make_unique<Entry>();
      ne->key = r->key;
      ne->g = r->g;
      ne->nrays = r->nrays;
      ne->seed = r->seed;
      Entry* raw = ne.get();
      lk.unlock();
      std::string err;
      raptr_status bs = build(raw, &err);
      lk.lock();
      if (bs != RAPTR_OK) {
        drop(raw);
        fail_request(r, bs, "matrix build failed: " + err);
        it = queue.erase(it);
        cv_done.notify_all();
        changed = true;
        continue;
      }
      cache.put(r->key, raw->matrix_bytes);
      entries[r->key] = std::move(ne);
      e = raw;
      r->cold = true;
      // the queue may have changed while unlocked: restart the scan
      it = std::find(queue.begin(), queue.end(), r);
      if (it == queue.end()) break;
    }
    // measurement on the device (stream-ordered allocation: no device-wide
    // synchronisation while other batches run)
    DeviceScope ds(device);
    cudaError_t ce = pool ? cudaMallocFromPoolAsync(&r->y_dev, size_t(e->m) * sizeof(float), pool, e->stream)
                          : cudaMallocAsync(&r->y_dev, size_t(e->m) * sizeof(float), e->stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(r->y_dev, r->y_host.data(), size_t(e->m) * sizeof(float), cudaMemcpyHostToDevice,
                           e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) {
      (void)cudaGetLastError();
      if (r->y_dev) cudaFreeAsync(r->y_dev, e->stream);
      r->y_dev = nullptr;
      break;  // retry when memory frees up
    }
    std::vector<float>().swap(r->y_host);
    state_bytes += e->m * 4;
    r->state = 1;
    r->t_admit = Clock::now();
    e->active.push_back(r);
    e->dirty = true;
    cache.pin(r->key);
    cache.touch(r->key);
    it = queue.erase(it);
    changed = true;
  }
  return changed;
}

void raptr_server::loop() {
  DeviceScope ds(device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    auto busy = [&] {
      for (auto& kv : entries)
        if (!kv.second->active.empty() || kv.second->in_flight) return true;
      return false;
    };
    cv_work.wait(lk, [&] { return stop || !queue.empty() || busy(); });
    if (stop) break;
    admit(lk);
    // every batch advances on its own: start an iteration wherever the
    // device is idle for that geometry
    std::vector<Entry*> start;
    for (auto& kv : entries)
      if (!kv.second->in_flight && !kv.second->active.empty()) start.push_back(kv.second.get());
    for (Entry* e : start) {
      e->members = e->active;
      e->in_flight = true;
    }
    lk.unlock();
    for (Entry* e : start) {
      e->launch_status = RAPTR_OK;
      if (e->dirty && relayout(e) != cudaSuccess) {
        e->launch_status = RAPTR_ERR_NOMEM;
        e->launch_error = "batch relayout failed";
      } else {
        // all frames in sweeps of at most 64 (a multiple of 4 frames): one
        // 64-frame sweep takes 112 ms at 70^3, two of 32 take 120 ms
        e->launch_status = raptr_mlem_batch(e->ctx, e->m, e->n, e->K, 1, e->rp, e->col, e->hval, e->rscale, e->cp,
                                            e->trow, e->htval, e->rank, e->Y, e->s, e->X(), 1, 64, nullptr,
                                            e->stream);
        if (e->launch_status != RAPTR_OK) e->launch_error = raptr_last_error();
      }
      cudaEventRecord(e->done_ev, e->stream);
    }
    // collect iterations that have ended; finished images to the host
    std::vector<Entry*> ended;
    std::vector<std::vector<std::pair<Request*, std::vector<float>>>> finished;
    {
      std::vector<Entry*> flying;
      lk.lock();
      for (auto& kv : entries)
        if (kv.second->in_flight) flying.push_back(kv.second.get());
      lk.unlock();
      for (Entry* e : flying) {
        if (cudaEventQuery(e->done_ev) != cudaSuccess) continue;
        ended.push_back(e);
        finished.emplace_back();
        if (e->launch_status != RAPTR_OK) continue;
        for (Request* r : e->members) {
          if (r->done + 1 < r->n_iter) continue;
          std::vector<float> x(size_t(e->n));
          frame_extract_kernel<<<grid_of(e->n), 256, 0, e->stream>>>(e->n, e->K, r->slot, e->X(), e->tmp);
          note_launches(1);
          cudaMemcpyAsync(x.data(), e->tmp, size_t(e->n) * sizeof(float), cudaMemcpyDeviceToHost, e->stream);
          cudaStreamSynchronize(e->stream);
          finished.back().emplace_back(r, std::move(x));
        }
      }
    }
    if (ended.empty()) {
      // nothing ended yet: give the device a moment
      std::this_thread::sleep_for(std::chrono::microseconds(200));
      lk.lock();
      continue;
    }
    lk.lock();
    for (size_t i = 0; i < ended.size(); i++) {
      Entry* e = ended[i];
      e->in_flight = false;
      if (e->launch_status != RAPTR_OK) {
        for (Request* r : e->members) {
          if (r->state != 1) continue;
          cudaFreeAsync(r->y_dev, e->stream);
          r->y_dev = nullptr;
          state_bytes -= e->m * 4;
          cache.unpin(r->key);
          fail_request(r, e->launch_status, e->launch_error);
        }
      } else {
        st.iterations += int64_t(e->members.size());
        st.batch_steps++;
        for (Request* r : e->members) r->done++;
        for (auto& f : finished[i]) {
          Request* r = f.first;
          r->x_host = std::move(f.second);
          r->state = 2;
          r->t_done = Clock::now();
          cudaFreeAsync(r->y_dev, e->stream);
          r->y_dev = nullptr;
          state_bytes -= e->m * 4;
          cache.unpin(r->key);
          st.completed++;
        }
      }
      e->members.clear();
      const size_t before = e->active.size();
      e->active.erase(std::remove_if(e->active.begin(), e->active.end(), [](Request* r) { return r->state != 1; }),
                      e->active.end());
      if (e->active.size() != before) e->dirty = true;
      cache.put(e->key, e->matrix_bytes + e->batch_bytes());
    }
    cv_done.notify_all();
  }
}

extern "C" {

raptr_status raptr_server_create(int32_t device, const raptr_server_opts* opts, raptr_server** out) {
  if (!out || !opts || opts->hbm_budget_bytes <= 0 || opts->max_frames < 1 || opts->max_frames > 64)
    return set_error(RAPTR_ERR_INVALID, "bad server options");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return set_error(RAPTR_ERR_CUDA, "no such device");
  raptr_server* s = new raptr_server;
  s->device = device;
  s->opts = *opts;
  s->cache = LruBudget<std::string>(opts->hbm_budget_bytes);
  {
    DeviceScope ds(device);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&s->pool, &props) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
      (void)cudaGetLastError();
      s->pool = nullptr;  // the default pool then
    }
  }
  s->worker = std::thread([s] { s->loop(); });
  *out = s;
  return RAPTR_OK;
}

raptr_status raptr_server_destroy(raptr_server* s) {
  if (!s) return RAPTR_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->worker.join();
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto& kv : s->requests) {
    Request* r = kv.second.get();
    if (r->state < 2) s->fail_request(r, RAPTR_ERR_INVALID, "server destroyed");
    cudaFree(r->y_dev);
  }
  for (auto& kv : s->entries) s->drop(kv.second.get());
  if (s->pool) {
    DeviceScope ds(s->device);
    cudaDeviceSynchronize();
    cudaMemPoolDestroy(s->pool);
  }
  s->cv_done.notify_all();
  delete s;
  return RAPTR_OK;
}

raptr_status raptr_server_submit(raptr_server* s, const raptr_geom* g, int32_t nrays, uint32_t seed,
                                 const float* h_y, int32_t n_iter, int64_t* request_id) {
  if (!s || !g || !h_y || !request_id || nrays <= 0 || n_iter <= 0) return set_error(RAPTR_ERR_INVALID, "bad argument");
  auto r = std::make_unique<Request>();
  r->g = *g;
  r->nrays = nrays;
  r->seed = seed;
  r->n_iter = n_iter;
  r->key = key_of(*g, nrays, seed);
  const int64_t m = channels_of(*g);
  if (m <= 0 || voxels_of(*g) <= 0) return set_error(RAPTR_ERR_INVALID, "empty geometry");
  r->y_host.assign(h_y, h_y + m);
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  r->id = s->next_id++;
  *request_id = r->id;
  s->queue.push_back(r.get());
  s->requests[r->id] = std::move(r);
  s->st.submitted++;
  s->cv_work.notify_all();
  return RAPTR_OK;
}

raptr_status raptr_server_wait(raptr_server* s, int64_t request_id, float* h_x, int32_t timeout_ms,
                               raptr_request_stats* stats) {
  if (!s) return RAPTR_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(request_id);
  if (it == s->requests.end()) return set_error(RAPTR_ERR_INVALID, "unknown request (already collected?)");
  Request* r = it->second.get();
  auto ready = [&] { return r->state >= 2; };
  if (timeout_ms < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return set_error(RAPTR_ERR_TIMEOUT, "request not finished");
  raptr_status st_ = r->state == 2 ? RAPTR_OK : r->status;
  if (st_ != RAPTR_OK) set_error(st_, r->error);
  if (stats) {
    stats->queue_ms = r->state == 2 ? ms_between(r->t_submit, r->t_admit) : 0.0;
    stats->run_ms = r->state == 2 ? ms_between(r->t_admit, r->t_done) : 0.0;
    stats->total_ms = ms_between(r->t_submit, r->t_done);
    stats->iterations = r->done;
    stats->frames_max = r->frames_max;
    stats->cold_build = r->cold ? 1 : 0;
  }
  if (st_ == RAPTR_OK && h_x) std::memcpy(h_x, r->x_host.data(), r->x_host.size() * sizeof(float));
  s->requests.erase(it);
  return st_;
}

raptr_status raptr_server_get_stats(raptr_server* s, raptr_server_stats* out) {
  if (!s || !out) return RAPTR_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident_matrices = int64_t(s->entries.size());
  out->resident_bytes = s->cache.used() + s->state_bytes;
  out->queued = int64_t(s->queue.size());
  int64_t running = 0;
  for (auto& kv : s->entries) running += int64_t(kv.second->active.size());
  out->running = running;
  return RAPTR_OK;
}

}  // extern "C"
