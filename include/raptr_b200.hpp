/*
 * raptr_b200.hpp -- the reference's C++ template API over the raptr_b200 C ABI.
 *
 * Host-side, header-only.  Code written against raptr's trait classes and
 * wrapper functions compiles against this header instead and runs on the
 * B200 kernels of libraptr_b200.so:
 *
 *   trait classes (same names, constructors and accessors)
 *     VoxelGrid / DefaultVoxelGrid                   src/VoxelGrid.hpp:37-263
 *     DefaultVoxelGridLinId, DefaultVoxelGridIdx/y/z src/VoxelGridLinIndex.hpp:69-221
 *     MeasurementSetup / DefaultMeasurementSetup     src/MeasurementSetup.hpp:36-351
 *     DefaultMeasurementSetupLinId, ...Id0z/Id0y/Id1z/Id1y/Ida
 *                                                    src/MeasurementSetupLinIndex.hpp:78-320
 *     DefaultMeasurementSetupTrafo2CartCoord{First,Secnd}Pixel[_inplace]
 *                                                    src/MeasurementSetupTrafo2CartCoord.hpp:85-466
 *     DefaultMeasurementList                         src/MeasurementList.hpp:66-128
 *     WritableGrid, WritableGridTraits, GridAdapter  src/H5DensityWriter.hpp:40-89, src/GridAdapter.hpp:39-65
 *   functions (same signatures)
 *     getWorkqueue (both overloads)                  src/getWorkqueue.hpp:149-243
 *     systemMatrixCalculation                        src/wrappers.hpp:185-266
 *     CSRmv<float>                                   src/csrmv.hpp:72-83
 *     convertCoo2Csr, convertCsr2Ecsr                src/cusparseWrapper.hpp:53-60, src/convertCsr2Ecsr.hpp:51-64
 *     divides, dividesMultiplies, scales, sum        src/mlemOperations.hpp:44-169
 *
 * The reference passes the geometry to its kernels through __constant__
 * memory set with cudaMemcpyToSymbol (src/tests/reco.cu:84-93); here
 * raptr::set_device_constants(grid, setup, nrays) plays that part for the
 * functions above.  Failures throw raptr::Exception (the reference throws
 * cudaException or exits).
 */
#ifndef RAPTR_B200_HPP
#define RAPTR_B200_HPP

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "raptr_b200.h"
#include "raptr_b200_h5.h"

#ifndef RAPTR_HD
#if defined(__CUDACC__)
#define RAPTR_HD __host__ __device__
#else
#define RAPTR_HD
#endif
#endif

namespace raptr {

class Exception : public std::runtime_error {
 public:
  explicit Exception(const std::string& what) : std::runtime_error(what) {}
};

inline void check(raptr_status s, const char* what) {
  if (s != RAPTR_OK) throw Exception(std::string(what) + ": " + raptr_last_error());
}

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Exception(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace raptr

/* ------------------------------------------------------------------------ */
/* Voxel grid                                                                */
/* ------------------------------------------------------------------------ */

template <typename T, typename ConcreteVoxelGrid>
class VoxelGrid {
 public:
  RAPTR_HD T gridox() const { return static_cast<const ConcreteVoxelGrid*>(this)->gridox(); }
  RAPTR_HD T gridoy() const { return static_cast<const ConcreteVoxelGrid*>(this)->gridoy(); }
  RAPTR_HD T gridoz() const { return static_cast<const ConcreteVoxelGrid*>(this)->gridoz(); }
  RAPTR_HD T griddx() const { return static_cast<const ConcreteVoxelGrid*>(this)->griddx(); }
  RAPTR_HD T griddy() const { return static_cast<const ConcreteVoxelGrid*>(this)->griddy(); }
  RAPTR_HD T griddz() const { return static_cast<const ConcreteVoxelGrid*>(this)->griddz(); }
  RAPTR_HD int gridnx() const { return static_cast<const ConcreteVoxelGrid*>(this)->gridnx(); }
  RAPTR_HD int gridny() const { return static_cast<const ConcreteVoxelGrid*>(this)->gridny(); }
  RAPTR_HD int gridnz() const { return static_cast<const ConcreteVoxelGrid*>(this)->gridnz(); }
};

template <typename T>
class DefaultVoxelGrid : public VoxelGrid<T, DefaultVoxelGrid<T> > {
  T o_[3];
  T d_[3];
  int n_[3];

 public:
  RAPTR_HD DefaultVoxelGrid() {}
  RAPTR_HD DefaultVoxelGrid(T const gridO0, T const gridO1, T const gridO2, T const gridD0, T const gridD1,
                            T const gridD2, int const gridN0, int const gridN1, int const gridN2) {
    o_[0] = gridO0; o_[1] = gridO1; o_[2] = gridO2;
    d_[0] = gridD0; d_[1] = gridD1; d_[2] = gridD2;
    n_[0] = gridN0; n_[1] = gridN1; n_[2] = gridN2;
  }
  RAPTR_HD T gridox() const { return o_[0]; }
  RAPTR_HD T gridoy() const { return o_[1]; }
  RAPTR_HD T gridoz() const { return o_[2]; }
  RAPTR_HD T griddx() const { return d_[0]; }
  RAPTR_HD T griddy() const { return d_[1]; }
  RAPTR_HD T griddz() const { return d_[2]; }
  RAPTR_HD int gridnx() const { return n_[0]; }
  RAPTR_HD int gridny() const { return n_[1]; }
  RAPTR_HD int gridnz() const { return n_[2]; }
};

/* Linear voxel id, x slowest and z fastest (src/VoxelGridLinIndex.hpp:74-80). */
template <typename ConcreteVG>
struct DefaultVoxelGridLinId {
  RAPTR_HD int operator()(int const idx, int const idy, int const idz, ConcreteVG const* const vg) const {
    return idx * (vg->gridnz() * vg->gridny()) + idy * vg->gridnz() + idz;
  }
};
template <typename ConcreteVG>
struct DefaultVoxelGridIdx {
  RAPTR_HD int operator()(int const linId, ConcreteVG const* const vg) const {
    return linId / (vg->gridnz() * vg->gridny());
  }
};
template <typename ConcreteVG>
struct DefaultVoxelGridIdy {
  RAPTR_HD int operator()(int const linId, ConcreteVG const* const vg) const {
    return (linId % (vg->gridnz() * vg->gridny())) / vg->gridnz();
  }
};
template <typename ConcreteVG>
struct DefaultVoxelGridIdz {
  RAPTR_HD int operator()(int const linId, ConcreteVG const* const vg) const {
    return (linId % (vg->gridnz() * vg->gridny())) % vg->gridnz();
  }
};

/* ------------------------------------------------------------------------ */
/* Measurement setup                                                         */
/* ------------------------------------------------------------------------ */

template <typename T, typename ConcreteMeasurementSetup>
class MeasurementSetup {
 public:
  RAPTR_HD T pos0x() const { return self().pos0x(); }
  RAPTR_HD T pos1x() const { return self().pos1x(); }
  RAPTR_HD int na() const { return self().na(); }
  RAPTR_HD int n0z() const { return self().n0z(); }
  RAPTR_HD int n0y() const { return self().n0y(); }
  RAPTR_HD int n1z() const { return self().n1z(); }
  RAPTR_HD int n1y() const { return self().n1y(); }
  RAPTR_HD T da() const { return self().da(); }
  RAPTR_HD T segx() const { return self().segx(); }
  RAPTR_HD T segy() const { return self().segy(); }
  RAPTR_HD T segz() const { return self().segz(); }

 private:
  RAPTR_HD const ConcreteMeasurementSetup& self() const { return *static_cast<const ConcreteMeasurementSetup*>(this); }
};

template <typename T>
class DefaultMeasurementSetup : public MeasurementSetup<T, DefaultMeasurementSetup<T> > {
  T pos0x_, pos1x_;
  int na_;
  T da_;
  int n0z_, n0y_, n1z_, n1y_;
  T segx_, segy_, segz_;

 public:
  DefaultMeasurementSetup() {}
  /* Argument order of src/MeasurementSetup.hpp:214-220. */
  DefaultMeasurementSetup(T pos0x, T pos1x, int na, int n0z, int n0y, int n1z, int n1y, T da, T segx, T segy, T segz)
      : pos0x_(pos0x), pos1x_(pos1x), na_(na), da_(da), n0z_(n0z), n0y_(n0y), n1z_(n1z), n1y_(n1y), segx_(segx),
        segy_(segy), segz_(segz) {}
  RAPTR_HD T pos0x() const { return pos0x_; }
  RAPTR_HD T pos1x() const { return pos1x_; }
  RAPTR_HD int na() const { return na_; }
  RAPTR_HD T da() const { return da_; }
  RAPTR_HD int n0z() const { return n0z_; }
  RAPTR_HD int n0y() const { return n0y_; }
  RAPTR_HD int n1z() const { return n1z_; }
  RAPTR_HD int n1y() const { return n1y_; }
  RAPTR_HD T segx() const { return segx_; }
  RAPTR_HD T segy() const { return segy_; }
  RAPTR_HD T segz() const { return segz_; }
};

/* Channel id (ida, id0z, id0y, id1z, id1y), id1y fastest
 * (src/MeasurementSetupLinIndex.hpp:82-91 and inverses). */
template <typename MS>
struct DefaultMeasurementSetupLinId {
  RAPTR_HD int operator()(int const id0z, int const id0y, int const id1z, int const id1y, int const ida,
                          MS const* const m) const {
    return (((ida * m->n0z() + id0z) * m->n0y() + id0y) * m->n1z() + id1z) * m->n1y() + id1y;
  }
};
template <typename MS>
struct DefaultMeasurementSetupIda {
  RAPTR_HD int operator()(int const linId, MS const* const m) const {
    return linId / (m->n1y() * m->n1z() * m->n0y() * m->n0z());
  }
};
template <typename MS>
struct DefaultMeasurementSetupId0z {
  RAPTR_HD int operator()(int const linId, MS const* const m) const {
    return (linId % (m->n1y() * m->n1z() * m->n0y() * m->n0z())) / (m->n1y() * m->n1z() * m->n0y());
  }
};
template <typename MS>
struct DefaultMeasurementSetupId0y {
  RAPTR_HD int operator()(int const linId, MS const* const m) const {
    return (linId % (m->n1y() * m->n1z() * m->n0y())) / (m->n1y() * m->n1z());
  }
};
template <typename MS>
struct DefaultMeasurementSetupId1z {
  RAPTR_HD int operator()(int const linId, MS const* const m) const {
    return (linId % (m->n1y() * m->n1z())) / m->n1y();
  }
};
template <typename MS>
struct DefaultMeasurementSetupId1y {
  RAPTR_HD int operator()(int const linId, MS const* const m) const { return linId % m->n1y(); }
};

/* ------------------------------------------------------------------------ */
/* Crystal -> Cartesian transforms                                           */
/* ------------------------------------------------------------------------ */

namespace raptr {
namespace detail {

/* 3x4 affine map of a crystal: scale by the segment edges, move into the
 * crystal, rotate about y by ida*da degrees; the float expression of the
 * angle and the operation order are those of
 * src/MeasurementSetupTrafo2CartCoord.hpp:99-147. */
template <typename T>
inline void crystal_map(T m[12], T posx, int idz, int idy, int ny, int nz, T segx, T segy, T segz, int ida, T da) {
  T edges[3] = {segx, segy, segz};
  T pos[3];
  pos[0] = posx;
  pos[1] = (idy - T(.5) * (ny - 1)) * edges[1];
  pos[2] = (idz - T(.5) * (nz - 1)) * edges[2];
  T s = sinf(T(M_PI) * ida * da / T(180.0));
  T c = cosf(T(M_PI) * ida * da / T(180.0));
  m[0] = c * edges[0];
  m[1] = T(0.);
  m[2] = s * edges[2];
  m[3] = c * (pos[0] - T(.5) * edges[0]) + s * (pos[2] - T(.5) * edges[2]);
  m[4] = T(0.);
  m[5] = edges[1];
  m[6] = T(0.);
  m[7] = pos[1] - T(.5) * edges[1];
  m[8] = -s * edges[0];
  m[9] = T(0.);
  m[10] = c * edges[2];
  m[11] = -s * (pos[0] - T(.5) * edges[0]) + c * (pos[2] - T(.5) * edges[2]);
}

template <typename T>
inline void apply_map(const T m[12], const T in[3], T out[3]) {
  T t[3] = {in[0], in[1], in[2]};
  for (int r = 0; r < 3; r++)
    out[r] = m[4 * r + 0] * t[0] + m[4 * r + 1] * t[1] + m[4 * r + 2] * t[2] + m[4 * r + 3] * T(1.);
}

}  // namespace detail
}  // namespace raptr

template <typename T, typename MS>
class DefaultMeasurementSetupTrafo2CartCoordFirstPixel {
 public:
  void operator()(T* const cart, T const* const box, int const id0z, int const id0y, int const ida,
                  MS const* const m) const {
    T mat[12];
    raptr::detail::crystal_map<T>(mat, m->pos0x(), id0z, id0y, m->n0y(), m->n0z(), m->segx(), m->segy(), m->segz(),
                                  ida, m->da());
    raptr::detail::apply_map<T>(mat, box, cart);
  }
};

template <typename T, typename MS>
class DefaultMeasurementSetupTrafo2CartCoordSecndPixel {
 public:
  void operator()(T* const cart, T const* const box, int const id1z, int const id1y, int const ida,
                  MS const* const m) const {
    T mat[12];
    raptr::detail::crystal_map<T>(mat, m->pos1x(), id1z, id1y, m->n1y(), m->n1z(), m->segx(), m->segy(), m->segz(),
                                  ida, m->da());
    raptr::detail::apply_map<T>(mat, box, cart);
  }
};

template <typename T, typename MS>
class DefaultMeasurementSetupTrafo2CartCoordFirstPixel_inplace {
 public:
  void operator()(T* const coords, int const id0z, int const id0y, int const ida, MS const* const m) const {
    T in[3] = {coords[0], coords[1], coords[2]};
    DefaultMeasurementSetupTrafo2CartCoordFirstPixel<T, MS>()(coords, in, id0z, id0y, ida, m);
  }
};

template <typename T, typename MS>
class DefaultMeasurementSetupTrafo2CartCoordSecndPixel_inplace {
 public:
  void operator()(T* const coords, int const id1z, int const id1y, int const ida, MS const* const m) const {
    T in[3] = {coords[0], coords[1], coords[2]};
    DefaultMeasurementSetupTrafo2CartCoordSecndPixel<T, MS>()(coords, in, id1z, id1y, ida, m);
  }
};

/* ------------------------------------------------------------------------ */
/* Measurement list and writable grid                                        */
/* ------------------------------------------------------------------------ */

template <typename T, typename ConcreteMeasurementList>
class MeasurementList {
 public:
  int cnlId(int const listId) const { return static_cast<const ConcreteMeasurementList*>(this)->cnlId(listId); }
  T val(int const listId) const { return static_cast<const ConcreteMeasurementList*>(this)->val(listId); }
};

template <typename T>
class DefaultMeasurementList : public MeasurementList<T, DefaultMeasurementList<T> > {
  std::vector<int> cnl_;
  std::vector<T> val_;

 public:
  explicit DefaultMeasurementList(int const size) : cnl_(size_t(size), 0), val_(size_t(size), T(0)) {}
  int cnlId(int const listId) const { return cnl_[size_t(listId)]; }
  T val(int const listId) const { return val_[size_t(listId)]; }
  int size() const { return int(cnl_.size()); }
  void set(int const listId, int const cnlId, T const val) {
    if (listId < 0 || listId >= size()) throw raptr::Exception("DefaultMeasurementList::set: listId out of bounds");
    cnl_[size_t(listId)] = cnlId;
    val_[size_t(listId)] = val;
  }
  const int* data() const { return cnl_.data(); }
};

template <typename T>
struct WritableGridTraits {
  typedef T CoordType;
};

template <typename ConcreteWritableGrid, typename ConcreteWritableGridTraits>
class WritableGrid {
 public:
  typedef typename ConcreteWritableGridTraits::CoordType CoordType;
  void getOrigin(CoordType* const origin) const { static_cast<const ConcreteWritableGrid*>(this)->getOrigin(origin); }
  void getVoxelSize(CoordType* const s) const { static_cast<const ConcreteWritableGrid*>(this)->getVoxelSize(s); }
  void getNumberOfVoxels(int* const n) const { static_cast<const ConcreteWritableGrid*>(this)->getNumberOfVoxels(n); }
};

template <typename TVoxelGrid, typename T>
class GridAdapter : public WritableGrid<GridAdapter<TVoxelGrid, T>, WritableGridTraits<T> > {
  TVoxelGrid const* const grid_;

 public:
  explicit GridAdapter(TVoxelGrid const* const grid) : grid_(grid) {}
  void getOrigin(T* const o) const { o[0] = grid_->gridox(); o[1] = grid_->gridoy(); o[2] = grid_->gridoz(); }
  void getVoxelSize(T* const d) const { d[0] = grid_->griddx(); d[1] = grid_->griddy(); d[2] = grid_->griddz(); }
  void getNumberOfVoxels(int* const n) const { n[0] = grid_->gridnx(); n[1] = grid_->gridny(); n[2] = grid_->gridnz(); }
};

/* ------------------------------------------------------------------------ */
/* Geometry hand-over and the device constants of the reference              */
/* ------------------------------------------------------------------------ */

namespace raptr {

template <typename VG, typename MS>
inline raptr_geom make_geom(VG const& g, MS const& s) {
  raptr_geom r;
  r.grid_o[0] = float(g.gridox()); r.grid_o[1] = float(g.gridoy()); r.grid_o[2] = float(g.gridoz());
  r.grid_d[0] = float(g.griddx()); r.grid_d[1] = float(g.griddy()); r.grid_d[2] = float(g.griddz());
  r.grid_n[0] = g.gridnx(); r.grid_n[1] = g.gridny(); r.grid_n[2] = g.gridnz();
  r.pos0x = float(s.pos0x()); r.pos1x = float(s.pos1x());
  r.na = s.na(); r.n0z = s.n0z(); r.n0y = s.n0y(); r.n1z = s.n1z(); r.n1y = s.n1y();
  r.da = float(s.da()); r.segx = float(s.segx()); r.segy = float(s.segy()); r.segz = float(s.segz());
  return r;
}

/* Per-thread state that stands for the reference's __constant__ grid_const,
 * setup_const and nrays_const (src/device_constant_memory.hpp:34-46). */
struct DeviceConstants {
  raptr_geom geom{};
  int nrays = 0;
  uint32_t seed = 1251;
  int device = 0;
  int32_t sm_flags = 0; /* raptr_sm_build flags of systemMatrixCalculation */
  std::shared_ptr<raptr_ctx> ctx;
};

inline DeviceConstants& device_constants() {
  static thread_local DeviceConstants c;
  return c;
}

/* The counterpart of the three cudaMemcpyToSymbol calls of
 * src/tests/reco.cu:84-93. */
template <typename VG, typename MS>
inline void set_device_constants(VG const& grid, MS const& setup, int nrays, uint32_t seed = 1251) {
  DeviceConstants& c = device_constants();
  c.geom = make_geom(grid, setup);
  c.nrays = nrays;
  c.seed = seed;
  check_cuda(cudaGetDevice(&c.device), "cudaGetDevice");
  raptr_ctx* ctx = nullptr;
  check(raptr_ctx_create(&c.geom, c.device, &ctx), "raptr_ctx_create");
  c.ctx = std::shared_ptr<raptr_ctx>(ctx, [](raptr_ctx* p) { raptr_ctx_destroy(p); });
}

/* Flags for the builds of systemMatrixCalculation on this thread:
 * RAPTR_SM_KEEP_ZEROS keeps every candidate of a row, exact zeros included,
 * which is the reference's structure; the default (0) drops exact zeros. */
inline void set_sm_flags(int32_t flags) { device_constants().sm_flags = flags; }

inline raptr_ctx* current_ctx() {
  DeviceConstants& c = device_constants();
  if (!c.ctx) throw Exception("raptr::set_device_constants(grid, setup, nrays) has not been called");
  return c.ctx.get();
}

/* Scoped device buffer for the shims' temporaries. */
template <typename T>
struct DeviceBuffer {
  T* p = nullptr;
  explicit DeviceBuffer(size_t n) { check_cuda(cudaMalloc(&p, (n ? n : 1) * sizeof(T)), "cudaMalloc"); }
  ~DeviceBuffer() { cudaFree(p); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

}  // namespace raptr

/* ------------------------------------------------------------------------ */
/* Wrapper functions with the reference's signatures                         */
/* ------------------------------------------------------------------------ */

/* Candidate search with the resumable cursor (listId, vxlId), at most n
 * entries (src/getWorkqueue.hpp:149-191). */
template <typename T, typename ConcreteList, typename ConcreteVG, typename ConcreteVGidx, typename ConcreteVGidy,
          typename ConcreteVGidz, typename ConcreteMS, typename ConcreteMSid0z, typename ConcreteMSid0y,
          typename ConcreteMSid1z, typename ConcreteMSid1y, typename ConcreteMSida,
          typename ConcreteMSTrafo2CartCoordFirstPixel, typename ConcreteMSTrafo2CartCoordSecndPixel>
int getWorkqueue(std::vector<int>& returnCnlId, std::vector<int>& returnVxlId, int& listId, int& vxlId,
                 ConcreteList const* const list, ConcreteVG const* const grid, ConcreteMS const* const setup,
                 int const n) {
  if (!returnCnlId.empty() || !returnVxlId.empty()) throw raptr::Exception("getWorkqueue: return vector not empty!");
  if (n <= 0) return 0;
  raptr_geom g = raptr::make_geom(*grid, *setup);
  int dev = 0;
  raptr::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  raptr_ctx* ctx = nullptr;
  raptr::check(raptr_ctx_create(&g, dev, &ctx), "raptr_ctx_create");
  std::unique_ptr<raptr_ctx, raptr_status (*)(raptr_ctx*)> guard(ctx, raptr_ctx_destroy);
  const int nl = list->size();
  std::vector<int> h_list(size_t(nl > 0 ? nl : 1));
  for (int i = 0; i < nl; i++) h_list[size_t(i)] = list->cnlId(i);
  raptr::DeviceBuffer<int32_t> d_list(static_cast<size_t>(nl)), d_c(static_cast<size_t>(n)),
      d_v(static_cast<size_t>(n));
  raptr::check_cuda(cudaMemcpy(d_list.p, h_list.data(), size_t(nl) * sizeof(int32_t), cudaMemcpyHostToDevice),
                    "cudaMemcpy");
  int64_t li = listId, vi = vxlId, found = 0;
  raptr::check(raptr_workqueue(ctx, d_list.p, nl, &li, &vi, n, d_c.p, d_v.p, &found, nullptr), "raptr_workqueue");
  returnCnlId.resize(size_t(found));
  returnVxlId.resize(size_t(found));
  if (found > 0) {
    raptr::check_cuda(cudaMemcpy(returnCnlId.data(), d_c.p, size_t(found) * sizeof(int), cudaMemcpyDeviceToHost),
                      "cudaMemcpy");
    raptr::check_cuda(cudaMemcpy(returnVxlId.data(), d_v.p, size_t(found) * sizeof(int), cudaMemcpyDeviceToHost),
                      "cudaMemcpy");
  }
  listId = int(li);
  vxlId = int(vi);
  return int(found);
}

/* Unlimited search (src/getWorkqueue.hpp:207-243). */
template <typename T, typename ConcreteList, typename ConcreteVG, typename ConcreteVGidx, typename ConcreteVGidy,
          typename ConcreteVGidz, typename ConcreteMS, typename ConcreteMSid0z, typename ConcreteMSid0y,
          typename ConcreteMSid1z, typename ConcreteMSid1y, typename ConcreteMSida,
          typename ConcreteMSTrafo2CartCoordFirstPixel, typename ConcreteMSTrafo2CartCoordSecndPixel>
int getWorkqueue(std::vector<int>& returnCnlId, std::vector<int>& returnVxlId, int& listId, int& vxlId,
                 ConcreteList const* const list, ConcreteVG const* const grid, ConcreteMS const* const setup) {
  const int nvox = grid->gridnx() * grid->gridny() * grid->gridnz();
  const int bound = int(std::min<long long>((long long)(list->size()) * nvox, 2147483647LL));
  return getWorkqueue<T, ConcreteList, ConcreteVG, ConcreteVGidx, ConcreteVGidy, ConcreteVGidz, ConcreteMS,
                      ConcreteMSid0z, ConcreteMSid0y, ConcreteMSid1z, ConcreteMSid1y, ConcreteMSida,
                      ConcreteMSTrafo2CartCoordFirstPixel, ConcreteMSTrafo2CartCoordSecndPixel>(
      returnCnlId, returnVxlId, listId, vxlId, list, grid, setup, bound);
}

/* System matrix rows of the channels yRowId_devi[0 .. *nY_host) as ECSR
 * (src/wrappers.hpp:185-266): aEcsrCnlPtr_devi (int row pointers),
 * aVxlId_devi and aVal_devi (buffers of the reference's dense bound, rows x
 * voxels); *nnz_devi is increased by the number of entries.  The COO row
 * ids and the CSR over all channels are internal to the reference's
 * pipeline and are not produced (aCnlId_devi, aCsrCnlPtr_devi untouched).
 * Geometry and ray count come from raptr::set_device_constants.  Exact
 * zeros are dropped unless raptr::set_sm_flags(RAPTR_SM_KEEP_ZEROS) was
 * called: then every candidate is kept, as the reference stores them. */
template <typename T, typename ListSizeType, typename GridSizeType, typename MemArrSizeType, typename RayGen,
          typename Handle>
void systemMatrixCalculation(int* const aEcsrCnlPtr_devi, GridSizeType* const aVxlId_devi, T* const aVal_devi,
                             MemArrSizeType* const nnz_devi, int* const aCnlId_devi, int* const aCsrCnlPtr_devi,
                             int* const yRowId_devi, ListSizeType const* const& nY_host, Handle const& handle) {
  static_assert(std::is_same<T, float>::value, "values are float");
  static_assert(sizeof(GridSizeType) == 4, "voxel ids are 32-bit");
  (void)aCnlId_devi;
  (void)aCsrCnlPtr_devi;
  (void)handle;
  raptr::DeviceConstants& c = raptr::device_constants();
  raptr_ctx* ctx = raptr::current_ctx();
  const int64_t m = int64_t(*nY_host);
  const int64_t nvox = int64_t(c.geom.grid_n[0]) * c.geom.grid_n[1] * c.geom.grid_n[2];
  raptr::DeviceBuffer<int64_t> rp(size_t(m + 1));
  int64_t nnz = 0;
  raptr::check(raptr_sm_build(ctx, yRowId_devi, m, c.nrays, c.seed, nullptr, c.sm_flags, m * nvox, rp.p,
                              reinterpret_cast<int32_t*>(aVxlId_devi), aVal_devi, &nnz, nullptr),
               "raptr_sm_build");
  raptr::check(raptr_row_ptr_narrow(rp.p, m + 1, aEcsrCnlPtr_devi, nullptr), "raptr_row_ptr_narrow");
  MemArrSizeType cur = 0;
  raptr::check_cuda(cudaMemcpy(&cur, nnz_devi, sizeof(MemArrSizeType), cudaMemcpyDeviceToHost), "cudaMemcpy");
  cur += MemArrSizeType(nnz);
  raptr::check_cuda(cudaMemcpy(nnz_devi, &cur, sizeof(MemArrSizeType), cudaMemcpyHostToDevice), "cudaMemcpy");
}

/* y = alpha*op(A)*x + beta*y on an int-row-pointer CSR (src/csrmv.hpp:61-83);
 * transA 0 = non-transposed, 1 = transposed (the cusparseOperation_t values). */
template <typename T>
struct CSRmv;

template <>
struct CSRmv<float> {
  template <typename Handle, typename Op, typename Descr>
  void operator()(Handle handle, Op transA, int m, int n, int nnz, float* const alpha, Descr descrA,
                  float* const csrValA, int* const csrRowPtrA, int* const csrColIdA, float* const x,
                  float* const beta, float* const y) const {
    (void)handle;
    (void)descrA;
    (void)nnz;
    raptr::DeviceBuffer<int64_t> rp(size_t(m) + 1);
    raptr::check(raptr_row_ptr_widen(csrRowPtrA, int64_t(m) + 1, rp.p, nullptr), "raptr_row_ptr_widen");
    raptr::check(raptr_spmv(int32_t(transA), m, n, rp.p, csrColIdA, csrValA, *alpha, x, *beta, y, nullptr),
                 "raptr_spmv");
  }
};

/* Row pointers of all m rows from sorted COO row ids (src/cusparseWrapper.hpp:53-60). */
template <typename Handle>
int convertCoo2Csr(int* const csrRowPtr, int const* const cooRowId, Handle const& handle, int const nnz, int const m) {
  (void)handle;
  raptr::DeviceBuffer<int64_t> rp(size_t(m) + 1);
  raptr::check(raptr_coo2csr(cooRowId, nnz, m, rp.p, nullptr), "raptr_coo2csr");
  raptr::check(raptr_row_ptr_narrow(rp.p, int64_t(m) + 1, csrRowPtr, nullptr), "raptr_row_ptr_narrow");
  return 0;
}

/* ECSR from CSR (src/convertCsr2Ecsr.hpp:51-64). */
inline void convertCsr2Ecsr(int* const ecsrRowPtr, int* const yRowId, int const nnzr, int* const csrRowPtr,
                            int const m) {
  raptr::DeviceBuffer<int64_t> csr(size_t(m) + 1), ecsr(size_t(nnzr) + 1);
  raptr::check(raptr_row_ptr_widen(csrRowPtr, int64_t(m) + 1, csr.p, nullptr), "raptr_row_ptr_widen");
  raptr::check(raptr_csr2ecsr(ecsr.p, yRowId, nnzr, csr.p, m, nullptr), "raptr_csr2ecsr");
  raptr::check(raptr_row_ptr_narrow(ecsr.p, int64_t(nnzr) + 1, ecsrRowPtr, nullptr), "raptr_row_ptr_narrow");
}

/* Element-wise MLEM operations (src/mlemOperations.hpp:44-169). */
template <typename T>
void divides(T* const& result, T* const& dividend, T* const& divisor, int const n) {
  static_assert(std::is_same<T, float>::value, "float only");
  raptr::check(raptr_divides(result, dividend, divisor, n, nullptr), "raptr_divides");
}

template <typename T>
void dividesMultiplies(T* const& result, T* const& a, T* const& b, T* const& c, int const n) {
  static_assert(std::is_same<T, float>::value, "float only");
  raptr::check(raptr_divides_multiplies(result, a, b, c, n, nullptr), "raptr_divides_multiplies");
}

template <typename T>
void scales(T* const& x, T const alpha, int const n) {
  static_assert(std::is_same<T, float>::value, "float only");
  raptr::check(raptr_scales(x, alpha, n, nullptr), "raptr_scales");
}

template <typename T>
T sum(T* const& x, int const n) {
  static_assert(std::is_same<T, float>::value, "float only");
  double s = 0.0;
  raptr::check(raptr_sum(x, n, &s, nullptr), "raptr_sum");
  return T(s);
}

/* ------------------------------------------------------------------------ */
/* HDF5 measurement and density files (src/H5Reader.hpp:34-102,               */
/* src/H5DensityWriter.hpp:97-232, src/wrappers.hpp:330-482) over             */
/* raptr_b200_h5.h                                                            */
/* ------------------------------------------------------------------------ */

namespace raptr {
inline void check_h5(int st, const std::string& what) {
  if (st != RAPTR_H5_OK) throw Exception(what + ": " + raptr_h5_last_error());
}

inline std::vector<float> read_dataset(std::string const& fn, const char* name) {
  int64_t count = 0;
  check_h5(raptr_h5_read_f32(fn.c_str(), name, nullptr, 0, &count), "read " + fn);
  std::vector<float> v(static_cast<size_t>(count));
  check_h5(raptr_h5_read_f32(fn.c_str(), name, v.data(), count, &count), "read " + fn);
  return v;
}
}  // namespace raptr

/* Reads the "messung" dataset of a measurement file (H5Reader::read). */
class H5Reader {
  std::string fn_;

 public:
  typedef float Value_t;
  explicit H5Reader(std::string const& fn) : fn_(fn) {}
  bool is_open() const {
    int32_t rank = 0;
    return raptr_h5_dataset_info(fn_.c_str(), "messung", &rank, nullptr) == RAPTR_H5_OK;
  }
  int sizeOfFile() const {
    int64_t count = 0;
    raptr::check_h5(raptr_h5_read_f32(fn_.c_str(), "messung", nullptr, 0, &count), "read " + fn_);
    return int(count);
  }
  void read(Value_t* mem) const {
    std::vector<float> v = raptr::read_dataset(fn_, "messung");
    std::copy(v.begin(), v.end(), mem);
  }
};

/* Writes the "density" dataset with the grid attributes. */
template <typename TGrid>
class H5DensityWriter {
  std::string fn_;

 public:
  explicit H5DensityWriter(std::string const& fn) : fn_(fn) {}
  void write(float const* mem, TGrid const& grid) const {
    typename TGrid::CoordType o[3], d[3];
    int n[3];
    grid.getOrigin(o);
    grid.getVoxelSize(d);
    grid.getNumberOfVoxels(n);
    float lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
      lo[k] = static_cast<float>(o[k]);
      hi[k] = lo[k] + n[k] * static_cast<float>(d[k]);
    }
    const int32_t nn[3] = {n[0], n[1], n[2]};
    raptr::check_h5(raptr_h5_write_density(fn_.c_str(), mem, nn, lo, hi), "write " + fn_);
  }
};

/* Nonzero counts of a measurement file as a sparse vector (channel ids in
 * ascending order, values). */
template <typename T>
void readHDF5_MeasVct(std::vector<int>& vctId, std::vector<T>& vctVal, int& vctNnz, std::string const& ifn) {
  std::vector<float> y = raptr::read_dataset(ifn, "messung");
  vctId.clear();
  vctVal.clear();
  for (size_t i = 0; i < y.size(); i++)
    if (y[i] != 0.f) {
      vctId.push_back(int(i));
      vctVal.push_back(T(y[i]));
    }
  vctNnz = int(vctId.size());
}

/* The measured channels of a measurement file (measurement list). */
template <typename T>
void readHDF5_MeasList(std::vector<int>& ml, int& mlN, std::string const& ifn) {
  std::vector<T> v;
  readHDF5_MeasVct(ml, v, mlN, ifn);
}

/* The density of a density file, x slowest. */
template <typename T>
std::vector<T> readHDF5_Density(std::string const& ifn) {
  std::vector<float> d = raptr::read_dataset(ifn, "density");
  return std::vector<T>(d.begin(), d.end());
}

template <typename T>
void writeHDF5_Density(T const* const density, std::string const ofn, DefaultVoxelGrid<T> const& grid) {
  static_assert(std::is_same<T, float>::value, "float only");
  GridAdapter<DefaultVoxelGrid<T>, T> ga(&grid);
  H5DensityWriter<GridAdapter<DefaultVoxelGrid<T>, T> >(ofn).write(density, ga);
}

#endif /* RAPTR_B200_HPP */
