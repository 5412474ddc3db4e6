/*
 * Host-side harness around the reference's own templated code.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile from the reference
 * sources where they lie (REF_SRC), into oracle/_ref/.  Nothing of the
 * reference is copied here: this file only #includes its headers and
 * instantiates its templates on the host, so that the oracle restatement in
 * oracle/oracle.cpp can be checked against the reference's own arithmetic.
 *
 * Instantiated reference code (paths relative to the raptr source tree):
 *   getWorkqueue            src/getWorkqueue.hpp:149-243
 *   intersectionLength      src/getSystemMatrixDeviceOnly.cu:129-174
 *   Trafo*_inplace / Trafo* src/MeasurementSetupTrafo2CartCoord.hpp:85-466
 *   getChords               src/ChordsCalc_lowlevel.hpp:194-379
 *   index functors          src/VoxelGridLinIndex.hpp, src/MeasurementSetupLinIndex.hpp
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>
using std::max;
using std::min;

/* ChordsCalc_lowlevel.hpp calls its helper templates before defining them;
 * these declarations (signatures only) make the names visible to getChords. */
template <typename val_t> __host__ __device__ void getCrossesPlanes(bool[], val_t const[], val_t const[], val_t const[], int const[]);
template <typename val_t> __host__ __device__ val_t alphaFromId(int const, int const, val_t const[], val_t const[], val_t const[], int const[]);
template <typename val_t> __host__ __device__ val_t phiFromAlpha(val_t const, int const, val_t const[], val_t const[], val_t const[], int const[]);
template <typename val_t> __host__ __device__ void getAlphaDimmin(val_t[], val_t const[], val_t const[], val_t const[], int const[]);
template <typename val_t> __host__ __device__ void getAlphaDimmax(val_t[], val_t const[], val_t const[], val_t const[], int const[]);
template <typename val_t> __host__ __device__ void getAlphaMin(val_t*, bool*, val_t const[], bool const[]);
template <typename val_t> __host__ __device__ void getAlphaMax(val_t*, bool*, val_t const[], bool const[]);
template <typename val_t> __host__ __device__ val_t getLength(val_t const[]);
template <typename val_t> __host__ __device__ void getAlphaDimup(val_t[], val_t const[], val_t const[]);
template <typename val_t> __host__ __device__ void getIdDimup(int[], val_t const[]);

#include "typedefs.hpp"
#include "getWorkqueue.hpp"
#include "getSystemMatrixDeviceOnly.cu"

namespace {

VG make_grid(const float* go, const float* gd, const int32_t* gn) {
  return VG(go[0], go[1], go[2], gd[0], gd[1], gd[2], gn[0], gn[1], gn[2]);
}

MS make_setup(float pos0x, float pos1x, int32_t na, int32_t n0z, int32_t n0y, int32_t n1z, int32_t n1y, float da,
              float segx, float segy, float segz) {
  return MS(pos0x, pos1x, na, n0z, n0y, n1z, n1y, da, segx, segy, segz);
}

}  // namespace

extern "C" {

/* Reference struct layout shared with oracle.cpp (OGeom). */
struct RGeom {
  float grid_o[3];
  float grid_d[3];
  int32_t grid_n[3];
  float pos0x, pos1x;
  int32_t na, n0z, n0y, n1z, n1y;
  float da, segx, segy, segz;
};

int ref_abi_version(void) { return 1; }

/* getWorkqueue with a limit of n entries and a resumable cursor. */
int64_t ref_workqueue(const RGeom* g, const int32_t* list, int64_t nlist, int32_t* list_id, int32_t* vxl_id, int32_t n,
                      int32_t* out_cnl, int32_t* out_vxl) {
  VG grid = make_grid(g->grid_o, g->grid_d, g->grid_n);
  MS setup = make_setup(g->pos0x, g->pos1x, g->na, g->n0z, g->n0y, g->n1z, g->n1y, g->da, g->segx, g->segy, g->segz);
  ML ml(static_cast<int>(nlist));
  for (int64_t i = 0; i < nlist; i++) ml.set(int(i), list[i], 1.f);
  std::vector<int> c, v;
  int li = *list_id, vi = *vxl_id;
  int found = getWorkqueue<val_t, ML, VG, Idx, Idy, Idz, MS, Id0z, Id0y, Id1z, Id1y, Ida, Trafo0, Trafo1>(
      c, v, li, vi, &ml, &grid, &setup, n);
  for (int i = 0; i < found; i++) { out_cnl[i] = c[i]; out_vxl[i] = v[i]; }
  *list_id = li;
  *vxl_id = vi;
  return found;
}

float ref_intersection_length(const float* vxl_box, const float* ray) { return intersectionLength<float>(vxl_box, ray); }

/* Transforms unit-cube points into a crystal, in place (RandRayGen path,
 * src/RayGenerators.hpp:61-62) or out of place (getWorkqueue path). */
void ref_trafo(const RGeom* g, int32_t det, int32_t inplace, int32_t ida, int32_t idz, int32_t idy, const float* in,
               float* out) {
  MS setup = make_setup(g->pos0x, g->pos1x, g->na, g->n0z, g->n0y, g->n1z, g->n1y, g->da, g->segx, g->segy, g->segz);
  if (inplace) {
    float c[3] = {in[0], in[1], in[2]};
    if (det == 0) Trafo0_inplace()(c, idz, idy, ida, &setup);
    else Trafo1_inplace()(c, idz, idy, ida, &setup);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2];
  } else {
    if (det == 0) Trafo0()(out, in, idz, idy, ida, &setup);
    else Trafo1()(out, in, idz, idy, ida, &setup);
  }
}

void ref_channel_split(const RGeom* g, int32_t cnl, int32_t* out5) {
  MS setup = make_setup(g->pos0x, g->pos1x, g->na, g->n0z, g->n0y, g->n1z, g->n1y, g->da, g->segx, g->segy, g->segz);
  out5[0] = Ida()(cnl, &setup);
  out5[1] = Id0z()(cnl, &setup);
  out5[2] = Id0y()(cnl, &setup);
  out5[3] = Id1z()(cnl, &setup);
  out5[4] = Id1y()(cnl, &setup);
}

int32_t ref_channel_lin(const RGeom* g, int32_t id0z, int32_t id0y, int32_t id1z, int32_t id1y, int32_t ida) {
  MS setup = make_setup(g->pos0x, g->pos1x, g->na, g->n0z, g->n0y, g->n1z, g->n1y, g->da, g->segx, g->segy, g->segz);
  return DefaultMeasurementSetupLinId<MS>()(id0z, id0y, id1z, id1y, ida, &setup);
}

void ref_voxel_split(const RGeom* g, int32_t lin, int32_t* out3) {
  VG grid = make_grid(g->grid_o, g->grid_d, g->grid_n);
  out3[0] = Idx()(lin, &grid);
  out3[1] = Idy()(lin, &grid);
  out3[2] = Idz()(lin, &grid);
}

int32_t ref_voxel_lin(const RGeom* g, int32_t ix, int32_t iy, int32_t iz) {
  VG grid = make_grid(g->grid_o, g->grid_d, g->grid_n);
  return DefaultVoxelGridLinId<VG>()(ix, iy, iz, &grid);
}

/* The reference matrix algorithm on the CPU: candidates from getWorkqueue,
 * each value the mean over rays of intersectionLength
 * (src/getSystemMatrixDeviceOnly.cu:202-246).  Ray endpoints are made from
 * caller-supplied unit-cube coordinates (n_list * nrays * 6) with the
 * reference's in-place transforms, the way RandRayGen does
 * (src/RayGenerators.hpp:55-62).  Returns the number of entries; writes at
 * most cap of them. */
int64_t ref_sysmat(const RGeom* g, const int32_t* list, int64_t nlist, int32_t nrays, const float* unit_coords,
                   int64_t cap, int32_t* out_cnl, int32_t* out_vxl, float* out_val) {
  VG grid = make_grid(g->grid_o, g->grid_d, g->grid_n);
  MS setup = make_setup(g->pos0x, g->pos1x, g->na, g->n0z, g->n0y, g->n1z, g->n1y, g->da, g->segx, g->segy, g->segz);
  int64_t k = 0;
  std::vector<float> rays(size_t(nrays) * 6);
  for (int64_t li = 0; li < nlist; li++) {
    ML ml(1);
    ml.set(0, list[li], 1.f);
    std::vector<int> c, v;
    int l0 = 0, v0 = 0;
    getWorkqueue<val_t, ML, VG, Idx, Idy, Idz, MS, Id0z, Id0y, Id1z, Id1y, Ida, Trafo0, Trafo1>(c, v, l0, v0, &ml, &grid,
                                                                                                &setup);
    int cnl = list[li];
    int id0z = Id0z()(cnl, &setup), id0y = Id0y()(cnl, &setup), id1z = Id1z()(cnl, &setup),
        id1y = Id1y()(cnl, &setup), ida = Ida()(cnl, &setup);
    for (int r = 0; r < nrays; r++) {
      float* ray = &rays[size_t(r) * 6];
      const float* u = unit_coords + (li * int64_t(nrays) + r) * 6;
      for (int i = 0; i < 6; i++) ray[i] = u[i];
      Trafo0_inplace()(&ray[0], id0z, id0y, ida, &setup);
      Trafo1_inplace()(&ray[3], id1z, id1y, ida, &setup);
    }
    for (size_t e = 0; e < c.size(); e++) {
      int vxl = v[e];
      int sep[3] = {Idx()(vxl, &grid), Idy()(vxl, &grid), Idz()(vxl, &grid)};
      float box[6];
      box[0] = grid.gridox() + sep[0] * (grid.griddx());
      box[1] = grid.gridoy() + sep[1] * (grid.griddy());
      box[2] = grid.gridoz() + sep[2] * (grid.griddz());
      box[3] = grid.gridox() + (sep[0] + 1) * (grid.griddx());
      box[4] = grid.gridoy() + (sep[1] + 1) * (grid.griddy());
      box[5] = grid.gridoz() + (sep[2] + 1) * (grid.griddz());
      float a(0.);
      for (int r = 0; r < nrays; r++) a += intersectionLength(box, &rays[size_t(r) * 6]);
      a /= nrays;
      if (k < cap) { out_cnl[k] = c[e]; out_vxl[k] = vxl; out_val[k] = a; }
      k++;
    }
  }
  return k;
}

/* getChords for one ray; `cap` bounds the number of chords written, since
 * the reference does not bound it (src/ChordsCalc_lowlevel.hpp:314-378).
 * Returns the number of chords found. */
int64_t ref_get_chords(const float* ray, const float* gridO, const float* gridD, const int32_t* gridN, int64_t cap,
                       float* chords, int32_t* ids) {
  int64_t nmax = int64_t(gridN[0]) + gridN[1] + gridN[2] + 3;
  std::vector<float> ch(nmax, 0.f);
  std::vector<int> vid(3 * nmax, 0);
  int gn[3] = {gridN[0], gridN[1], gridN[2]};
  getChords<float>(ch.data(), vid.data(), int(nmax), ray, gridO, gridD, gn);
  int64_t n = 0;
  while (n < nmax && ch[n] != 0.f) n++;
  for (int64_t i = 0; i < n && i < cap; i++) {
    chords[i] = ch[i];
    ids[3 * i + 0] = vid[3 * i + 0];
    ids[3 * i + 1] = vid[3 * i + 1];
    ids[3 * i + 2] = vid[3 * i + 2];
  }
  return n;
}

}  // extern "C"
