// Shared pieces of the command-line drivers (reco, backprojection,
// pureSMCalculation): geometry from the input files and the environment,
// timing, device buffers.
//
// The reference compiles its geometry in (src/real_measurementsetup_defines.h,
// src/voxelgrid_defines.h).  These drivers read it at run time instead:
//   detector segments and angles: the shape of the measurement's "messung"
//     dataset (angles, z0, y0, z1, y1);
//   the remaining setup (RAPTR_SETUP="pos0x,pos1x,da,segx,segy,segz", metres
//     and degrees), by default the reference's compiled-in values;
//   the voxel grid: the attributes of a density file when the driver reads
//     one (reco: the sensitivity), else RAPTR_GRID="nx,ny,nz,ox,oy,oz,dx,dy,dz";
//   rays: Philox keyed by (RAPTR_SEED, default 1251, channel).
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>
#include <vector>

#include "raptr_b200.hpp"

namespace drv {

inline std::vector<double> env_list(const char* name) {
  std::vector<double> v;
  const char* s = std::getenv(name);
  if (!s) return v;
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ',')) v.push_back(std::atof(tok.c_str()));
  return v;
}

inline uint32_t seed() {
  const char* s = std::getenv("RAPTR_SEED");
  return s ? uint32_t(std::strtoul(s, nullptr, 10)) : 1251u;
}

// Setup from the measurement file's dims and RAPTR_SETUP.
inline void setup_from(const std::string& meas, raptr_geom* g) {
  int32_t rank = 0;
  int64_t d[8] = {0};
  raptr::check_h5(raptr_h5_dataset_info(meas.c_str(), "messung", &rank, d), "read " + meas);
  if (rank != 5) throw raptr::Exception(meas + ": \"messung\" must have 5 dimensions");
  g->na = int32_t(d[0]);
  g->n0z = int32_t(d[1]);
  g->n0y = int32_t(d[2]);
  g->n1z = int32_t(d[3]);
  g->n1y = int32_t(d[4]);
  std::vector<double> s = env_list("RAPTR_SETUP");
  if (!s.empty() && s.size() != 6) throw raptr::Exception("RAPTR_SETUP needs pos0x,pos1x,da,segx,segy,segz");
  if (s.empty()) s = {-0.457, 0.457, 2.0, 0.020, 0.004, 0.004};
  g->pos0x = float(s[0]);
  g->pos1x = float(s[1]);
  g->da = float(s[2]);
  g->segx = float(s[3]);
  g->segy = float(s[4]);
  g->segz = float(s[5]);
}

// Grid from a density file's attributes.
inline void grid_from_density(const std::string& fn, raptr_geom* g) {
  int32_t n[3];
  float lo[3], hi[3];
  raptr::check_h5(raptr_h5_read_density_grid(fn.c_str(), n, lo, hi), "read " + fn);
  for (int k = 0; k < 3; k++) {
    g->grid_n[k] = n[k];
    g->grid_o[k] = lo[k];
    g->grid_d[k] = (hi[k] - lo[k]) / float(n[k]);
  }
}

// Grid from RAPTR_GRID.
inline void grid_from_env(raptr_geom* g) {
  std::vector<double> v = env_list("RAPTR_GRID");
  if (v.size() != 9) throw raptr::Exception("set RAPTR_GRID=nx,ny,nz,ox,oy,oz,dx,dy,dz (metres)");
  for (int k = 0; k < 3; k++) {
    g->grid_n[k] = int32_t(v[size_t(k)]);
    g->grid_o[k] = float(v[size_t(3 + k)]);
    g->grid_d[k] = float(v[size_t(6 + k)]);
  }
}

inline DefaultVoxelGrid<float> voxel_grid(const raptr_geom& g) {
  return DefaultVoxelGrid<float>(g.grid_o[0], g.grid_o[1], g.grid_o[2], g.grid_d[0], g.grid_d[1], g.grid_d[2],
                                 g.grid_n[0], g.grid_n[1], g.grid_n[2]);
}

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

// The measured channels' rows of the system matrix (ECSR of the reference).
struct Rows {
  raptr_ctx* ctx = nullptr;
  raptr_matrix* A = nullptr;
  int64_t m = 0, n = 0, nnz = 0;
  ~Rows() {
    if (A) raptr_matrix_destroy(A);
    if (ctx) raptr_ctx_destroy(ctx);
  }
};

inline void build_rows(const raptr_geom& g, const std::vector<int>& channels, int nrays, Rows* r) {
  raptr::check(raptr_ctx_create(&g, 0, &r->ctx), "raptr_ctx_create");
  raptr::DeviceBuffer<int32_t> d(channels.size());
  raptr::check_cuda(cudaMemcpy(d.p, channels.data(), channels.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
                    "cudaMemcpy");
  raptr::check(raptr_sm_build_alloc(r->ctx, d.p, int64_t(channels.size()), nrays, seed(), nullptr, 0, &r->A, nullptr),
               "raptr_sm_build_alloc");
  int64_t* rp;
  int32_t* col;
  float* val;
  raptr::check(raptr_matrix_info(r->A, &r->m, &r->n, &r->nnz, &rp, &col, &val), "raptr_matrix_info");
}

inline int usage(const char* const* lines, int nargs, int argc) {
  std::fprintf(stderr, "Error: Wrong number of arguments (got %d). Expected %d:\n", argc - 1, nargs);
  for (int i = 0; i < nargs; i++) std::fprintf(stderr, "  %s\n", lines[i]);
  return EXIT_FAILURE;
}

}  // namespace drv
