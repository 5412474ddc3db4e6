/*
 * CPU oracle for the raptr reconstruction hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain C++ restatement of the
 * reference algorithm (ComputationalRadiationPhysics/raptr) used as the
 * checker for the CUDA library.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it.  The product library never links,
 * loads or calls anything in oracle/.
 *
 * Every float operation below is written in the order the reference writes
 * it and the file is compiled with -ffp-contract=off, so that for identical
 * inputs the results are bit-identical to the reference's float arithmetic.
 *
 * Reference files cited as path:line relative to the raptr source tree.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

/* Same field order and meaning as DefaultVoxelGrid (src/VoxelGrid.hpp:151-176)
 * and DefaultMeasurementSetup (src/MeasurementSetup.hpp:181-220). */
struct OGeom {
  float   grid_o[3];
  float   grid_d[3];
  int32_t grid_n[3];
  float   pos0x, pos1x;
  int32_t na, n0z, n0y, n1z, n1y;
  float   da, segx, segy, segz;
};

}  // extern "C"

namespace {

/* ------------------------------------------------------------------------ */
/* Index maps                                                                */
/* ------------------------------------------------------------------------ */

/* Voxel linear id, x slowest, z fastest: src/VoxelGridLinIndex.hpp:74-80,
 * inverse :121-125 (x), :166-172 (y), :213-220 (z). */
inline void voxel_split(const OGeom& g, int64_t lin, int ids[3]) {
  int64_t nyz = int64_t(g.grid_n[1]) * g.grid_n[2];
  ids[0] = int(lin / nyz);
  int64_t r = lin % nyz;
  ids[1] = int(r / g.grid_n[2]);
  ids[2] = int(r % g.grid_n[2]);
}

/* Channel linear id (ida, id0z, id0y, id1z, id1y), id1y fastest:
 * src/MeasurementSetupLinIndex.hpp:82-91, inverses :129-133, :172-178,
 * :217-224, :263-271, :310-319. */
struct ChannelIds { int ida, id0z, id0y, id1z, id1y; };

inline ChannelIds channel_split(const OGeom& g, int64_t cnl) {
  ChannelIds c;
  int64_t s4 = int64_t(g.n1y) * g.n1z * g.n0y * g.n0z;
  int64_t s3 = int64_t(g.n1y) * g.n1z * g.n0y;
  int64_t s2 = int64_t(g.n1y) * g.n1z;
  int64_t s1 = g.n1y;
  c.ida = int(cnl / s4);
  int64_t t = cnl % s4;
  c.id0z = int(t / s3);
  t %= s3;
  c.id0y = int(t / s2);
  t %= s2;
  c.id1z = int(t / s1);
  c.id1y = int(t % s1);
  return c;
}

/* ------------------------------------------------------------------------ */
/* Crystal -> Cartesian transform                                            */
/* ------------------------------------------------------------------------ */

/* Per-angle sine/cosine, computed exactly as the reference computes the
 * argument: sinf(T(M_PI)*ida*da/T(180.0)) evaluated left to right in float.
 * src/MeasurementSetupTrafo2CartCoord.hpp:110-111 (and :215-216, :321-322,
 * :426-427). */
inline void angle_sincos(float da, int ida, float* s, float* c) {
  volatile float pi = float(M_PI);
  float arg = pi * float(ida);
  arg = arg * da;
  arg = arg / 180.0f;
  *s = sinf(arg);
  *c = cosf(arg);
}

/* The 3x4 affine map of src/MeasurementSetupTrafo2CartCoord.hpp:99-131:
 * scale by the segment edges, translate into the crystal box, rotate about y. */
template <typename T>
void trafo_matrix(T m[12], T posx, int idz, int idy, int ny, int nz, T segx,
                  T segy, T segz, T sin_, T cos_) {
  T edges[3] = {segx, segy, segz};
  T pos[3];
  pos[0] = posx;
  pos[1] = (idy - T(.5) * (ny - 1)) * edges[1];
  pos[2] = (idz - T(.5) * (nz - 1)) * edges[2];
  m[0 * 4 + 0] = cos_ * edges[0];
  m[0 * 4 + 1] = T(0.);
  m[0 * 4 + 2] = sin_ * edges[2];
  m[0 * 4 + 3] = cos_ * (pos[0] - T(.5) * edges[0]) + sin_ * (pos[2] - T(.5) * edges[2]);
  m[1 * 4 + 0] = T(0.);
  m[1 * 4 + 1] = edges[1];
  m[1 * 4 + 2] = T(0.);
  m[1 * 4 + 3] = pos[1] - T(.5) * edges[1];
  m[2 * 4 + 0] = -sin_ * edges[0];
  m[2 * 4 + 1] = T(0.);
  m[2 * 4 + 2] = cos_ * edges[2];
  m[2 * 4 + 3] = -sin_ * (pos[0] - T(.5) * edges[0]) + cos_ * (pos[2] - T(.5) * edges[2]);
}

/* Application of the matrix: src/MeasurementSetupTrafo2CartCoord.hpp:134-147. */
template <typename T>
void trafo_apply(const T m[12], const T in[3], T out[3]) {
  T tmp[3] = {in[0], in[1], in[2]};
  out[0] = m[0 * 4 + 0] * tmp[0] + m[0 * 4 + 1] * tmp[1] + m[0 * 4 + 2] * tmp[2] + m[0 * 4 + 3] * T(1.);
  out[1] = m[1 * 4 + 0] * tmp[0] + m[1 * 4 + 1] * tmp[1] + m[1 * 4 + 2] * tmp[2] + m[1 * 4 + 3] * T(1.);
  out[2] = m[2 * 4 + 0] * tmp[0] + m[2 * 4 + 1] * tmp[1] + m[2 * 4 + 2] * tmp[2] + m[2 * 4 + 3] * T(1.);
}

struct ChannelTrafo {
  float m0[12];  // first detector pixel
  float m1[12];  // second detector pixel
};

inline ChannelTrafo channel_trafo(const OGeom& g, const ChannelIds& c) {
  float s, co;
  angle_sincos(g.da, c.ida, &s, &co);
  ChannelTrafo t;
  trafo_matrix<float>(t.m0, g.pos0x, c.id0z, c.id0y, g.n0y, g.n0z, g.segx, g.segy, g.segz, s, co);
  trafo_matrix<float>(t.m1, g.pos1x, c.id1z, c.id1y, g.n1y, g.n1z, g.segx, g.segy, g.segz, s, co);
  return t;
}

/* ------------------------------------------------------------------------ */
/* Candidate test (enclosing cylinder)                                       */
/* ------------------------------------------------------------------------ */

/* src/distancePointLine.h:40-43 */
inline float absolute3(const float a[3]) { return sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

/* src/distancePointLine.h:67-72, :89-101 */
inline float distance_point_line(const float a[3], const float b[3], const float p[3]) {
  float ap[3], ab[3], c[3];
  for (int d = 0; d < 3; d++) {
    ap[d] = p[d] - a[d];
    ab[d] = b[d] - a[d];
  }
  for (int d = 0; d < 3; d++) c[d] = ab[(d + 1) % 3] * ap[(d + 2) % 3] - ab[(d + 2) % 3] * ap[(d + 1) % 3];
  return absolute3(c) / absolute3(ab);
}

struct ChannelLine {
  float c0[3], c1[3];  // crystal centres
  float sum_radii;
};

/* Crystal centres and sum of radii: src/getWorkqueue.hpp:70-89,
 * src/getSystemMatrixDeviceOnly.cu:95-104. */
inline ChannelLine channel_line(const OGeom& g, const ChannelTrafo& t) {
  ChannelLine l;
  float centre[3] = {0.5f, 0.5f, 0.5f};
  trafo_apply<float>(t.m0, centre, l.c0);
  trafo_apply<float>(t.m1, centre, l.c1);
  float ve[3] = {g.grid_d[0], g.grid_d[1], g.grid_d[2]};
  float pe[3] = {g.segx, g.segy, g.segz};
  l.sum_radii = 0.5f * (absolute3(ve) + absolute3(pe));
  return l;
}

/* src/getWorkqueue.hpp:91-98, src/getSystemMatrixDeviceOnly.cu:106-116 */
inline bool candidate_test(const OGeom& g, const ChannelLine& l, int ix, int iy, int iz) {
  float v[3];
  v[0] = g.grid_o[0] + (ix + 0.5f) * g.grid_d[0];
  v[1] = g.grid_o[1] + (iy + 0.5f) * g.grid_d[1];
  v[2] = g.grid_o[2] + (iz + 0.5f) * g.grid_d[2];
  return distance_point_line(l.c0, l.c1, v) < l.sum_radii;
}

/* Conservative z-index interval of voxel centres of row (ix, iy) that can
 * pass the cylinder test.  Used only to prune the scan; every voxel in the
 * interval is still decided by candidate_test, and the interval is widened
 * so that it always contains every passing voxel. */
inline bool row_z_interval(const OGeom& g, const ChannelLine& l, int ix, int iy, int* z0, int* z1) {
  double a[3] = {l.c0[0], l.c0[1], l.c0[2]};
  double u[3] = {double(l.c1[0]) - a[0], double(l.c1[1]) - a[1], double(l.c1[2]) - a[2]};
  double nu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  for (int d = 0; d < 3; d++) u[d] /= nu;
  double R = double(l.sum_radii) * 1.01 + 1e-3 * double(g.grid_d[0] + g.grid_d[1] + g.grid_d[2]);
  double dx = g.grid_o[0] + (ix + 0.5) * g.grid_d[0] - a[0];
  double dy = g.grid_o[1] + (iy + 0.5) * g.grid_d[1] - a[1];
  double w = dx * u[0] + dy * u[1];
  double a2 = 1.0 - u[2] * u[2];
  double c0 = dx * dx + dy * dy - w * w - R * R;
  int nz = g.grid_n[2];
  if (a2 < 1e-9) {
    if (c0 < 0) { *z0 = 0; *z1 = nz - 1; return true; }
    return false;
  }
  double b1 = -2.0 * u[2] * w;
  double disc = b1 * b1 - 4.0 * a2 * c0;
  if (disc < 0) return false;
  double sq = std::sqrt(disc);
  double zlo = a[2] + (-b1 - sq) / (2 * a2);
  double zhi = a[2] + (-b1 + sq) / (2 * a2);
  double flo = (zlo - g.grid_o[2]) / g.grid_d[2] - 0.5;
  double fhi = (zhi - g.grid_o[2]) / g.grid_d[2] - 0.5;
  if (fhi < -3.0 || flo > nz + 2.0) return false;
  long lo = long(std::floor(flo)) - 2;
  long hi = long(std::ceil(fhi)) + 2;
  if (lo < 0) lo = 0;
  if (hi > nz - 1) hi = nz - 1;
  if (lo > hi) return false;
  *z0 = int(lo);
  *z1 = int(hi);
  return true;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as   */
/* easy as 1, 2, 3", SC'11).  Rays are keyed by (seed, channel) and counted  */
/* by (ray, half).                                                           */
/* ------------------------------------------------------------------------ */

inline void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = uint64_t(0xD2511F53u) * c0;
    uint64_t p1 = uint64_t(0xCD9E8D57u) * c2;
    uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
    uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 24 random bits -> float in (0, 1], exactly representable. */
inline float u01(uint32_t x) { return float((x >> 8) + 1u) * (1.0f / 16777216.0f); }

/* Six uniforms of ray `ray` of channel `cnl`: words 0-3 of block 0 and
 * words 0-1 of block 1. */
inline void ray_uniforms(uint32_t seed, int64_t cnl, int64_t ray, float u[6]) {
  uint32_t key[2] = {seed, uint32_t(cnl)};
  uint32_t c0[4] = {uint32_t(ray), 0u, 0u, 0u};
  uint32_t c1[4] = {uint32_t(ray), 1u, 0u, 0u};
  uint32_t o0[4], o1[4];
  philox4x32_10(c0, key, o0);
  philox4x32_10(c1, key, o1);
  u[0] = u01(o0[0]); u[1] = u01(o0[1]); u[2] = u01(o0[2]);
  u[3] = u01(o0[3]); u[4] = u01(o1[0]); u[5] = u01(o1[1]);
}

/* Random ray of a channel, src/RayGenerators.hpp:55-62: uniforms 0-2 into
 * the first pixel, 3-5 into the second. */
inline void make_ray(const ChannelTrafo& t, const float u[6], float ray[6]) {
  trafo_apply<float>(t.m0, &u[0], &ray[0]);
  trafo_apply<float>(t.m1, &u[3], &ray[3]);
}

/* ------------------------------------------------------------------------ */
/* Intersection length of a line with a box                                  */
/* ------------------------------------------------------------------------ */

/* src/getSystemMatrixDeviceOnly.cu:129-174 with the masked min/max of
 * src/ChordsCalc_lowlevel.hpp:49-175.  Dimensions the ray does not cross
 * are skipped by the masks (the reference leaves them unconstrained). */
inline float intersection_length(const float v[6], const float r[6]) {
  bool s[3];
  for (int d = 0; d < 3; d++) s[d] = r[d] != r[3 + d];
  if (!(s[0] || s[1] || s[2])) return 0.f;
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int d = 0; d < 3; d++) {
    if (s[d]) {
      lo[d] = (v[d] - r[d]) / (r[3 + d] - r[d]);
      hi[d] = (v[3 + d] - r[d]) / (r[3 + d] - r[d]);
      if (hi[d] < lo[d]) std::swap(lo[d], hi[d]);
    }
  }
  bool gmin = false, gmax = false;
  float amin = 0.f, amax = 0.f;
  for (int d = 0; d < 3; d++) {
    if (!s[d]) continue;
    if (!gmin) { amin = lo[d]; gmin = true; } else amin = std::max(amin, lo[d]);
    if (!gmax) { amax = hi[d]; gmax = true; } else amax = std::min(amax, hi[d]);
  }
  if (!(amin < amax)) return 0.f;
  float dx = r[3] - r[0], dy = r[4] - r[1], dz = r[5] - r[2];
  return (amax - amin) * sqrtf(dx * dx + dy * dy + dz * dz);
}

/* Voxel box corners: src/getSystemMatrixDeviceOnly.cu:207-219. */
inline void voxel_box(const OGeom& g, int ix, int iy, int iz, float v[6]) {
  v[0] = g.grid_o[0] + ix * (g.grid_d[0]);
  v[1] = g.grid_o[1] + iy * (g.grid_d[1]);
  v[2] = g.grid_o[2] + iz * (g.grid_d[2]);
  v[3] = g.grid_o[0] + (ix + 1) * (g.grid_d[0]);
  v[4] = g.grid_o[1] + (iy + 1) * (g.grid_d[1]);
  v[5] = g.grid_o[2] + (iz + 1) * (g.grid_d[2]);
}

/* ------------------------------------------------------------------------ */
/* Exact traversal: visits exactly the voxels with intersection_length > 0   */
/* ------------------------------------------------------------------------ */

/* Plane parameter of plane i of dimension d along the ray; the same
 * quotient as intersection_length forms for a voxel face. */
inline float plane_alpha(const OGeom& g, const float r[6], int d, int i) {
  float p = g.grid_o[d] + i * (g.grid_d[d]);
  return (p - r[d]) / (r[3 + d] - r[d]);
}

/* Calls f(ix, iy, iz, L) for every grid voxel whose intersection_length with
 * the ray is positive, with L bit-identical to intersection_length. */
template <typename F>
void walk_ray(const OGeom& g, const float r[6], F&& f) {
  bool s[3];
  int ncross = 0;
  for (int d = 0; d < 3; d++) { s[d] = r[d] != r[3 + d]; ncross += s[d]; }
  if (ncross == 0) return;
  const float INF = INFINITY;
  float dx = r[3] - r[0], dy = r[4] - r[1], dz = r[5] - r[2];
  float len = sqrtf(dx * dx + dy * dy + dz * dz);
  int step[3] = {0, 0, 0};
  float amin_g = -INF, amax_g = INF;
  for (int d = 0; d < 3; d++) {
    if (!s[d]) continue;
    step[d] = (r[3 + d] > r[d]) ? 1 : -1;
    float a0 = plane_alpha(g, r, d, 0);
    float a1 = plane_alpha(g, r, d, g.grid_n[d]);
    float lo = std::min(a0, a1), hi = std::max(a0, a1);
    amin_g = std::max(amin_g, lo);
    amax_g = std::min(amax_g, hi);
  }
  if (!(amin_g < amax_g)) return;
  int id[3] = {0, 0, 0};
  float lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    if (!s[d]) { lo[d] = -INF; hi[d] = INF; continue; }
    int n = g.grid_n[d];
    float pos = r[d] + amin_g * (r[3 + d] - r[d]);
    long i = long(std::floor((pos - g.grid_o[d]) / g.grid_d[d]));
    if (i < 0) i = 0;
    if (i > n - 1) i = n - 1;
    auto lo_of = [&](long k) { return step[d] > 0 ? plane_alpha(g, r, d, int(k)) : plane_alpha(g, r, d, int(k + 1)); };
    auto hi_of = [&](long k) { return step[d] > 0 ? plane_alpha(g, r, d, int(k + 1)) : plane_alpha(g, r, d, int(k)); };
    for (int guard = 0; guard < 64 && i >= 0 && i < n && !(hi_of(i) > amin_g); guard++) i += step[d];
    for (int guard = 0; guard < 64 && i >= 0 && i < n && lo_of(i) > amin_g; guard++) i -= step[d];
    if (i < 0 || i >= n) return;
    id[d] = int(i);
    lo[d] = lo_of(i);
    hi[d] = hi_of(i);
  }
  int guard_max = g.grid_n[0] + g.grid_n[1] + g.grid_n[2] + 8;
  for (int it = 0; it < guard_max; it++) {
    float a_lo = std::max(lo[0], std::max(lo[1], lo[2]));
    float a_hi = std::min(hi[0], std::min(hi[1], hi[2]));
    if (a_lo < a_hi) {
      float L = (a_hi - a_lo) * len;
      if (ncross == 3) {
        f(id[0], id[1], id[2], L);
      } else {
        /* A dimension the ray does not cross is unconstrained (reference
         * semantics): every index along it gets the same length. */
        int r0[3], r1[3];
        for (int d = 0; d < 3; d++) {
          r0[d] = s[d] ? id[d] : 0;
          r1[d] = s[d] ? id[d] : g.grid_n[d] - 1;
        }
        for (int a = r0[0]; a <= r1[0]; a++)
          for (int b = r0[1]; b <= r1[1]; b++)
            for (int c = r0[2]; c <= r1[2]; c++) f(a, b, c, L);
      }
    }
    float t = a_hi;
    if (!(t < amax_g)) break;
    bool out = false;
    for (int d = 0; d < 3; d++) {
      if (s[d] && hi[d] == t) {
        id[d] += step[d];
        if (id[d] < 0 || id[d] >= g.grid_n[d]) { out = true; break; }
        lo[d] = hi[d];
        hi[d] = step[d] > 0 ? plane_alpha(g, r, d, id[d] + 1) : plane_alpha(g, r, d, id[d]);
      }
    }
    if (out) break;
  }
}

/* ------------------------------------------------------------------------ */
/* Result containers                                                         */
/* ------------------------------------------------------------------------ */

struct CsrResult {
  std::vector<int64_t> row_ptr;
  std::vector<int32_t> col;
  std::vector<float> val;
};

struct WqResult {
  std::vector<int32_t> cnl, vxl;
};

inline int nthreads_or(int n) {
#ifdef _OPENMP
  return n > 0 ? n : omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

}  // namespace

/* ========================================================================== */
/* extern "C" surface used by oracle/oracle.py                                */
/* ========================================================================== */
extern "C" {

int ora_abi_version(void) { return 1; }

void ora_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) { philox4x32_10(ctr, key, out); }

void ora_ray_uniforms(uint32_t seed, int64_t cnl, int64_t ray, float* u) { ray_uniforms(seed, cnl, ray, u); }

/* Unit-cube coordinates of rays [0, nrays) of each listed channel
 * (n * nrays * 6 floats). */
void ora_ray_uniforms_batch(uint32_t seed, const int32_t* cnl, int64_t n, int32_t nrays, float* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++)
    for (int32_t r = 0; r < nrays; r++) ray_uniforms(seed, cnl[i], r, out + (i * nrays + r) * 6);
}

void ora_channel_split(const OGeom* g, int64_t cnl, int32_t* out5) {
  ChannelIds c = channel_split(*g, cnl);
  out5[0] = c.ida; out5[1] = c.id0z; out5[2] = c.id0y; out5[3] = c.id1z; out5[4] = c.id1y;
}

int64_t ora_channel_lin(const OGeom* g, int32_t id0z, int32_t id0y, int32_t id1z, int32_t id1y, int32_t ida) {
  return int64_t(ida) * (int64_t(g->n1y) * g->n1z * g->n0y * g->n0z) + int64_t(id0z) * (int64_t(g->n1y) * g->n1z * g->n0y) +
         int64_t(id0y) * (int64_t(g->n1y) * g->n1z) + int64_t(id1z) * g->n1y + id1y;
}

void ora_voxel_split(const OGeom* g, int64_t lin, int32_t* out3) {
  int ids[3];
  voxel_split(*g, lin, ids);
  out3[0] = ids[0]; out3[1] = ids[1]; out3[2] = ids[2];
}

void ora_angle_sincos(const OGeom* g, int32_t ida, float* s, float* c) { angle_sincos(g->da, ida, s, c); }

/* Float transform of `n` unit-cube points into pixel (idz, idy) of detector
 * `det` at angle `ida`. */
void ora_trafo_f(const OGeom* g, int32_t det, int32_t ida, int32_t idz, int32_t idy, const float* in, float* out, int64_t n) {
  float s, c, m[12];
  angle_sincos(g->da, ida, &s, &c);
  if (det == 0)
    trafo_matrix<float>(m, g->pos0x, idz, idy, g->n0y, g->n0z, g->segx, g->segy, g->segz, s, c);
  else
    trafo_matrix<float>(m, g->pos1x, idz, idy, g->n1y, g->n1z, g->segx, g->segy, g->segz, s, c);
  for (int64_t i = 0; i < n; i++) trafo_apply<float>(m, in + 3 * i, out + 3 * i);
}

/* Double-precision transform with the reference's float sine/cosine calls
 * (sinf/cosf applied to a double argument), as instantiated by the
 * reference's own unit test with val_t = double
 * (src/tests/MeasurementSetupTrafo2CartCoordUT.cu:58-63). */
void ora_trafo_d(double pos0x, double pos1x, int32_t n0z, int32_t n0y, int32_t n1z, int32_t n1y, double da, double segx,
                 double segy, double segz, int32_t det, int32_t ida, int32_t idz, int32_t idy, const double* in,
                 double* out) {
  double s = sinf(double(M_PI) * ida * da / double(180.0));
  double c = cosf(double(M_PI) * ida * da / double(180.0));
  double m[12];
  if (det == 0)
    trafo_matrix<double>(m, pos0x, idz, idy, n0y, n0z, segx, segy, segz, s, c);
  else
    trafo_matrix<double>(m, pos1x, idz, idy, n1y, n1z, segx, segy, segz, s, c);
  trafo_apply<double>(m, in, out);
}

int ora_candidate_test(const OGeom* g, int64_t cnl, int64_t vxl) {
  ChannelIds c = channel_split(*g, cnl);
  ChannelTrafo t = channel_trafo(*g, c);
  ChannelLine l = channel_line(*g, t);
  int ids[3];
  voxel_split(*g, vxl, ids);
  return candidate_test(*g, l, ids[0], ids[1], ids[2]) ? 1 : 0;
}

float ora_intersection_length(const float* vxl_box, const float* ray) { return intersection_length(vxl_box, ray); }

/* Ray endpoints of rays [0, nrays) of each listed channel. */
void ora_rays(const OGeom* g, const int32_t* cnl, int64_t n, int32_t nrays, uint32_t seed, float* out) {
  for (int64_t i = 0; i < n; i++) {
    ChannelTrafo t = channel_trafo(*g, channel_split(*g, cnl[i]));
    for (int32_t r = 0; r < nrays; r++) {
      float u[6];
      ray_uniforms(seed, cnl[i], r, u);
      make_ray(t, u, out + (i * nrays + r) * 6);
    }
  }
}

/* Chords of one ray via the exact traversal: returns the number written
 * (at most cap) and the total number found. */
int64_t ora_walk_ray(const OGeom* g, const float* ray, int32_t* vxl_out, float* len_out, int64_t cap) {
  int64_t k = 0;
  int64_t nyz = int64_t(g->grid_n[1]) * g->grid_n[2];
  walk_ray(*g, ray, [&](int ix, int iy, int iz, float L) {
    if (k < cap) {
      vxl_out[k] = int32_t(ix * nyz + int64_t(iy) * g->grid_n[2] + iz);
      len_out[k] = L;
    }
    k++;
  });
  return k;
}

/* Candidate search, the scan order and resumable cursor of
 * getWorkqueue/getWorkqueueEntry (src/getWorkqueue.hpp:53-133, :149-191):
 * list-major, voxel-minor; at most max_out entries; the cursor (list_id,
 * vxl_id) is advanced past the last entry returned.  `pruned` != 0 skips
 * voxels that provably fail the test (same result, faster). */
int64_t ora_workqueue(const OGeom* g, const int32_t* list, int64_t nlist, int64_t* cur_list, int64_t* cur_vxl,
                      int64_t max_out, int32_t* out_cnl, int32_t* out_vxl, int pruned) {
  int64_t nvox = int64_t(g->grid_n[0]) * g->grid_n[1] * g->grid_n[2];
  int64_t nyz = int64_t(g->grid_n[1]) * g->grid_n[2];
  int64_t found = 0;
  if (max_out <= 0) return 0;
  int64_t li = *cur_list, vi = *cur_vxl;
  /* Records a candidate and moves the cursor one voxel past it, wrapping to
   * the next list entry at the end of the grid (src/getWorkqueue.hpp:103-112).
   * Returns true when max_out entries have been returned. */
  auto take = [&](int64_t cnl, int64_t v) {
    out_cnl[found] = int32_t(cnl);
    out_vxl[found] = int32_t(v);
    found++;
    if (v < nvox - 1) { *cur_list = li; *cur_vxl = v + 1; }
    else { *cur_list = li + 1; *cur_vxl = 0; }
    return found >= max_out;
  };
  for (; li < nlist; li++, vi = 0) {
    int64_t cnl = list[li];
    ChannelLine l = channel_line(*g, channel_trafo(*g, channel_split(*g, cnl)));
    if (!pruned) {
      for (int64_t v = vi; v < nvox; v++) {
        int ids[3];
        voxel_split(*g, v, ids);
        if (candidate_test(*g, l, ids[0], ids[1], ids[2]) && take(cnl, v)) return found;
      }
    } else {
      int ids[3];
      voxel_split(*g, vi, ids);
      for (int ix = ids[0]; ix < g->grid_n[0]; ix++)
        for (int iy = (ix == ids[0] ? ids[1] : 0); iy < g->grid_n[1]; iy++) {
          int z0, z1;
          if (!row_z_interval(*g, l, ix, iy, &z0, &z1)) continue;
          int zs = (ix == ids[0] && iy == ids[1]) ? std::max(z0, ids[2]) : z0;
          for (int iz = zs; iz <= z1; iz++)
            if (candidate_test(*g, l, ix, iy, iz) && take(cnl, ix * nyz + int64_t(iy) * g->grid_n[2] + iz))
              return found;
        }
    }
  }
  *cur_list = nlist;
  *cur_vxl = 0;
  return found;
}

/* Number of candidates of each listed channel (full voxel range). */
void ora_candidate_counts(const OGeom* g, const int32_t* list, int64_t nlist, int64_t* counts, int nthreads) {
  int nt = nthreads_or(nthreads);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt)
  for (int64_t li = 0; li < nlist; li++) {
    ChannelLine l = channel_line(*g, channel_trafo(*g, channel_split(*g, list[li])));
    int64_t k = 0;
    for (int ix = 0; ix < g->grid_n[0]; ix++)
      for (int iy = 0; iy < g->grid_n[1]; iy++) {
        int z0, z1;
        if (!row_z_interval(*g, l, ix, iy, &z0, &z1)) continue;
        for (int iz = z0; iz <= z1; iz++) k += candidate_test(*g, l, ix, iy, iz);
      }
    counts[li] = k;
  }
}

/* -------------------------------------------------------------------------- */
/* System matrix rows                                                          */
/* -------------------------------------------------------------------------- */

/* Build the rows of the listed channels.
 *   method 0: the reference algorithm -- for every candidate voxel, the mean
 *             over rays of intersection_length (src/getSystemMatrixDeviceOnly.cu:
 *             185-246, src/getSystemMatrixFromWorkqueue.cu:216-264).
 *   method 1: the exact traversal with sums taken in ray order, which gives
 *             bit-identical values to method 0 in far less time.
 * Rays come from `rays` (n * nrays * 6 floats) when non-null, else from the
 * Philox stream keyed by (seed, channel).
 * keep_zeros != 0 keeps every candidate (the reference's COO structure);
 * otherwise exact zeros are dropped.  Columns are ascending within a row. */
void* ora_sysmat_build(const OGeom* g, const int32_t* list, int64_t nlist, int32_t nrays, uint32_t seed,
                       const float* rays, int method, int keep_zeros, int nthreads) {
  CsrResult* res = new CsrResult;
  int64_t nvox = int64_t(g->grid_n[0]) * g->grid_n[1] * g->grid_n[2];
  int64_t nyz = int64_t(g->grid_n[1]) * g->grid_n[2];
  std::vector<std::vector<int32_t>> rc(nlist);
  std::vector<std::vector<float>> rv(nlist);
  int nt = nthreads_or(nthreads);
#pragma omp parallel num_threads(nt)
  {
    std::vector<float> acc(method == 1 ? nvox : 0, 0.f);
    std::vector<unsigned char> touched(method == 1 ? nvox : 0, 0);
    std::vector<int32_t> touched_list;
    std::vector<float> rayv(size_t(nrays) * 6);
#pragma omp for schedule(dynamic, 4)
    for (int64_t li = 0; li < nlist; li++) {
      int64_t cnl = list[li];
      ChannelTrafo t = channel_trafo(*g, channel_split(*g, cnl));
      ChannelLine l = channel_line(*g, t);
      for (int32_t r = 0; r < nrays; r++) {
        if (rays) {
          std::memcpy(&rayv[size_t(r) * 6], rays + (li * int64_t(nrays) + r) * 6, 6 * sizeof(float));
        } else {
          float u[6];
          ray_uniforms(seed, cnl, r, u);
          make_ray(t, u, &rayv[size_t(r) * 6]);
        }
      }
      std::vector<int32_t>& oc = rc[li];
      std::vector<float>& ov = rv[li];
      if (method == 0) {
        for (int ix = 0; ix < g->grid_n[0]; ix++)
          for (int iy = 0; iy < g->grid_n[1]; iy++) {
            int z0, z1;
            if (!row_z_interval(*g, l, ix, iy, &z0, &z1)) continue;
            for (int iz = z0; iz <= z1; iz++) {
              if (!candidate_test(*g, l, ix, iy, iz)) continue;
              float box[6];
              voxel_box(*g, ix, iy, iz, box);
              float a = 0.f;
              for (int32_t r = 0; r < nrays; r++) a += intersection_length(box, &rayv[size_t(r) * 6]);
              a /= nrays;
              if (keep_zeros || a != 0.f) {
                oc.push_back(int32_t(ix * nyz + int64_t(iy) * g->grid_n[2] + iz));
                ov.push_back(a);
              }
            }
          }
      } else {
        touched_list.clear();
        for (int32_t r = 0; r < nrays; r++) {
          walk_ray(*g, &rayv[size_t(r) * 6], [&](int ix, int iy, int iz, float L) {
            int64_t v = ix * nyz + int64_t(iy) * g->grid_n[2] + iz;
            if (!touched[v]) { touched[v] = 1; touched_list.push_back(int32_t(v)); }
            acc[v] += L;
          });
        }
        if (keep_zeros) {
          for (int ix = 0; ix < g->grid_n[0]; ix++)
            for (int iy = 0; iy < g->grid_n[1]; iy++) {
              int z0, z1;
              if (!row_z_interval(*g, l, ix, iy, &z0, &z1)) continue;
              for (int iz = z0; iz <= z1; iz++) {
                if (!candidate_test(*g, l, ix, iy, iz)) continue;
                int64_t v = ix * nyz + int64_t(iy) * g->grid_n[2] + iz;
                float a = acc[v];
                a /= nrays;
                oc.push_back(int32_t(v));
                ov.push_back(a);
              }
            }
        } else {
          std::sort(touched_list.begin(), touched_list.end());
          for (int32_t v : touched_list) {
            int ids[3];
            voxel_split(*g, v, ids);
            if (!candidate_test(*g, l, ids[0], ids[1], ids[2])) continue;
            float a = acc[v];
            a /= nrays;
            if (a != 0.f) { oc.push_back(v); ov.push_back(a); }
          }
        }
        for (int32_t v : touched_list) { acc[v] = 0.f; touched[v] = 0; }
      }
    }
  }
  res->row_ptr.resize(nlist + 1);
  res->row_ptr[0] = 0;
  for (int64_t i = 0; i < nlist; i++) res->row_ptr[i + 1] = res->row_ptr[i] + int64_t(rc[i].size());
  res->col.resize(res->row_ptr[nlist]);
  res->val.resize(res->row_ptr[nlist]);
  for (int64_t i = 0; i < nlist; i++) {
    std::copy(rc[i].begin(), rc[i].end(), res->col.begin() + res->row_ptr[i]);
    std::copy(rv[i].begin(), rv[i].end(), res->val.begin() + res->row_ptr[i]);
  }
  return res;
}

int64_t ora_csr_nnz(void* h) { return static_cast<CsrResult*>(h)->row_ptr.back(); }

void ora_csr_copy(void* h, int64_t* row_ptr, int32_t* col, float* val) {
  CsrResult* r = static_cast<CsrResult*>(h);
  std::copy(r->row_ptr.begin(), r->row_ptr.end(), row_ptr);
  std::copy(r->col.begin(), r->col.end(), col);
  std::copy(r->val.begin(), r->val.end(), val);
}

void ora_csr_free(void* h) { delete static_cast<CsrResult*>(h); }

/* -------------------------------------------------------------------------- */
/* Sparse formats                                                              */
/* -------------------------------------------------------------------------- */

/* COO sort in row-major column-minor order (src/cooSort.hpp:47-98). */
void ora_coo_sort(float* val, int32_t* row, int32_t* col, int64_t n) {
  std::vector<int64_t> idx(n);
  for (int64_t i = 0; i < n; i++) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
    return row[a] < row[b] || (row[a] == row[b] && col[a] < col[b]);
  });
  std::vector<float> v(n);
  std::vector<int32_t> rr(n), cc(n);
  for (int64_t i = 0; i < n; i++) { v[i] = val[idx[i]]; rr[i] = row[idx[i]]; cc[i] = col[idx[i]]; }
  std::copy(v.begin(), v.end(), val);
  std::copy(rr.begin(), rr.end(), row);
  std::copy(cc.begin(), cc.end(), col);
}

/* COO row indices -> CSR row pointers (the contract of cusparseXcoo2csr used
 * at src/cusparseWrapper.hpp:53-60): histogram then exclusive scan. */
void ora_coo2csr(const int32_t* rows, int64_t nnz, int64_t m, int64_t* row_ptr) {
  std::vector<int64_t> cnt(m + 1, 0);
  for (int64_t i = 0; i < nnz; i++) cnt[rows[i] + 1]++;
  row_ptr[0] = 0;
  for (int64_t i = 0; i < m; i++) row_ptr[i + 1] = row_ptr[i] + cnt[i + 1];
}

/* CSR -> ECSR (src/convertCsr2Ecsr.hpp:51-64). */
void ora_csr2ecsr(int64_t* ecsr, const int32_t* yrow, int64_t nnzr, const int64_t* csr, int64_t m) {
  for (int64_t i = 0; i < nnzr; i++) ecsr[i] = csr[yrow[i]];
  ecsr[nnzr] = csr[m];
}

/* -------------------------------------------------------------------------- */
/* SpMV and MLEM                                                               */
/* -------------------------------------------------------------------------- */

/* y = alpha*op(A)*x + beta*y, op 0 = non-transposed, 1 = transposed
 * (the CSRmv contract, src/csrmv.hpp:31-66).  beta == 0 does not read y. */
}  // extern "C"

namespace {
template <typename T>
void spmv_t(int op, int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val, T alpha, const T* x,
            T beta, T* y) {
  if (op == 0) {
    for (int64_t i = 0; i < m; i++) {
      T s = 0;
      for (int64_t k = rp[i]; k < rp[i + 1]; k++) s += T(val[k]) * x[col[k]];
      y[i] = (beta == T(0)) ? alpha * s : alpha * s + beta * y[i];
    }
  } else {
    for (int64_t j = 0; j < n; j++) y[j] = (beta == T(0)) ? T(0) : beta * y[j];
    for (int64_t i = 0; i < m; i++)
      for (int64_t k = rp[i]; k < rp[i + 1]; k++) y[col[k]] += alpha * T(val[k]) * x[i];
  }
}

}  // namespace

extern "C" {

void ora_spmv_f32(int op, int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val, float alpha,
                  const float* x, float beta, float* y) {
  spmv_t<float>(op, m, n, rp, col, val, alpha, x, beta, y);
}

void ora_spmv_f64(int op, int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val, double alpha,
                  const double* x, double beta, double* y) {
  spmv_t<double>(op, m, n, rp, col, val, alpha, x, beta, y);
}

/* Element-wise MLEM operations (src/mlemOperations.hpp:44-169). */
void ora_divides(float* res, const float* a, const float* b, int64_t n) {
  for (int64_t i = 0; i < n; i++) res[i] = a[i] / b[i];
}

void ora_divides_multiplies(float* res, const float* a, const float* b, const float* c, int64_t n) {
  for (int64_t i = 0; i < n; i++) {
    float dvs = c[i];
    dvs += float(dvs == 0.);
    res[i] = a[i] * b[i] / dvs;
  }
}

void ora_scales(float* x, float alpha, int64_t n) {
  for (int64_t i = 0; i < n; i++) x[i] = alpha * x[i];
}

float ora_sum(const float* x, int64_t n) {
  float s = 0.f;
  for (int64_t i = 0; i < n; i++) s += x[i];
  return s;
}

/* Column sums of all rows in double: the sensitivity image. */
void ora_column_sums_f64(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val, double* s) {
  for (int64_t j = 0; j < n; j++) s[j] = 0.0;
  for (int64_t i = 0; i < m; i++)
    for (int64_t k = rp[i]; k < rp[i + 1]; k++) s[col[k]] += double(val[k]);
}

}  // extern "C"

namespace {

/* The transposed operand of the oracle's MLEM: for every column its rows in
 * ascending order with their values.  Summing a column's products in that
 * order adds them exactly as the sequential scatter y[col[k]] += a*x[i]
 * over rows i = 0, 1, ... does, so the back projection below is the same,
 * bit for bit, as spmv_t(1, ...) while its columns run in parallel. */
struct Csc {
  std::vector<int64_t> cp;
  std::vector<int32_t> row;
  std::vector<float> val;
};

Csc csc_of(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val) {
  Csc t;
  const int64_t nnz = rp[m];
  t.cp.assign(size_t(n) + 1, 0);
  for (int64_t k = 0; k < nnz; k++) t.cp[size_t(col[k]) + 1]++;
  for (int64_t j = 0; j < n; j++) t.cp[size_t(j) + 1] += t.cp[size_t(j)];
  t.row.resize(size_t(nnz));
  t.val.resize(size_t(nnz));
  std::vector<int64_t> next(t.cp.begin(), t.cp.end() - 1);
  for (int64_t i = 0; i < m; i++)
    for (int64_t k = rp[i]; k < rp[i + 1]; k++) {
      const int64_t p = next[size_t(col[k])]++;
      t.row[size_t(p)] = int32_t(i);
      t.val[size_t(p)] = val[k];
    }
  return t;
}

/* y = A x (op N, one row at a time, in entry order) and c = A^T e (op T,
 * one column at a time, in row order): the sums of spmv_t with alpha 1 and
 * beta 0, in the same order, rows / columns in parallel. */
template <typename T>
void forward_rows(int64_t m, const int64_t* rp, const int32_t* col, const float* val, const T* x, T* y) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < m; i++) {
    T s = 0;
    for (int64_t k = rp[i]; k < rp[i + 1]; k++) s += T(val[k]) * x[col[k]];
    y[i] = T(1) * s;
  }
}

template <typename T>
void back_columns(int64_t n, const Csc& t, const T* e, T* c) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t j = 0; j < n; j++) {
    T s = 0;
    for (int64_t p = t.cp[size_t(j)]; p < t.cp[size_t(j) + 1]; p++) s += T(1) * T(t.val[size_t(p)]) * e[t.row[size_t(p)]];
    c[j] = s;
  }
}

}  // namespace

extern "C" {

/* MLEM iterations in the order of src/tests/reco.cu:230-303 (single rank,
 * one chunk): c = 0; yt = A x; e = y / yt; c = A^T e; xx = x*c/(s + (s==0));
 * x = xx; x *= 1/sum(x).  `s` must already be normalised.  FP32 version
 * uses float vectors, FP64 version double vectors (same matrix values).
 * Every sum is taken in the order of the sequential CSRmv restatement
 * spmv_t (rows in entry order; columns in row order), so the result does
 * not depend on the thread count. */
void ora_mlem_f32(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val, const float* y,
                  const float* s, float* x, int32_t niter) {
  std::vector<float> yt(m), e(m), c(n), xx(n);
  const Csc t = csc_of(m, n, rp, col, val);
  for (int32_t it = 0; it < niter; it++) {
    forward_rows<float>(m, rp, col, val, x, yt.data());
    for (int64_t i = 0; i < m; i++) e[i] = y[i] / yt[i];
    back_columns<float>(n, t, e.data(), c.data());
    ora_divides_multiplies(xx.data(), x, c.data(), s, n);
    std::copy(xx.begin(), xx.end(), x);
    double norm = 0.0;
    for (int64_t j = 0; j < n; j++) norm += x[j];
    float scale = float(1. / float(norm));
    for (int64_t j = 0; j < n; j++) x[j] = scale * x[j];
  }
}

void ora_mlem_f64(int64_t m, int64_t n, const int64_t* rp, const int32_t* col, const float* val, const double* y,
                  const double* s, double* x, int32_t niter) {
  std::vector<double> yt(m), e(m), c(n);
  const Csc t = csc_of(m, n, rp, col, val);
  for (int32_t it = 0; it < niter; it++) {
    forward_rows<double>(m, rp, col, val, x, yt.data());
    for (int64_t i = 0; i < m; i++) e[i] = y[i] / yt[i];
    back_columns<double>(n, t, e.data(), c.data());
    for (int64_t j = 0; j < n; j++) {
      double dvs = s[j];
      dvs += double(dvs == 0.);
      x[j] = x[j] * c[j] / dvs;
    }
    double norm = 0.0;
    for (int64_t j = 0; j < n; j++) norm += x[j];
    for (int64_t j = 0; j < n; j++) x[j] = x[j] / norm;
  }
}

}  // extern "C"
