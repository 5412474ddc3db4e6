// Device-side geometry, exact arithmetic and random numbers shared by the
// raptr_b200 kernels.
//
// Every float operation that decides the structure or the values of the
// system matrix is written with explicit round-to-nearest intrinsics
// (__fmul_rn, __fadd_rn, __fsub_rn, __fdiv_rn, __fsqrt_rn), in the order
// the reference evaluates it, so no multiply-add contraction can change a
// result: the candidate test, the crystal transforms and the per-voxel
// intersection lengths are bit-identical to the reference's float arithmetic.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/raptr_b200.h"

namespace raptr {

#define RFMUL(a, b) __fmul_rn((a), (b))
#define RFADD(a, b) __fadd_rn((a), (b))
#define RFSUB(a, b) __fsub_rn((a), (b))
#define RFDIV(a, b) __fdiv_rn((a), (b))
#define RFSQRT(a) __fsqrt_rn((a))

// Geometry as passed to kernels (by value).  Same fields as raptr_geom.
struct DGeom {
  float o[3];
  float d[3];
  int n[3];
  float pos0x, pos1x;
  int na, n0z, n0y, n1z, n1y;
  float da, segx, segy, segz;
};

inline DGeom to_dgeom(const raptr_geom& g) {
  DGeom d;
  for (int i = 0; i < 3; i++) {
    d.o[i] = g.grid_o[i];
    d.d[i] = g.grid_d[i];
    d.n[i] = g.grid_n[i];
  }
  d.pos0x = g.pos0x; d.pos1x = g.pos1x;
  d.na = g.na; d.n0z = g.n0z; d.n0y = g.n0y; d.n1z = g.n1z; d.n1y = g.n1y;
  d.da = g.da; d.segx = g.segx; d.segy = g.segy; d.segz = g.segz;
  return d;
}

__host__ __device__ inline int num_channels(const DGeom& g) { return g.na * g.n0z * g.n0y * g.n1z * g.n1y; }

// Channel id -> (ida, id0z, id0y, id1z, id1y), id1y fastest
// (src/MeasurementSetupLinIndex.hpp:82-91 and its inverse functors).
struct ChannelIds {
  int ida, id0z, id0y, id1z, id1y;
};

__host__ __device__ inline ChannelIds channel_split(const DGeom& g, int cnl) {
  ChannelIds c;
  int s1 = g.n1y, s2 = g.n1y * g.n1z, s3 = s2 * g.n0y, s4 = s3 * g.n0z;
  c.ida = cnl / s4;
  int t = cnl - c.ida * s4;
  c.id0z = t / s3;
  t -= c.id0z * s3;
  c.id0y = t / s2;
  t -= c.id0y * s2;
  c.id1z = t / s1;
  c.id1y = t - c.id1z * s1;
  return c;
}

// Per-channel state: both crystal transforms, the crystal centres, the
// centre-line direction and its length, the cylinder radius.
struct Channel {
  float m0[12];
  float m1[12];
  float c0[3];
  float ab[3];     // c1 - c0
  float abs_ab;    // |c1 - c0|
  float radius;    // 0.5*(|voxel diagonal| + |crystal diagonal|)
};

// Transform matrix of a crystal (src/MeasurementSetupTrafo2CartCoord.hpp:99-131):
// scale by the segment edges, translate into the crystal, rotate about y.
__device__ __forceinline__ void trafo_matrix(float m[12], float posx, int idz, int idy, int ny, int nz, float segx,
                                             float segy, float segz, float s, float c) {
  float pos1 = RFMUL(RFSUB(float(idy), RFMUL(0.5f, float(ny - 1))), segy);
  float pos2 = RFMUL(RFSUB(float(idz), RFMUL(0.5f, float(nz - 1))), segz);
  float hx = RFSUB(posx, RFMUL(0.5f, segx));
  float hz = RFSUB(pos2, RFMUL(0.5f, segz));
  m[0] = RFMUL(c, segx);
  m[1] = 0.f;
  m[2] = RFMUL(s, segz);
  m[3] = RFADD(RFMUL(c, hx), RFMUL(s, hz));
  m[4] = 0.f;
  m[5] = segy;
  m[6] = 0.f;
  m[7] = RFSUB(pos1, RFMUL(0.5f, segy));
  m[8] = RFMUL(-s, segx);
  m[9] = 0.f;
  m[10] = RFMUL(c, segz);
  m[11] = RFADD(RFMUL(-s, hx), RFMUL(c, hz));
}

// Matrix application (src/MeasurementSetupTrafo2CartCoord.hpp:134-147).
__device__ __forceinline__ void trafo_apply(const float* m, float u0, float u1, float u2, float out[3]) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float* q = m + 4 * r;
    out[r] = RFADD(RFADD(RFADD(RFMUL(q[0], u0), RFMUL(q[1], u1)), RFMUL(q[2], u2)), RFMUL(q[3], 1.0f));
  }
}

__device__ __forceinline__ float norm3_exact(float a, float b, float c) {
  return RFSQRT(RFADD(RFADD(RFMUL(a, a), RFMUL(b, b)), RFMUL(c, c)));
}

// Builds the channel state; `sincos` holds (sin, cos) per angle step,
// computed on the host with the same float expression the reference uses.
__device__ inline void channel_setup(const DGeom& g, const float2* sincos, int cnl, Channel& ch) {
  ChannelIds id = channel_split(g, cnl);
  float2 sc = sincos[id.ida];
  trafo_matrix(ch.m0, g.pos0x, id.id0z, id.id0y, g.n0y, g.n0z, g.segx, g.segy, g.segz, sc.x, sc.y);
  trafo_matrix(ch.m1, g.pos1x, id.id1z, id.id1y, g.n1y, g.n1z, g.segx, g.segy, g.segz, sc.x, sc.y);
  float c0[3], c1[3];
  trafo_apply(ch.m0, 0.5f, 0.5f, 0.5f, c0);
  trafo_apply(ch.m1, 0.5f, 0.5f, 0.5f, c1);
  for (int d = 0; d < 3; d++) {
    ch.c0[d] = c0[d];
    ch.ab[d] = RFSUB(c1[d], c0[d]);
  }
  ch.abs_ab = norm3_exact(ch.ab[0], ch.ab[1], ch.ab[2]);
  float rv = norm3_exact(g.d[0], g.d[1], g.d[2]);
  float rp = norm3_exact(g.segx, g.segy, g.segz);
  ch.radius = RFMUL(0.5f, RFADD(rv, rp));
}

// Enclosing-cylinder test of voxel (ix, iy, iz): distance of the voxel centre
// from the line through both crystal centres below the sum of radii
// (src/getSystemMatrixDeviceOnly.cu:78-117, src/distancePointLine.h:40-101).
__device__ __forceinline__ bool candidate_test(const DGeom& g, const Channel& ch, int ix, int iy, int iz) {
  float p0 = RFADD(g.o[0], RFMUL(RFADD(float(ix), 0.5f), g.d[0]));
  float p1 = RFADD(g.o[1], RFMUL(RFADD(float(iy), 0.5f), g.d[1]));
  float p2 = RFADD(g.o[2], RFMUL(RFADD(float(iz), 0.5f), g.d[2]));
  float ap0 = RFSUB(p0, ch.c0[0]), ap1 = RFSUB(p1, ch.c0[1]), ap2 = RFSUB(p2, ch.c0[2]);
  float cx = RFSUB(RFMUL(ch.ab[1], ap2), RFMUL(ch.ab[2], ap1));
  float cy = RFSUB(RFMUL(ch.ab[2], ap0), RFMUL(ch.ab[0], ap2));
  float cz = RFSUB(RFMUL(ch.ab[0], ap1), RFMUL(ch.ab[1], ap0));
  float dist = RFDIV(norm3_exact(cx, cy, cz), ch.abs_ab);
  return dist < ch.radius;
}

// Conservative z-interval of the voxel row (ix, iy) that can pass the
// cylinder test.  Only prunes the scan: every voxel inside is still decided
// by candidate_test, and the interval is widened (radius +2%, two voxels on
// each side) so that it contains every passing voxel.
__device__ inline bool row_z_interval(const DGeom& g, const Channel& ch, int ix, int iy, int* z0, int* z1) {
  float inv = 1.0f / ch.abs_ab;
  float ux = ch.ab[0] * inv, uy = ch.ab[1] * inv, uz = ch.ab[2] * inv;
  float R = ch.radius * 1.02f + 0.05f * fmaxf(g.d[0], fmaxf(g.d[1], g.d[2]));
  float dx = g.o[0] + (ix + 0.5f) * g.d[0] - ch.c0[0];
  float dy = g.o[1] + (iy + 0.5f) * g.d[1] - ch.c0[1];
  float w = dx * ux + dy * uy;
  float a2 = 1.0f - uz * uz;
  float c0 = dx * dx + dy * dy - w * w - R * R;
  int nz = g.n[2];
  if (a2 < 1e-6f) {
    if (c0 < 0.f) { *z0 = 0; *z1 = nz - 1; return true; }
    return false;
  }
  float b1 = -2.0f * uz * w;
  float disc = b1 * b1 - 4.0f * a2 * c0;
  if (disc < 0.f) return false;
  float sq = sqrtf(disc);
  float zlo = ch.c0[2] + (-b1 - sq) / (2.f * a2);
  float zhi = ch.c0[2] + (-b1 + sq) / (2.f * a2);
  float flo = (zlo - g.o[2]) / g.d[2] - 0.5f;
  float fhi = (zhi - g.o[2]) / g.d[2] - 0.5f;
  if (fhi < -3.0f || flo > float(nz) + 2.0f) return false;
  int lo = int(floorf(flo)) - 2;
  int hi = int(ceilf(fhi)) + 2;
  lo = lo < 0 ? 0 : lo;
  hi = hi > nz - 1 ? nz - 1 : hi;
  if (lo > hi) return false;
  *z0 = lo;
  *z1 = hi;
  return true;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Key (seed, channel),
// counter (ray, half, 0, 0); 24 random bits -> float in (0, 1].
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
#ifdef __CUDA_ARCH__
    uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
#else
    uint64_t p0 = uint64_t(0xD2511F53u) * c[0], p1 = uint64_t(0xCD9E8D57u) * c[2];
    uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0), hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
#endif
    uint32_t n0 = hi1 ^ c[1] ^ k0;
    uint32_t n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__host__ __device__ __forceinline__ float u01(uint32_t x) { return float((x >> 8) + 1u) * (1.0f / 16777216.0f); }

// Endpoints of ray `ray` of the channel: uniforms 0-2 into the first
// crystal, 3-5 into the second (src/RayGenerators.hpp:55-62).
__device__ __forceinline__ void make_ray(const Channel& ch, uint32_t seed, int cnl, int ray, float r[6]) {
  uint32_t a[4] = {uint32_t(ray), 0u, 0u, 0u};
  uint32_t b[4] = {uint32_t(ray), 1u, 0u, 0u};
  philox4x32_10(a, seed, uint32_t(cnl));
  philox4x32_10(b, seed, uint32_t(cnl));
  trafo_apply(ch.m0, u01(a[0]), u01(a[1]), u01(a[2]), &r[0]);
  trafo_apply(ch.m1, u01(a[3]), u01(b[0]), u01(b[1]), &r[3]);
}

// The warp's next work item: lane 0 draws it from the counter at `next`
// and broadcasts it.  Called by all 32 lanes together.  The row passes draw
// kRowChunk rows at a time: one draw per row (5.14M draws on one address)
// makes the forward pass twice as slow, one per 16 rows takes 7 % off the
// grid stride's time.
constexpr int kRowChunk = 16;
__device__ __forceinline__ int64_t warp_next(unsigned long long* next, int lane) {
  unsigned long long q = 0;
  if (lane == 0) q = atomicAdd(next, 1ull);
  return int64_t(__shfl_sync(0xffffffffu, q, 0));
}

}  // namespace raptr
