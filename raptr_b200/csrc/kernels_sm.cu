// System-matrix rows, ray endpoints and the enclosing-cylinder candidate
// search, for sm_100a.
//
// Row build (one CTA per channel row):
//   1. thread 0 builds the channel state (both crystal transforms from the
//      per-angle sine/cosine table, crystal centres, cylinder radius);
//   2. every thread generates rays r = tid, tid+T, ... (Philox keyed by
//      (seed, channel)) and walks each through the grid.  The walk visits
//      exactly the voxels whose intersection length with the ray is positive
//      and computes that length with the same float operations as the
//      reference's intersectionLength (src/getSystemMatrixDeviceOnly.cu:129-174):
//      per-axis plane parameters (face - start)/(end - start), masked max of
//      the entry parameters, masked min of the exit parameters, and
//      (exit - entry) * |end - start|.  Lengths are summed in shared memory:
//      into dense per-slab windows of the voxels the row's rays can reach
//      when the two crystals lie on opposite sides of the grid along x or z,
//      else into an open-addressing hash table keyed by voxel id;
//   3. the sums are compacted keeping voxels that pass the exact cylinder
//      test (the reference only evaluates candidates,
//      src/getSystemMatrixDeviceOnly.cu:433-470), put in voxel-id order
//      (x-slab windows already are; the others are bitonic-sorted), divided
//      by the ray count and written to the row's staging slot.
// The rows are therefore emitted already in (row, column) order: no global
// COO sort (src/cooSort.hpp:75-99) and no coo->csr pass are needed; a scan
// of the row lengths and a gather place them into CSR.
//
// This translation unit is compiled with -fmad=false in addition to the
// explicit round-to-nearest intrinsics used on every exact path.
#include <algorithm>
#include <climits>
#include <cstdint>

#include "common.cuh"
#include "internal.h"

namespace raptr {

namespace {

constexpr int kProbeLimit = 128;

__device__ __forceinline__ float plane_alpha(float o, float d, int i, float r0, float dir) {
  return RFDIV(RFSUB(RFADD(o, RFMUL(float(i), d)), r0), dir);
}

// RN(a / b) from y = RN(1 / b) (P. Markstein's correction, IBM J. R&D 34(1),
// 1990), applied twice so that the first correction brings q within one ulp.
__device__ __forceinline__ float div_rcp(float a, float b, float y) {
  float q = __fmul_rn(a, y);
  float r = __fmaf_rn(-q, b, a);
  q = __fmaf_rn(r, y, q);
  r = __fmaf_rn(-q, b, a);
  return __fmaf_rn(r, y, q);
}

// plane_alpha with the division by a precomputed reciprocal rc = RN(1/dir)
// (exact as RN(num/dir), see div_rcp); a dir whose reciprocal is not a
// normal float takes the division itself.
__device__ __forceinline__ float plane_alpha_r(float o, float d, int i, float r0, float dir, float rc) {
  const float num = RFSUB(RFADD(o, RFMUL(float(i), d)), r0);
  if (!(fabsf(dir) >= 1e-30f && fabsf(dir) <= 1e30f)) return RFDIV(num, dir);
  return div_rcp(num, dir, rc);
}

// Origin, pitch and size of axis k of the grid for a k known only at run
// time: selects, so that the by-value geometry stays in the constant bank
// instead of being copied to local memory for an indexed access.
__device__ __forceinline__ float axis_o(const DGeom& g, int k) { return k == 0 ? g.o[0] : (k == 1 ? g.o[1] : g.o[2]); }
__device__ __forceinline__ float axis_d(const DGeom& g, int k) { return k == 0 ? g.d[0] : (k == 1 ? g.d[1] : g.d[2]); }
__device__ __forceinline__ int axis_n(const DGeom& g, int k) { return k == 0 ? g.n[0] : (k == 1 ? g.n[1] : g.n[2]); }

// Shared-memory accumulation table: keys (voxel id, -1 = empty) and sums.
template <int H>
struct RowTable {
  int* keys;
  float* vals;
  int* overflow;

  __device__ __forceinline__ void add(int key, float v) const {
    constexpr int LOG2H = (H == 2048) ? 11 : (H == 4096) ? 12 : (H == 8192) ? 13 : 14;
    unsigned h = (unsigned(key) * 2654435761u) >> (32 - LOG2H);
#pragma unroll 1
    for (int p = 0; p < kProbeLimit; p++) {
      int k = reinterpret_cast<volatile int*>(keys)[h];
      if (k == key) {
        atomicAdd(&vals[h], v);
        return;
      }
      if (k < 0) {
        int old = atomicCAS(&keys[h], -1, key);
        if (old < 0 || old == key) {
          atomicAdd(&vals[h], v);
          return;
        }
      }
      h = (h + 1) & (H - 1);
    }
    *overflow = 1;
  }
};

// Where the step walk adds a voxel's length.  KeyIndex tracks the voxel id
// and adds to the row's hash table; DenseIndex tracks the voxel's slot in
// the row's slab windows (below) and adds to it directly.  begin() takes the
// ray's step directions, set() places the index at a voxel, advance() moves
// it one voxel along the axis the walk steps (x if ax, else y if ay, else z).
template <int H>
struct KeyIndex {
  const RowTable<H>* table;
  int nyz, nz;
  int key, k0, k1, k2;
  __device__ __forceinline__ void begin(const int step[3]) {
    k0 = step[0] * nyz;
    k1 = step[1] * nz;
    k2 = step[2];
  }
  __device__ __forceinline__ void set(int i0, int i1, int i2) { key = i0 * nyz + i1 * nz + i2; }
  __device__ __forceinline__ void advance(bool ax, bool ay) { key += ax ? k0 : (ay ? k1 : k2); }
  __device__ __forceinline__ void add(float L) const { table->add(key, L); }
};

// Slab windows of a row whose rays all cross the grid in the same direction
// along the slab axis A (x or z): for every slab s of A the rays' voxels lie
// in a window [ulo[s], ulo[s]+wu) x [vlo[s], vlo[s]+wv) of the other two
// axes U < V (y, z for A = x; x, y for A = z), which holds wu*wv dense slots
// from slot s*wu*wv on (slot = base[s] + iu*wv + iv).  A step in U moves the
// slot by +-wv, in V by +-1, in A by dk[s] (the base difference to the next
// slab in the rays' direction).  No key is stored or compared.
template <int A>
struct DenseIndex {
  float* acc;
  const int* base;
  const int* dk;
  int wv, nslots;
  int slot, sa, ka, sta, ku, kv;
  __device__ __forceinline__ void begin(const int step[3]) {
    sta = step[A];
    ku = step[A == 0 ? 1 : 0] * wv;
    kv = step[A == 0 ? 2 : 1];
  }
  __device__ __forceinline__ void set(int i0, int i1, int i2) {
    sa = A == 0 ? i0 : i2;
    slot = A == 0 ? base[i0] + i1 * wv + i2 : base[i2] + i0 * wv + i1;
    ka = dk[sa];
  }
  __device__ __forceinline__ void advance(bool ax, bool ay) {
    if (A == 0) {
      slot += ax ? ka : (ay ? ku : kv);
      sa = ax ? sa + sta : sa;
    } else {
      slot += ax ? ku : (ay ? kv : ka);
      sa = (ax || ay) ? sa : sa + sta;
    }
    ka = dk[sa];
  }
  __device__ __forceinline__ void add(float L) const {
    // a slot outside the windows goes to the spare slot at nslots, which
    // the row checks afterwards (no branch in the step loop)
    atomicAdd(&acc[unsigned(slot) < unsigned(nslots) ? slot : nslots], L);
  }
};

// Visits every grid voxel whose intersection length with ray r is positive.
// A ray that crosses the planes of all three axes takes the step loop,
// which adds the lengths through the index `ix`; any other ray takes the
// general loop, which adds through emit(ix, iy, iz, L): a ray parallel to
// the planes of some axis (start and end coordinate equal) leaves that axis
// unconstrained, as the reference's masked min/max does, and every
// candidate voxel along it gets the length.  UNROLL is the step loop's
// unroll factor (the arithmetic of each step is the same for any).
template <bool OISO, int UNROLL, class Emit, class Index>
__device__ __forceinline__ void walk_ray(const DGeom& g, const Channel& ch, const float r[6], int part, Emit& emit,
                                         Index& ix, int* bad_walk) {
  float dir[3];
  bool s[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    dir[d] = RFSUB(r[3 + d], r[d]);
    s[d] = r[d] != r[3 + d];
  }
  if (!(s[0] || s[1] || s[2])) return;
  float rc[3];
#pragma unroll
  for (int d = 0; d < 3; d++) rc[d] = s[d] ? __frcp_rn(dir[d]) : 0.f;
  const float len = norm3_exact(dir[0], dir[1], dir[2]);
  int step[3] = {0, 0, 0};
  float amin_g = -INFINITY, amax_g = INFINITY;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (s[d]) {
      step[d] = (r[3 + d] > r[d]) ? 1 : -1;
      float a0 = plane_alpha_r(g.o[d], g.d[d], 0, r[d], dir[d], rc[d]);
      float a1 = plane_alpha_r(g.o[d], g.d[d], g.n[d], r[d], dir[d], rc[d]);
      amin_g = fmaxf(amin_g, fminf(a0, a1));
      amax_g = fminf(amax_g, fmaxf(a0, a1));
    }
  }
  if (!(amin_g < amax_g)) return;
  int id[3];
  float lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    id[d] = 0;
    lo[d] = -INFINITY;
    hi[d] = INFINITY;
    if (s[d]) {
      const int n = g.n[d];
      float pos = r[d] + amin_g * dir[d];
      int i = int(floorf(__fdividef(pos - g.o[d], g.d[d])));  // a guess: corrected below
      i = min(max(i, 0), n - 1);
      // Exact correction against the plane parameters: find the voxel whose
      // interval [lo, hi) contains the entry parameter.
      float l, h;
#pragma unroll 1
      for (int guard = 0; guard < 64; guard++) {
        float pa = plane_alpha_r(g.o[d], g.d[d], i, r[d], dir[d], rc[d]);
        float pb = plane_alpha_r(g.o[d], g.d[d], i + 1, r[d], dir[d], rc[d]);
        l = step[d] > 0 ? pa : pb;
        h = step[d] > 0 ? pb : pa;
        if (!(h > amin_g)) {
          i += step[d];
        } else if (l > amin_g) {
          i -= step[d];
        } else {
          break;
        }
        if (i < 0 || i >= n) {
          *bad_walk = 1;
          return;
        }
      }
      id[d] = i;
      lo[d] = l;
      hi[d] = h;
    }
  }
  const bool all3 = s[0] && s[1] && s[2];
  const int guard_max = g.n[0] + g.n[1] + g.n[2] + 8;
  // The step loop computes plane parameters exactly as plane_alpha_r did
  // for the grid's bounding planes (same operations and reciprocals), which
  // keeps every step inside the grid; a direction component outside the
  // range where plane_alpha_r uses the reciprocal goes to the general loop.
  bool in_range = true;
#pragma unroll
  for (int d = 0; d < 3; d++) in_range = in_range && fabsf(dir[d]) >= 1e-30f && fabsf(dir[d]) <= 1e30f;
  if (all3 && in_range) {
    // One axis per step, chosen with selects (no runtime array index):
    // the axis whose next plane comes first.  Planes of two axes at the same
    // parameter take two steps; the voxel between them has zero length (its
    // reference value is zero) and is dropped when the row is compacted.
    int i0 = id[0], i1 = id[1], i2 = id[2];
    float lo0 = lo[0], lo1 = lo[1], lo2 = lo[2];
    float hi0 = hi[0], hi1 = hi[1], hi2 = hi[2];
    const float y0 = rc[0], y1 = rc[1], y2 = rc[2];
    ix.begin(step);
    ix.set(i0, i1, i2);
    // Staggered start: the walk begins at a plane of the dominant axis D,
    // part/256 of the way along the ray, runs to the exit, then wraps
    // around to the entry and runs up to that plane.  No voxel straddles a
    // plane of D, so every voxel is still visited once with the same
    // lengths, while the threads of a row -- nearly parallel rays of one
    // channel -- sit on different voxels at any step instead of adding to
    // the same shared-memory accumulator at once.
    const int s0 = i0, s1 = i1, s2 = i2;
    const Index six = ix;
    const float sl0 = lo0, sl1 = lo1, sl2 = lo2, sh0 = hi0, sh1 = hi1, sh2 = hi2;
    float stop = amax_g, a_split = amax_g;
    bool wrapped = true;
    if (part > 0) {
      const float dx = fabsf(dir[0]), dy = fabsf(dir[1]), dz = fabsf(dir[2]);
      const int D = (dx >= dy) ? ((dx >= dz) ? 0 : 2) : ((dy >= dz) ? 1 : 2);
      const float oD = D == 0 ? g.o[0] : (D == 1 ? g.o[1] : g.o[2]);
      const float pD = D == 0 ? g.d[0] : (D == 1 ? g.d[1] : g.d[2]);
      const float rD = D == 0 ? r[0] : (D == 1 ? r[1] : r[2]);
      const float dD = D == 0 ? dir[0] : (D == 1 ? dir[1] : dir[2]);
      const float cD = D == 0 ? rc[0] : (D == 1 ? rc[1] : rc[2]);
      const int stD = D == 0 ? step[0] : (D == 1 ? step[1] : step[2]);
      const int nD = D == 0 ? g.n[0] : (D == 1 ? g.n[1] : g.n[2]);
      const int iD = D == 0 ? i0 : (D == 1 ? i1 : i2);
      const float hD = D == 0 ? hi0 : (D == 1 ? hi1 : hi2);
      const int span = int(__fdividef(fabsf((amax_g - amin_g) * dD), pD)) + 1;
      const int k = (part * span) >> 8;
      const int is = iD + stD * k;
      if (k > 0 && is >= 0 && is < nD) {
        const float as = plane_alpha_r(oD, pD, stD > 0 ? is : is + 1, rD, dD, cD);
        if (as > hD && as < amax_g) {
          int ni[3];
          float nl[3], nh[3];
          bool ok = true;
#pragma unroll
          for (int d = 0; d < 3; d++) {
            if (d == D) {
              ni[d] = is;
              nl[d] = as;
              nh[d] = plane_alpha_r(oD, pD, stD > 0 ? is + 1 : is, rD, dD, cD);
            } else {
              // the voxel of axis d whose interval [lo, hi) holds as
              int i = int(floorf(__fdividef(r[d] + as * dir[d] - g.o[d], g.d[d])));
              i = min(max(i, 0), g.n[d] - 1);
              float l = 0.f, h = 0.f;
              bool found = false;
#pragma unroll 1
              for (int guard = 0; guard < 64 && !found; guard++) {
                const float pa = plane_alpha_r(g.o[d], g.d[d], i, r[d], dir[d], rc[d]);
                const float pb = plane_alpha_r(g.o[d], g.d[d], i + 1, r[d], dir[d], rc[d]);
                l = step[d] > 0 ? pa : pb;
                h = step[d] > 0 ? pb : pa;
                if (!(h > as))
                  i += step[d];
                else if (l > as)
                  i -= step[d];
                else
                  found = true;
                if (i < 0 || i >= g.n[d]) break;
              }
              ok = ok && found;
              ni[d] = i;
              nl[d] = l;
              nh[d] = h;
            }
          }
          if (ok) {
            i0 = ni[0];
            i1 = ni[1];
            i2 = ni[2];
            lo0 = nl[0];
            lo1 = nl[1];
            lo2 = nl[2];
            hi0 = nh[0];
            hi1 = nh[1];
            hi2 = nh[2];
            ix.set(i0, i1, i2);
            a_split = as;
            wrapped = false;
          }
        }
      }
    }
    // Loop state per axis: the parameter of the next plane (hi) and the index
    // of the plane after it times the step direction, as a float (exact
    // small integers), so that it grows by one per step on every axis; the
    // pitch carries the direction instead (q*pd = (-q)*(-pd) exactly).  The
    // entry parameter of the current voxel is the previous step's exit
    // (prev).
    const float ps0 = step[0] > 0 ? g.d[0] : -g.d[0];
    const float ps1 = step[1] > 0 ? g.d[1] : -g.d[1];
    const float ps2 = step[2] > 0 ? g.d[2] : -g.d[2];
    float q0 = float(step[0] > 0 ? i0 + 2 : 1 - i0);
    float q1 = float(step[1] > 0 ? i1 + 2 : 1 - i1);
    float q2 = float(step[2] > 0 ? i2 + 2 : 1 - i2);
    float prev = fmaxf(lo0, fmaxf(lo1, lo2));
    const float sq0 = float(step[0] > 0 ? s0 + 2 : 1 - s0);
    const float sq1 = float(step[1] > 0 ? s1 + 2 : 1 - s1);
    const float sq2 = float(step[2] > 0 ? s2 + 2 : 1 - s2);
    const float sprev = fmaxf(sl0, fmaxf(sl1, sl2));
#pragma unroll UNROLL
    for (int it = 0; it < guard_max; it++) {
      const float a_hi = fminf(hi0, fminf(hi1, hi2));
      // A voxel between two planes at the same parameter gets length 0; it
      // is added all the same (no branch) and dropped with the other
      // zero sums when the row is compacted.
      ix.add(RFMUL(RFSUB(a_hi, prev), len));
      // The next plane lies before the exit, so it is not the grid's last
      // plane of its axis, and the step stays inside the grid.
      if (!(a_hi < stop)) {
        if (wrapped) return;
        // the second leg: from the entry up to the split plane
        q0 = sq0;
        q1 = sq1;
        q2 = sq2;
        hi0 = sh0;
        hi1 = sh1;
        hi2 = sh2;
        ix = six;
        prev = sprev;
        stop = a_split;
        wrapped = true;
        continue;
      }
      const bool ax = hi0 == a_hi;
      const bool ay = !ax && hi1 == a_hi;
      const float q = ax ? q0 : (ay ? q1 : q2);
      const float o = OISO ? g.o[0] : (ax ? g.o[0] : (ay ? g.o[1] : g.o[2]));
      const float pd = ax ? ps0 : (ay ? ps1 : ps2);
      const float r0 = ax ? r[0] : (ay ? r[1] : r[2]);
      const float dd = ax ? dir[0] : (ay ? dir[1] : dir[2]);
      const float yy = ax ? y0 : (ay ? y1 : y2);
      const float hn = div_rcp(RFSUB(RFADD(o, RFMUL(q, pd)), r0), dd, yy);
      const float qn = RFADD(q, 1.0f);
      ix.advance(ax, ay);
      q0 = ax ? qn : q0;
      q1 = ay ? qn : q1;
      q2 = (!ax && !ay) ? qn : q2;
      hi0 = ax ? hn : hi0;
      hi1 = ay ? hn : hi1;
      hi2 = (!ax && !ay) ? hn : hi2;
      prev = a_hi;
    }
    *bad_walk = 1;
    return;
  }
#pragma unroll 1
  for (int it = 0; it < guard_max; it++) {
    float a_lo = fmaxf(lo[0], fmaxf(lo[1], lo[2]));
    float a_hi = fminf(hi[0], fminf(hi[1], hi[2]));
    if (a_lo < a_hi) {
      float L = RFMUL(RFSUB(a_hi, a_lo), len);
      if (all3) {
        emit(id[0], id[1], id[2], L);
      } else {
        int r0[3], r1[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          r0[d] = s[d] ? id[d] : 0;
          r1[d] = s[d] ? id[d] : g.n[d] - 1;
        }
        for (int a = r0[0]; a <= r1[0]; a++)
          for (int b = r0[1]; b <= r1[1]; b++)
            for (int c = r0[2]; c <= r1[2]; c++)
              if (candidate_test(g, ch, a, b, c)) emit(a, b, c, L);
      }
    }
    if (!(a_hi < amax_g)) return;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (s[d] && hi[d] == a_hi) {
        id[d] += step[d];
        if (id[d] < 0 || id[d] >= g.n[d]) return;
        lo[d] = hi[d];
        hi[d] = plane_alpha(g.o[d], g.d[d], step[d] > 0 ? id[d] + 1 : id[d], r[d], dir[d]);
      }
    }
  }
  *bad_walk = 1;
}

// Block-wide exclusive scan of one int per thread; returns the prefix and
// sets *total.  `warp_sums` holds at least 32 ints.  Ends with a barrier.
template <int T>
__device__ __forceinline__ int block_exclusive_scan(int v, int* total, int* warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < T / 32) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < T / 32) warp_sums[lane] = w;  // inclusive
  }
  __syncthreads();
  int before = (warp > 0 ? warp_sums[warp - 1] : 0) + x - v;
  *total = warp_sums[T / 32 - 1];
  __syncthreads();
  return before;
}

constexpr int kMaxSlabs = 256;

// Dense slots of a row (floats) and the row kernel's dynamic shared memory:
// the hash table's H keys and H sums, or the dense windows, whichever is
// larger.  3H dense slots keep every row of the centred-cube workloads
// dense; at H = 4096 the 48 KB still leave four CTAs per SM, which the
// registers limit it to anyway.
__host__ __device__ constexpr int dense_slots(int H) { return H <= 4096 ? 3 * H : 2 * H; }
__host__ __device__ constexpr size_t row_smem_bytes(int H) {
  return size_t(H) * 8 > size_t(dense_slots(H)) * 4 ? size_t(H) * 8 : size_t(dense_slots(H)) * 4;
}

// Row-level decision for the slab windows: both crystals' boxes (corner
// AABBs) lie on opposite sides of the grid in x, so every ray of the row
// crosses the whole grid in the same x direction (xdir) and lies in the
// convex hull of the two boxes.
__device__ inline void crystal_boxes(const Channel& ch, float lo[2][3], float hi[2][3]) {
  for (int b = 0; b < 2; b++) {
    const float* m = b == 0 ? ch.m0 : ch.m1;
    for (int d = 0; d < 3; d++) {
      lo[b][d] = INFINITY;
      hi[b][d] = -INFINITY;
    }
    for (int c = 0; c < 8; c++) {
      float p[3];
      trafo_apply(m, float(c & 1), float((c >> 1) & 1), float((c >> 2) & 1), p);
      for (int d = 0; d < 3; d++) {
        lo[b][d] = fminf(lo[b][d], p[d]);
        hi[b][d] = fmaxf(hi[b][d], p[d]);
      }
    }
  }
}

// The voxel range along axis w that rays from box P (lower coordinate on
// the slab axis a) to box Q can reach within the slab [c0, c1] of axis a: a
// ray point at coordinate c is (1-t)*p + t*q with p in P, q in Q and t
// between (c - bP)/(bQ - bP) and (c - aP)/(aQ - aP) ([aP, bP], [aQ, bQ] the
// boxes' ranges along a), so its w lies between the extremes of the boxes'
// w bounds at those t, at both slab faces.  One voxel of margin on each
// side covers rounding.
__device__ inline void slab_window(const DGeom& g, int a, const float plo[3], const float phi[3],
                                   const float qlo[3], const float qhi[3], float c0, float c1, int w, int* ilo,
                                   int* ihi) {
  float wlo = INFINITY, whi = -INFINITY;
#pragma unroll
  for (int e = 0; e < 2; e++) {
    const float c = e == 0 ? c0 : c1;
    const float t1 = (c - phi[a]) / (qhi[a] - phi[a]);
    const float t2 = (c - plo[a]) / (qlo[a] - plo[a]);
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const float t = k == 0 ? t1 : t2;
      wlo = fminf(wlo, plo[w] + t * (qlo[w] - plo[w]));
      whi = fmaxf(whi, phi[w] + t * (qhi[w] - phi[w]));
    }
  }
  const int n = axis_n(g, w);
  int lo = int(floorf((wlo - axis_o(g, w)) / axis_d(g, w))) - 1;
  int hi = int(floorf((whi - axis_o(g, w)) / axis_d(g, w))) + 1;
  lo = min(max(lo, 0), n - 1);
  hi = min(max(hi, 0), n - 1);
  *ilo = lo;
  *ihi = max(lo, hi);
}

// The dense kernel's step-loop unroll factor by row capacity, measured on
// full builds: 6 at H = 4096 (70^3 x 5.14M channels: 2.04 s unrolled 1,
// 2.00 s by 2, 1.86 s by 4, 1.81 s by 6 and by 8; 8 spills), none at
// H = 8192 (100^3 x 1.71M channels: 1.23 s unrolled 1, 1.25 s by 4, 1.32 s
// by 6, 1.37 s by 8) nor at H = 2048 (40^3 x 143K channels: 8-9 ms either
// way, and unrolled it spills).
constexpr int dense_walk_unroll(int H) { return H == 4096 ? 6 : 1; }

// Row status the dense kernel leaves for the table kernel: the row is to be
// built with the hash table (it does not qualify for dense windows, or a
// ray left its windows).
constexpr int kRowToTable = -2;

// Bitonic sort of (keys, vals)[0, total) by key in shared memory (npad =
// the next power of two, padded with INT_MAX), then written to the row's
// staging slot and its length to *row_nnz.  Every thread of the CTA calls it.
template <int T>
__device__ void sort_and_write(int* keys, float* vals, int total, int32_t* __restrict__ st_col,
                               float* __restrict__ st_val, size_t base, int32_t* row_nnz) {
  const int tid = threadIdx.x;
  int npad = 1;
  while (npad < total) npad <<= 1;
  for (int i = total + tid; i < npad; i += T) keys[i] = INT_MAX;
  __syncthreads();
  for (int k = 2; k <= npad; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < (npad >> 1); t += T) {
        int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
        int p = i | j;
        bool asc = (i & k) == 0;
        int ki = keys[i], kp = keys[p];
        if ((ki > kp) == asc) {
          keys[i] = kp;
          keys[p] = ki;
          float vi = vals[i];
          vals[i] = vals[p];
          vals[p] = vi;
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < total; i += T) {
    st_col[base + i] = keys[i];
    st_val[base + i] = vals[i];
  }
  if (tid == 0) *row_nnz = total;
}

// Dense kernel: one CTA per row whose two crystals lie on opposite sides of
// the grid along x or z (generated rays only).  Every ray of such a row
// crosses the grid in the same direction along that slab axis and lies in
// the convex hull of the two crystal boxes, so the voxels its rays reach lie
// in per-slab windows, and the lengths are summed into dense slots of those
// windows: no key is stored, loaded or compared.  The voxels with a positive
// sum that pass the cylinder test are written in column order (x slabs are
// in column order already; z slabs are sorted).  A row that does not
// qualify, whose windows exceed dense_slots(H), or one of whose rays leaves
// its windows gets row_nnz = kRowToTable and is built by sm_table_kernel.
// Why the windows hold every voxel a ray visits: the hull bound is exact in
// real arithmetic, the walk visits voxels adjacent to the real ray's voxels
// at worst (rounding at plane ties), and the windows have a margin of one
// voxel on each side; the spare slot and the compaction's decode check
// catch a slot outside the windows' range regardless.
template <int H, int T, bool OISO>
__global__ void __launch_bounds__(T) sm_dense_kernel(DGeom g, const float2* __restrict__ sincos,
                                                     const int32_t* __restrict__ cnl_ids, int64_t row0, int nrays,
                                                     uint32_t seed, int32_t* __restrict__ st_col,
                                                     float* __restrict__ st_val, int32_t* __restrict__ row_nnz,
                                                     int32_t* __restrict__ flags, int32_t* __restrict__ reasons) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* acc = reinterpret_cast<float*>(smem);  // dense_slots(H) slots + the spare one
  int* keys = reinterpret_cast<int*>(smem);     // z slabs: the row's entries for the sort
  float* vals = reinterpret_cast<float*>(smem + H * sizeof(int));
  __shared__ Channel ch;
  __shared__ int bad_walk, dense_fail, win_u, win_v, sax, sdir;
  __shared__ float box_lo[2][3], box_hi[2][3];
  __shared__ int warp_sums[32];
  __shared__ int ulo[kMaxSlabs], vlo[kMaxSlabs], sbase[kMaxSlabs], sdk[kMaxSlabs];

  const int tid = threadIdx.x;
  const int64_t li = row0 + blockIdx.x;
  const int cnl = cnl_ids[li];
  if (cnl < 0 || cnl >= num_channels(g)) {
    if (tid == 0) {
      row_nnz[blockIdx.x] = -1;
      atomicOr(flags, 4);
    }
    return;
  }
  const int nyz = g.n[1] * g.n[2];
  const int nz = g.n[2];
  if (tid == 0) {
    channel_setup(g, sincos, cnl, ch);
    bad_walk = 0;
    dense_fail = 0;
    win_u = 0;
    win_v = 0;
    crystal_boxes(ch, box_lo, box_hi);
    // the slab axis: of x and z, the one along which the crystals lie on
    // opposite sides of the grid, the channel's dominant direction first
    // (its windows are the narrowest)
    int axis = -1, dir = 0;
    const int first = fabsf(ch.ab[0]) >= fabsf(ch.ab[2]) ? 0 : 2;
    for (int k = 0; k < 2 && axis < 0; k++) {
      const int a = k == 0 ? first : 2 - first;
      if (axis_n(g, a) > kMaxSlabs) continue;
      const float c0 = axis_o(g, a), c1 = axis_o(g, a) + float(axis_n(g, a)) * axis_d(g, a);
      const float m = 1e-6f * (1.0f + fabsf(c0) + fabsf(c1));
      if (box_hi[0][a] + m < c0 && box_lo[1][a] - m > c1) dir = 1;
      if (box_hi[1][a] + m < c0 && box_lo[0][a] - m > c1) dir = -1;
      if (dir != 0) axis = a;
    }
    sax = axis;
    sdir = dir;
  }
  __syncthreads();
  const int A = sax;
  if (A < 0) {
    if (tid == 0) {
      row_nnz[blockIdx.x] = kRowToTable;
      if (reasons) atomicAdd(reasons + 0, 1);
    }
    return;
  }
  const int iu_ax = A == 0 ? 1 : 0, iv_ax = A == 0 ? 2 : 1;
  const int na = axis_n(g, A);
  {
    const int p = sdir > 0 ? 0 : 1;  // the box at the lower coordinate along A
    for (int sl = tid; sl < na; sl += T) {
      const float c0 = axis_o(g, A) + float(sl) * axis_d(g, A), c1 = axis_o(g, A) + float(sl + 1) * axis_d(g, A);
      int u0, u1, v0, v1;
      slab_window(g, A, box_lo[p], box_hi[p], box_lo[1 - p], box_hi[1 - p], c0, c1, iu_ax, &u0, &u1);
      slab_window(g, A, box_lo[p], box_hi[p], box_lo[1 - p], box_hi[1 - p], c0, c1, iv_ax, &v0, &v1);
      ulo[sl] = u0;
      vlo[sl] = v0;
      atomicMax(&win_u, u1 - u0 + 1);
      atomicMax(&win_v, v1 - v0 + 1);
    }
  }
  __syncthreads();
  const int wu = win_u, wv = win_v;
  const int wuv = wu * wv;
  if (!((long long)na * wuv < (long long)dense_slots(H))) {  // + the spare slot
    if (tid == 0) {
      row_nnz[blockIdx.x] = kRowToTable;
      if (reasons) atomicAdd(reasons + 1, 1);
    }
    return;
  }
  const int nslots = na * wuv;
  for (int sl = tid; sl < na; sl += T) {
    const int b = sl * wuv - ulo[sl] * wv - vlo[sl];
    const int nb = sdir > 0 ? sl + 1 : sl - 1;
    const int bn = (nb >= 0 && nb < na) ? nb * wuv - ulo[nb] * wv - vlo[nb] : b;
    sbase[sl] = b;
    sdk[sl] = bn - b;
  }
  for (int i = tid; i <= nslots; i += T) acc[i] = 0.f;
  __syncthreads();

  {
    auto emit = [&](int ix, int iy, int iz, float L) {
      const int sa = A == 0 ? ix : iz;
      const int u = (A == 0 ? iy : ix) - ulo[sa], v = (A == 0 ? iz : iy) - vlo[sa];
      if (unsigned(u) < unsigned(wu) && unsigned(v) < unsigned(wv))
        atomicAdd(&acc[sa * wuv + u * wv + v], L);
      else
        dense_fail = 1;
    };
    // start offsets: the thread index bit-reversed, so that neighbouring
    // lanes start far apart along the ray
    const int part = int(__brev(threadIdx.x) >> 24);
    if (A == 0) {
      DenseIndex<0> dix{acc, sbase, sdk, wv, nslots};
      for (int ray = tid; ray < nrays; ray += T) {
        float r[6];
        make_ray(ch, seed, cnl, ray, r);
        if (sdir > 0 ? !(RFSUB(r[3], r[0]) > 0.f) : !(RFSUB(r[3], r[0]) < 0.f)) dense_fail = 1;
        walk_ray<OISO, dense_walk_unroll(H)>(g, ch, r, part, emit, dix, &bad_walk);
      }
    } else {
      DenseIndex<2> dix{acc, sbase, sdk, wv, nslots};
      for (int ray = tid; ray < nrays; ray += T) {
        float r[6];
        make_ray(ch, seed, cnl, ray, r);
        if (sdir > 0 ? !(RFSUB(r[5], r[2]) > 0.f) : !(RFSUB(r[5], r[2]) < 0.f)) dense_fail = 1;
        walk_ray<OISO, dense_walk_unroll(H)>(g, ch, r, part, emit, dix, &bad_walk);
      }
    }
  }
  __syncthreads();
  if (bad_walk) {
    if (tid == 0) {
      row_nnz[blockIdx.x] = -1;
      atomicOr(flags, 2);
    }
    return;
  }
  // a slot outside the windows was added to the spare slot: every thread
  // reads the same value and takes the same branch
  if (dense_fail || acc[nslots] != 0.f) {
    if (tid == 0) {
      row_nnz[blockIdx.x] = kRowToTable;
      if (reasons) atomicAdd(reasons + 2, 1);
    }
    return;
  }

  // Dense compaction layout: each warp takes a contiguous run of slots
  // (slab-major, then U, then V).
  constexpr int NW = T / 32;
  const int lane = tid & 31, w = tid >> 5;
  const int seg = ((nslots + NW - 1) / NW + 31) & ~31;
  const int b0 = min(w * seg, nslots), b1 = min(b0 + seg, nslots);
  auto voxel = [&](int slot, int* x, int* y, int* z) {
    const int sa = slot / wuv;
    const int rem = slot - sa * wuv;
    const int u = rem / wv;
    const int iu = ulo[sa] + u, iv = vlo[sa] + (rem - u * wv);
    *x = A == 0 ? sa : iu;
    *y = A == 0 ? iu : iv;
    *z = A == 0 ? iv : sa;
  };
  // First compaction pass: per warp, count the voxels with a positive sum
  // that pass the cylinder test and clear the others.  A positive slot that
  // decodes to a voxel outside the grid means the windows missed a voxel:
  // the row goes to the table kernel.
  {
    int cnt = 0;
    for (int b = b0; b < b1; b += 32) {
      const int slot = b + lane;
      bool keep = false;
      if (slot < b1) {
        const float v = acc[slot];
        if (v > 0.f) {
          int x, y, z;
          voxel(slot, &x, &y, &z);
          if (x < g.n[0] && y < g.n[1] && z < g.n[2]) {
            keep = candidate_test(g, ch, x, y, z);
          } else {
            dense_fail = 1;
          }
          if (!keep) acc[slot] = 0.f;
        }
      }
      cnt += __popc(__ballot_sync(0xffffffffu, keep));
    }
    if (lane == 0) warp_sums[w] = cnt;
  }
  __syncthreads();
  if (dense_fail) {
    if (tid == 0) {
      row_nnz[blockIdx.x] = kRowToTable;
      if (reasons) atomicAdd(reasons + 3, 1);
    }
    return;
  }
  // Second pass: after a scan of the warp counts, each warp writes its
  // voxels in slot order -- column order for x slabs; z slabs are sorted
  // below.
  const float fr = float(nrays);
  const size_t base = size_t(blockIdx.x) * H;
  int before = 0, total = 0;
  for (int k = 0; k < NW; k++) {
    const int c = warp_sums[k];
    before += k < w ? c : 0;
    total += c;
  }
  if (total > H) {
    if (tid == 0) {
      row_nnz[blockIdx.x] = -1;
      atomicOr(flags, 1);
    }
    return;
  }
  for (int b = b0; b < b1; b += 32) {
    const int slot = b + lane;
    const bool keep = slot < b1 && acc[slot] > 0.f;
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int pos = before + __popc(m & ((1u << lane) - 1u));
      int x, y, z;
      voxel(slot, &x, &y, &z);
      st_col[base + pos] = x * nyz + y * nz + z;
      st_val[base + pos] = RFDIV(acc[slot], fr);
    }
    before += __popc(m);
  }
  if (A == 0) {
    if (tid == 0) row_nnz[blockIdx.x] = total;
    return;
  }
  // z slabs: the entries ascend in z slab by slab, within a slab in (x, y).
  // Column order is (x, y, z): a counting sort by (x, y) over the box that
  // holds every slab's window places them, an entry's rank among the
  // entries of its (x, y) being the number of their z below its own (a z
  // bitmask per key).  When the box's counters do not fit beside the row's
  // staging in shared memory (or the grid has more than 96 z planes), the
  // bitonic sort does it.
  __shared__ int zbox[4];
  if (tid == 0) {
    zbox[0] = INT_MAX;
    zbox[1] = INT_MIN;
    zbox[2] = INT_MAX;
    zbox[3] = INT_MIN;
  }
  __syncthreads();
  for (int sl = tid; sl < na; sl += T) {
    atomicMin(&zbox[0], ulo[sl]);
    atomicMax(&zbox[1], ulo[sl] + wu);
    atomicMin(&zbox[2], vlo[sl]);
    atomicMax(&zbox[3], vlo[sl] + wv);
  }
  for (int i = tid; i < total; i += T) {
    keys[i] = st_col[base + i];
    vals[i] = st_val[base + i];
  }
  __syncthreads();
  const int wy = zbox[3] - zbox[2];
  const int nkeys = (zbox[1] - zbox[0]) * wy;
  constexpr int kKeyBytes = 16;  // counter + 96-bit z mask
  const int key_cap = int((row_smem_bytes(H) - size_t(H) * 8) / kKeyBytes);
  if (nkeys > key_cap || nz > 96) {
    sort_and_write<T>(keys, vals, total, st_col, st_val, base, row_nnz + blockIdx.x);
    return;
  }
  int* cnt = reinterpret_cast<int*>(smem + size_t(H) * 8);
  unsigned* zmask = reinterpret_cast<unsigned*>(cnt + nkeys);
  for (int i = tid; i < nkeys * 4; i += T) cnt[i] = 0;  // counters and masks
  __syncthreads();
  const int x0 = zbox[0], y0 = zbox[2];
  for (int i = tid; i < total; i += T) {
    const int c = keys[i];
    const int x = c / nyz, r = c - x * nyz, y = r / nz, z = r - y * nz;
    const int k = (x - x0) * wy + (y - y0);
    atomicAdd(&cnt[k], 1);
    atomicOr(&zmask[3 * k + (z >> 5)], 1u << (z & 31));
  }
  __syncthreads();
  // exclusive scan of the counters: each thread a run of consecutive keys
  {
    const int per = (nkeys + T - 1) / T;
    const int k0 = min(tid * per, nkeys), k1 = min(k0 + per, nkeys);
    int run = 0;
    for (int k = k0; k < k1; k++) run += cnt[k];
    int incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    int wbase = 0;
    for (int q = 0; q < w; q++) wbase += warp_sums[q];
    int off = wbase + incl - run;
    for (int k = k0; k < k1; k++) {
      const int c = cnt[k];
      cnt[k] = off;
      off += c;
    }
  }
  __syncthreads();
  for (int i = tid; i < total; i += T) {
    const int c = keys[i];
    const int x = c / nyz, r = c - x * nyz, y = r / nz, z = r - y * nz;
    const int k = (x - x0) * wy + (y - y0);
    const unsigned* m = zmask + 3 * k;
    const int zw = z >> 5;
    int rank = __popc(m[zw] & ((1u << (z & 31)) - 1u));
    if (zw > 0) rank += __popc(m[0]);
    if (zw > 1) rank += __popc(m[1]);
    st_col[base + cnt[k] + rank] = c;
    st_val[base + cnt[k] + rank] = vals[i];
  }
  if (tid == 0) row_nnz[blockIdx.x] = total;
}

// Table kernel: its rays (generated, or given in `rays`) summed per voxel in
// an open-addressing hash table of H keys in shared memory, then the voxels
// with a positive sum that pass the cylinder test sorted into column order.
// Each CTA takes rows blockIdx.x, blockIdx.x + gridDim.x, ... of the nrows.
// With only_flagged it builds only the rows the dense kernel left with
// kRowToTable and leaves the others alone (launched then with a small grid:
// most workloads leave none, and the blocks only read the row states).
template <int H, int T, bool OISO>
__global__ void __launch_bounds__(T) sm_table_kernel(DGeom g, const float2* __restrict__ sincos,
                                                     const int32_t* __restrict__ cnl_ids, int64_t row0, int64_t nrows,
                                                     int nrays, uint32_t seed, const float* __restrict__ rays,
                                                     int32_t* __restrict__ st_col, float* __restrict__ st_val,
                                                     int32_t* __restrict__ row_nnz, int32_t* __restrict__ flags,
                                                     int only_flagged) {
  extern __shared__ __align__(16) unsigned char smem[];
  int* keys = reinterpret_cast<int*>(smem);
  float* vals = reinterpret_cast<float*>(smem + H * sizeof(int));
  __shared__ Channel ch;
  __shared__ int overflow, bad_walk;
  __shared__ int warp_sums[32];

  const int tid = threadIdx.x;
  const int nyz = g.n[1] * g.n[2];
  const int nz = g.n[2];
  for (int64_t bi = blockIdx.x; bi < nrows; bi += gridDim.x) {
    if (only_flagged && row_nnz[bi] != kRowToTable) continue;
    const int64_t li = row0 + bi;
    const int cnl = cnl_ids[li];
    if (cnl < 0 || cnl >= num_channels(g)) {
      if (tid == 0) {
        row_nnz[bi] = -1;
        atomicOr(flags, 4);
      }
      continue;
    }
    __syncthreads();  // the previous row's use of the shared memory is over
    if (tid == 0) {
      channel_setup(g, sincos, cnl, ch);
      overflow = 0;
      bad_walk = 0;
    }
    for (int i = tid; i < H; i += T) {
      keys[i] = -1;
      vals[i] = 0.f;
    }
    __syncthreads();
    {
      RowTable<H> table{keys, vals, &overflow};
      KeyIndex<H> kix{&table, nyz, nz};
      auto emit = [&](int ix, int iy, int iz, float L) { table.add(ix * nyz + iy * nz + iz, L); };
      const int part = int(__brev(threadIdx.x) >> 24);
      for (int ray = tid; ray < nrays; ray += T) {
        float r[6];
        if (rays) {
          const float* src = rays + (li * int64_t(nrays) + ray) * 6;
#pragma unroll
          for (int k = 0; k < 6; k++) r[k] = src[k];
        } else {
          make_ray(ch, seed, cnl, ray, r);
        }
        walk_ray<OISO, 1>(g, ch, r, part, emit, kix, &bad_walk);
      }
    }
    __syncthreads();
    if (overflow || bad_walk) {
      if (tid == 0) {
        row_nnz[bi] = -1;
        atomicOr(flags, overflow ? 1 : 2);
      }
      continue;
    }
    // Compaction: keep voxels with a positive sum that pass the cylinder test.
    const float fr = float(nrays);
    constexpr int PER = H / T;
    int kr[PER];
    float vr[PER];
    int cnt = 0;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      int slot = j * T + tid;
      int key = keys[slot];
      float v = vals[slot];
      bool ok = key >= 0 && v > 0.f;
      if (ok) {
        int ix = key / nyz;
        int rem = key - ix * nyz;
        int iy = rem / nz;
        int iz = rem - iy * nz;
        ok = candidate_test(g, ch, ix, iy, iz);
      }
      kr[j] = ok ? key : -1;
      vr[j] = ok ? RFDIV(v, fr) : 0.f;
      cnt += ok ? 1 : 0;
    }
    int total = 0;
    int pos = block_exclusive_scan<T>(cnt, &total, warp_sums);
#pragma unroll
    for (int j = 0; j < PER; j++) {
      if (kr[j] >= 0) {
        keys[pos] = kr[j];
        vals[pos] = vr[j];
        pos++;
      }
    }
    sort_and_write<T>(keys, vals, total, st_col, st_val, size_t(bi) * H, row_nnz + bi);
  }
}

struct Level {
  int H, T;
};
constexpr Level kLevels[] = {{2048, 128}, {4096, 256}, {8192, 256}, {16384, 512}};
constexpr int kNumLevels = 4;

template <int H, int T>
cudaError_t launch_level(const DGeom& g, const float2* d_sincos, const int32_t* d_cnl, int64_t row0, int64_t nrows,
                         int nrays, uint32_t seed, const float* d_rays, int32_t* st_col, float* st_val,
                         int32_t* row_nnz, int32_t* d_flags, int32_t* d_reasons, int parts, cudaStream_t s) {
  // A grid with the same origin on every axis (the usual centred cube) lets
  // the walk's step skip selecting the origin.
  const bool oiso = g.o[0] == g.o[1] && g.o[1] == g.o[2];
  auto table = oiso ? sm_table_kernel<H, T, true> : sm_table_kernel<H, T, false>;
  const size_t table_smem = size_t(H) * 8;
  cudaError_t e = cudaFuncSetAttribute(table, cudaFuncAttributeMaxDynamicSharedMemorySize, int(table_smem));
  if (e != cudaSuccess) return e;
  if (d_rays) {
    // caller-supplied rays: the table builds every row, one CTA each
    table<<<unsigned(nrows), T, table_smem, s>>>(g, d_sincos, d_cnl, row0, nrows, nrays, seed, d_rays, st_col,
                                                  st_val, row_nnz, d_flags, 0);
    note_launches(1);
    return cudaGetLastError();
  }
  if (parts & 1) {
    auto dense = oiso ? sm_dense_kernel<H, T, true> : sm_dense_kernel<H, T, false>;
    const size_t dense_smem = row_smem_bytes(H);
    e = cudaFuncSetAttribute(dense, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dense_smem));
    if (e != cudaSuccess) return e;
    dense<<<unsigned(nrows), T, dense_smem, s>>>(g, d_sincos, d_cnl, row0, nrays, seed, st_col, st_val, row_nnz,
                                                 d_flags, d_reasons);
    note_launches(1);
  }
  if (parts & 2) {
    // the rows the dense kernel left to the table (a few per million on
    // the centred-cube workloads), four blocks per SM looking through the
    // row states
    const int64_t tb = std::min<int64_t>(nrows, 148 * 4);
    table<<<unsigned(tb), T, table_smem, s>>>(g, d_sincos, d_cnl, row0, nrows, nrays, seed, nullptr, st_col,
                                              st_val, row_nnz, d_flags, 1);
    note_launches(1);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// CSR placement
// ---------------------------------------------------------------------------

template <typename TCount>
__global__ void __launch_bounds__(1024) rows_scan_kernel(const TCount* __restrict__ row_nnz, int64_t n,
                                                         int64_t* __restrict__ row_ptr, int64_t* __restrict__ d_base) {
  __shared__ long long warp_sums[32];
  __shared__ long long carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry = *d_base;
  __syncthreads();
  for (int64_t t0 = 0; t0 < n; t0 += 1024) {
    int64_t i = t0 + tid;
    long long v = (i < n) ? (long long)row_nnz[i] : 0;
    v = v < 0 ? 0 : v;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      long long w = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    long long excl = carry + (warp > 0 ? warp_sums[warp - 1] : 0) + x - v;
    if (i < n) row_ptr[i] = excl;
    __syncthreads();
    if (tid == 0) carry += warp_sums[31];
    __syncthreads();
  }
  if (tid == 0) {
    row_ptr[n] = carry;
    *d_base = carry;
  }
}

__global__ void rows_gather_kernel(const int32_t* __restrict__ st_col, const float* __restrict__ st_val, int slot_cap,
                                   const int64_t* __restrict__ row_ptr, int64_t nrows, int64_t capacity,
                                   int32_t* __restrict__ col, float* __restrict__ val) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = w; r < nrows; r += nw) {
    const int64_t b = row_ptr[r], e = row_ptr[r + 1];
    const size_t src = size_t(r) * slot_cap;
    for (int64_t k = lane; k < e - b; k += 32) {
      if (b + k < capacity) {
        col[b + k] = st_col[src + k];
        val[b + k] = st_val[src + k];
      }
    }
  }
}

// For candidate k of row r (written by the workqueue fill in ascending
// voxel order), the value from the zero-free staged row, or 0.
__global__ void expand_kernel(const int32_t* __restrict__ st_col, const float* __restrict__ st_val, int slot_cap,
                              const int32_t* __restrict__ row_nnz, const int64_t* __restrict__ cand_ptr,
                              int64_t nrows, const int32_t* __restrict__ cand_vxl, float* __restrict__ out_val) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = w; r < nrows; r += nw) {
    const int64_t b = cand_ptr[r], e = cand_ptr[r + 1];
    const int32_t* rc = st_col + size_t(r) * slot_cap;
    const float* rv = st_val + size_t(r) * slot_cap;
    const int n = row_nnz[r];
    for (int64_t k = b + lane; k < e; k += 32) {
      int v = cand_vxl[k];
      int lo = 0, hi = n;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (rc[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      out_val[k] = (lo < n && rc[lo] == v) ? rv[lo] : 0.f;
    }
  }
}

__global__ void rays_kernel(DGeom g, const float2* __restrict__ sincos, const int32_t* __restrict__ cnl_ids,
                            int nrays, uint32_t seed, float* __restrict__ out) {
  __shared__ Channel ch;
  const int64_t li = blockIdx.x;
  const int cnl = cnl_ids[li];
  if (cnl < 0 || cnl >= num_channels(g)) {
    for (int64_t k = threadIdx.x; k < int64_t(nrays) * 6; k += blockDim.x) out[li * int64_t(nrays) * 6 + k] = NAN;
    return;
  }
  if (threadIdx.x == 0) channel_setup(g, sincos, cnl, ch);
  __syncthreads();
  for (int r = threadIdx.x; r < nrays; r += blockDim.x) {
    float v[6];
    make_ray(ch, seed, cnl, r, v);
    float* dst = out + (li * int64_t(nrays) + r) * 6;
#pragma unroll
    for (int k = 0; k < 6; k++) dst[k] = v[k];
  }
}

// ---------------------------------------------------------------------------
// Candidate search: one CTA per list entry, x-slab by x-slab; the voxel
// rows of a slab that can pass are flattened, tested 256 at a time and the
// passing voxels compacted in order with warp ballots.
// ---------------------------------------------------------------------------

constexpr int kWqThreads = 256;
constexpr int kWqMaxNy = 1024;

template <bool FILL>
__global__ void __launch_bounds__(kWqThreads) wq_kernel(DGeom g, const float2* __restrict__ sincos,
                                                        const int32_t* __restrict__ list, int64_t li0,
                                                        int64_t start_vxl, int64_t* __restrict__ counts,
                                                        const int64_t* __restrict__ offsets, int64_t max_out,
                                                        int32_t* __restrict__ out_cnl, int32_t* __restrict__ out_vxl,
                                                        int32_t* __restrict__ flags) {
  __shared__ Channel ch;
  __shared__ int zlo[kWqMaxNy];
  __shared__ int pre[kWqMaxNy + 1];
  __shared__ int warp_sums[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cnl = list[li0 + blockIdx.x];
  if (cnl < 0 || cnl >= num_channels(g)) {
    if (tid == 0) {
      if (!FILL) counts[blockIdx.x] = 0;
      if (flags) atomicOr(flags, 4);
    }
    return;
  }
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t nyz = int64_t(ny) * nz;
  int64_t start = (blockIdx.x == 0) ? start_vxl : 0;
  const int sx = int(start / nyz);
  const int sy = int((start % nyz) / nz);
  const int sz = int(start % nz);
  if (tid == 0) channel_setup(g, sincos, cnl, ch);
  __syncthreads();

  const int64_t out0 = FILL ? offsets[blockIdx.x] : 0;
  int64_t count = 0;
  for (int ix = sx; ix < nx; ix++) {
    if (FILL && out0 + count >= max_out) break;
    // Row intervals of this slab; thread t handles rows t, t+T, ...
    int local = 0;
    const int per = (ny + kWqThreads - 1) / kWqThreads;
    int lens[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      lens[q] = 0;
      int iy = tid * per + q;
      if (q < per && iy < ny) {
        int z0 = 0, z1 = -1;
        bool any = !(ix == sx && iy < sy) && row_z_interval(g, ch, ix, iy, &z0, &z1);
        if (any && ix == sx && iy == sy) z0 = max(z0, sz);
        int len = any ? max(z1 - z0 + 1, 0) : 0;
        zlo[iy] = z0;
        lens[q] = len;
        local += len;
      }
    }
    int total;
    int excl = block_exclusive_scan<kWqThreads>(local, &total, warp_sums);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int iy = tid * per + q;
      if (q < per && iy < ny) {
        pre[iy] = excl;
        excl += lens[q];
      }
    }
    if (tid == 0) pre[ny] = total;
    __syncthreads();
    for (int base = 0; base < total; base += kWqThreads) {
      int idx = base + tid;
      bool pass = false;
      int v = 0;
      if (idx < total) {
        int lo = 0, hi = ny;  // last row with pre[row] <= idx
        while (hi - lo > 1) {
          int mid = (lo + hi) >> 1;
          if (pre[mid] <= idx) lo = mid;
          else hi = mid;
        }
        int iy = lo;
        int iz = zlo[iy] + (idx - pre[iy]);
        pass = candidate_test(g, ch, ix, iy, iz);
        v = int(ix * nyz + int64_t(iy) * nz + iz);
      }
      unsigned bal = __ballot_sync(0xffffffffu, pass);
      if (lane == 0) warp_sums[warp] = __popc(bal);
      __syncthreads();
      int wpre = 0, btot = 0;
#pragma unroll
      for (int w = 0; w < kWqThreads / 32; w++) {
        int c = warp_sums[w];
        wpre += (w < warp) ? c : 0;
        btot += c;
      }
      if (FILL && pass) {
        int64_t p = out0 + count + wpre + __popc(bal & ((1u << lane) - 1u));
        if (p < max_out) {
          if (out_cnl) out_cnl[p] = cnl;
          out_vxl[p] = v;
        }
      }
      count += btot;
      __syncthreads();
    }
  }
  if (!FILL && tid == 0) counts[blockIdx.x] = count;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

int sm_num_levels() { return kNumLevels; }
int sm_level_capacity(int level) { return kLevels[level].H; }
int sm_level_threads(int level) { return kLevels[level].T; }

int sm_pick_level(const DGeom& g, int nrays) {
  long long span = (long long)g.n[0] + g.n[1] + g.n[2];
  if (nrays <= 128 && span <= 150) return 0;
  if (span <= 240) return 1;
  return 2;
}

cudaError_t launch_sm_rows(int level, const DGeom& g, const float2* d_sincos, const int32_t* d_cnl, int64_t row0,
                           int64_t nrows, int nrays, uint32_t seed, const float* d_rays, int32_t* st_col,
                           float* st_val, int32_t* row_nnz, int32_t* d_flags, cudaStream_t s,
                           int32_t* d_table_reasons, int parts) {
  if (nrows <= 0) return cudaSuccess;
  switch (level) {
    case 0: return launch_level<2048, 128>(g, d_sincos, d_cnl, row0, nrows, nrays, seed, d_rays, st_col, st_val, row_nnz, d_flags, d_table_reasons, parts, s);
    case 1: return launch_level<4096, 256>(g, d_sincos, d_cnl, row0, nrows, nrays, seed, d_rays, st_col, st_val, row_nnz, d_flags, d_table_reasons, parts, s);
    case 2: return launch_level<8192, 256>(g, d_sincos, d_cnl, row0, nrows, nrays, seed, d_rays, st_col, st_val, row_nnz, d_flags, d_table_reasons, parts, s);
    case 3: return launch_level<16384, 512>(g, d_sincos, d_cnl, row0, nrows, nrays, seed, d_rays, st_col, st_val, row_nnz, d_flags, d_table_reasons, parts, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_rows_scan(const int32_t* row_nnz, int64_t n, int64_t* row_ptr, int64_t* d_base, cudaStream_t s) {
  rows_scan_kernel<int32_t><<<1, 1024, 0, s>>>(row_nnz, n, row_ptr, d_base);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_rows_scan_i64(const int64_t* counts, int64_t n, int64_t* row_ptr, int64_t* d_base, cudaStream_t s) {
  rows_scan_kernel<int64_t><<<1, 1024, 0, s>>>(counts, n, row_ptr, d_base);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_rows_gather(const int32_t* st_col, const float* st_val, int slot_cap, const int64_t* row_ptr,
                               int64_t nrows, int64_t capacity, int32_t* col, float* val, cudaStream_t s) {
  if (nrows <= 0) return cudaSuccess;
  int64_t blocks = (nrows * 32 + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  rows_gather_kernel<<<unsigned(blocks), 256, 0, s>>>(st_col, st_val, slot_cap, row_ptr, nrows, capacity, col, val);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_expand_candidates(const int32_t* st_col, const float* st_val, int slot_cap, const int32_t* row_nnz,
                                     const int64_t* cand_ptr, int64_t nrows, int32_t* cand_vxl, float* out_val,
                                     cudaStream_t s) {
  if (nrows <= 0) return cudaSuccess;
  int64_t blocks = (nrows * 32 + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  expand_kernel<<<unsigned(blocks), 256, 0, s>>>(st_col, st_val, slot_cap, row_nnz, cand_ptr, nrows, cand_vxl,
                                                  out_val);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_rays(const DGeom& g, const float2* d_sincos, const int32_t* d_cnl, int64_t n, int nrays,
                        uint32_t seed, float* d_rays, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  rays_kernel<<<unsigned(n), 128, 0, s>>>(g, d_sincos, d_cnl, nrays, seed, d_rays);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_wq_count(const DGeom& g, const float2* d_sincos, const int32_t* d_list, int64_t li0, int64_t n,
                            int64_t start_vxl, int64_t* d_counts, int32_t* d_flags, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (g.n[1] > kWqMaxNy) return cudaErrorInvalidValue;
  wq_kernel<false><<<unsigned(n), kWqThreads, 0, s>>>(g, d_sincos, d_list, li0, start_vxl, d_counts, nullptr, 0,
                                                      nullptr, nullptr, d_flags);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_wq_fill(const DGeom& g, const float2* d_sincos, const int32_t* d_list, int64_t li0, int64_t n,
                           int64_t start_vxl, const int64_t* d_offsets, int64_t max_out, int32_t* d_cnl_out,
                           int32_t* d_vxl_out, int32_t* d_flags, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (g.n[1] > kWqMaxNy) return cudaErrorInvalidValue;
  wq_kernel<true><<<unsigned(n), kWqThreads, 0, s>>>(g, d_sincos, d_list, li0, start_vxl, nullptr, d_offsets,
                                                     max_out, d_cnl_out, d_vxl_out, d_flags);
  note_launches(1);
  return cudaGetLastError();
}

}  // namespace raptr
