// GPU voxelizer: voxelizeMeshToLattice (src/geometry/voxelizer.ts:86-281) on sm_100a.
//
// The BVH is built on the host with the reference's algorithm (bvh.ts:34-253: median
// split of the widest centroid extent, leaves of <= 4 triangles, children at
// consecutive indices) because the traversal order and node boxes decide which
// triangles a ray tests; the same tree on both sides makes the flags and link lists
// bit-exact.  The three passes run on the device in FP64 with no contraction (this
// file is compiled with -fmad=false):
//   1. one thread per (iy, iz) scanline of the mesh window: +X ray hits, sorted,
//      even counts fill [x_enter, x_exit], odd counts fall back to the 3-ray vote;
//   2. boundary detection over the window +-1, compacted in ascending cell order by
//      an exclusive scan;
//   3. one thread per (boundary cell, link): Bouzidi q by a segment query.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine_internal.h"

namespace aerosim {

namespace {

constexpr int kStack = 64;    // traversal stack depth (bvh.ts uses Int32Array(64))
constexpr int kMaxHits = 128; // scanline hits kept per ray

// ---------------------------------------------------------------------------
// Host BVH build, bvh.ts:34-253.
// ---------------------------------------------------------------------------
struct HostBvh {
  int tri_count = 0;
  std::vector<double> tri, nb, cen, tb;
  std::vector<int32_t> lof, cnt, tidx;
  double bmin[3] = {INFINITY, INFINITY, INFINITY};
  double bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  int next = 0;

  static double mn3(double a, double b, double c) { return js_min(js_min(a, b), c); }
  static double mx3(double a, double b, double c) { return js_max(js_max(a, b), c); }

  void node(int n, int first, int count) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = first; i < first + count; ++i) {
      const int t = tidx[i];
      for (int a = 0; a < 3; ++a) {
        if (tb[t * 6 + a] < lo[a]) lo[a] = tb[t * 6 + a];
        if (tb[t * 6 + 3 + a] > hi[a]) hi[a] = tb[t * 6 + 3 + a];
        const double c = cen[t * 3 + a];
        if (c < clo[a]) clo[a] = c;
        if (c > chi[a]) chi[a] = c;
      }
    }
    for (int a = 0; a < 3; ++a) {
      nb[n * 6 + a] = lo[a];
      nb[n * 6 + 3 + a] = hi[a];
    }
    if (count <= 4) {
      lof[n] = first;
      cnt[n] = count;
      return;
    }
    int axis = 0;
    double ext = chi[0] - clo[0], split = 0.5 * (clo[0] + chi[0]);
    if (chi[1] - clo[1] > ext) { axis = 1; ext = chi[1] - clo[1]; split = 0.5 * (clo[1] + chi[1]); }
    if (chi[2] - clo[2] > ext) { axis = 2; ext = chi[2] - clo[2]; split = 0.5 * (clo[2] + chi[2]); }
    if (ext <= 1e-12) {
      lof[n] = first;
      cnt[n] = count;
      return;
    }
    int i = first, j = first + count - 1;
    while (i <= j) {
      if (cen[tidx[i] * 3 + axis] < split) ++i;
      else std::swap(tidx[i], tidx[j--]);
    }
    int left = i - first;
    if (left == 0 || left == count) left = count >> 1;
    const int child = next;
    next += 2;
    lof[n] = child;
    cnt[n] = 0;
    node(child, first, left);
    node(child + 1, first + left, count - left);
  }

  void build(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx, const double* m) {
    tri_count = idx ? (int)(nidx / 3) : (int)(nverts / 3);
    tri.assign((size_t)tri_count * 9, 0.0);
    cen.assign((size_t)tri_count * 3, 0.0);
    tb.assign((size_t)tri_count * 6, 0.0);
    tidx.resize(tri_count);
    for (int t = 0; t < tri_count; ++t) {
      tidx[t] = t;
      double v[3][3];
      for (int k = 0; k < 3; ++k) {
        const int64_t vi = idx ? (int64_t)idx[t * 3 + k] : (int64_t)t * 3 + k;
        double x = pos[vi * 3], y = pos[vi * 3 + 1], z = pos[vi * 3 + 2];
        if (m) {  // THREE.Vector3.applyMatrix4 (column-major elements, perspective divide)
          const double w = 1.0 / (m[3] * x + m[7] * y + m[11] * z + m[15]);
          const double px = (m[0] * x + m[4] * y + m[8] * z + m[12]) * w;
          const double py = (m[1] * x + m[5] * y + m[9] * z + m[13]) * w;
          const double pz = (m[2] * x + m[6] * y + m[10] * z + m[14]) * w;
          x = px; y = py; z = pz;
        }
        v[k][0] = x; v[k][1] = y; v[k][2] = z;
      }
      for (int a = 0; a < 3; ++a) {
        tri[t * 9 + a] = v[0][a];
        tri[t * 9 + 3 + a] = v[1][a] - v[0][a];
        tri[t * 9 + 6 + a] = v[2][a] - v[0][a];
        cen[t * 3 + a] = (v[0][a] + v[1][a] + v[2][a]) / 3.0;
        tb[t * 6 + a] = mn3(v[0][a], v[1][a], v[2][a]);
        tb[t * 6 + 3 + a] = mx3(v[0][a], v[1][a], v[2][a]);
        if (tb[t * 6 + a] < bmin[a]) bmin[a] = tb[t * 6 + a];
        if (tb[t * 6 + 3 + a] > bmax[a]) bmax[a] = tb[t * 6 + 3 + a];
      }
    }
    const int nodes = std::max(1, tri_count * 2);
    nb.assign((size_t)nodes * 6, 0.0);
    lof.assign(nodes, 0);
    cnt.assign(nodes, 0);
    if (tri_count > 0) {
      next = 1;
      node(0, 0, tri_count);
    }
  }
};

struct BvhView {
  const double* tri;
  const double* nb;
  const int32_t* lof;
  const int32_t* cnt;
  const int32_t* tidx;
  int tri_count;
  double bmin[3], bmax[3];
};

enum { VOX_ERR_STACK = 1, VOX_ERR_HITS = 2 };

// bvh.ts:375-457 collectXScanlineHits (unsorted; the caller sorts).
__device__ int scanline_hits(const BvhView& b, double y, double z, double* hits, int* err) {
  if (b.tri_count == 0) return 0;
  const double py = y + 1.37e-8, pz = z + 2.93e-8;
  if (py < b.bmin[1] || py > b.bmax[1] || pz < b.bmin[2] || pz > b.bmax[2]) return 0;
  int stack[kStack];
  int sp = 0, n_hits = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const int n = stack[--sp];
    const double* nb = b.nb + (size_t)n * 6;
    if (py < nb[1] || py > nb[4] || pz < nb[2] || pz > nb[5]) continue;
    const int c = b.cnt[n];
    if (c > 0) {
      const int first = b.lof[n];
      for (int i = first; i < first + c; ++i) {
        const double* T = b.tri + (size_t)b.tidx[i] * 9;
        const double ax = T[0], ay = T[1], az = T[2];
        const double e1x = T[3], e1y = T[4], e1z = T[5];
        const double e2x = T[6], e2y = T[7], e2z = T[8];
        const double det = -e1y * e2z + e1z * e2y;
        if (fabs(det) < 1e-13) continue;
        const double inv = 1.0 / det;
        const double ty = py - ay, tz = pz - az;
        const double u = (-ty * e2z + tz * e2y) * inv;
        if (u < 0.0 || u > 1.0) continue;
        const double v = (ty * e1z - tz * e1y) * inv;
        if (v < 0.0 || u + v > 1.0) continue;
        if (n_hits < kMaxHits) hits[n_hits] = ax + u * e1x + v * e2x;
        else atomicOr(err, VOX_ERR_HITS);
        ++n_hits;
      }
    } else {
      if (sp + 2 > kStack) { atomicOr(err, VOX_ERR_STACK); return 0; }
      const int l = b.lof[n];
      stack[sp++] = l + 1;
      stack[sp++] = l;
    }
  }
  return n_hits < kMaxHits ? n_hits : kMaxHits;
}

// bvh.ts:499-589 countRayIntersections
__device__ int count_ray(const BvhView& b, double ox, double oy, double oz, double dx, double dy,
                         double dz, int* err) {
  const double ix = 1.0 / dx, iy = 1.0 / dy, iz = 1.0 / dz;
  int hits = 0;
  int stack[kStack];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const int n = stack[--sp];
    const double* nb = b.nb + (size_t)n * 6;
    const double tx1 = (nb[0] - ox) * ix, tx2 = (nb[3] - ox) * ix;
    double tmin = js_min(tx1, tx2), tmax = js_max(tx1, tx2);
    const double ty1 = (nb[1] - oy) * iy, ty2 = (nb[4] - oy) * iy;
    tmin = js_max(tmin, js_min(ty1, ty2));
    tmax = js_min(tmax, js_max(ty1, ty2));
    const double tz1 = (nb[2] - oz) * iz, tz2 = (nb[5] - oz) * iz;
    tmin = js_max(tmin, js_min(tz1, tz2));
    tmax = js_min(tmax, js_max(tz1, tz2));
    if (tmax < js_max(0, tmin)) continue;
    const int c = b.cnt[n];
    if (c > 0) {
      const int first = b.lof[n];
      for (int i = first; i < first + c; ++i) {
        const double* T = b.tri + (size_t)b.tidx[i] * 9;
        const double ax = T[0], ay = T[1], az = T[2];
        const double e1x = T[3], e1y = T[4], e1z = T[5];
        const double e2x = T[6], e2y = T[7], e2z = T[8];
        const double px = dy * e2z - dz * e2y;
        const double py = dz * e2x - dx * e2z;
        const double pz = dx * e2y - dy * e2x;
        const double det = e1x * px + e1y * py + e1z * pz;
        if (fabs(det) < 1e-13) continue;
        const double inv = 1.0 / det;
        const double tx = ox - ax, ty = oy - ay, tz = oz - az;
        const double u = (tx * px + ty * py + tz * pz) * inv;
        if (u < 0.0 || u > 1.0) continue;
        const double qx = ty * e1z - tz * e1y;
        const double qy = tz * e1x - tx * e1z;
        const double qz = tx * e1y - ty * e1x;
        const double v = (dx * qx + dy * qy + dz * qz) * inv;
        if (v < 0.0 || u + v > 1.0) continue;
        const double t = (e2x * qx + e2y * qy + e2z * qz) * inv;
        if (t > 1e-7) ++hits;
      }
    } else {
      if (sp + 2 > kStack) { atomicOr(err, VOX_ERR_STACK); return 0; }
      const int l = b.lof[n];
      stack[sp++] = l + 1;
      stack[sp++] = l;
    }
  }
  return hits;
}

// bvh.ts:464-497 isPointInside: 3 skew rays, 2-of-3 parity vote.
__device__ bool point_inside(const BvhView& b, double x, double y, double z, int* err) {
  if (x < b.bmin[0] || x > b.bmax[0] || y < b.bmin[1] || y > b.bmax[1] || z < b.bmin[2] ||
      z > b.bmax[2])
    return false;
  const double D[3][3] = {{1.0, 0.0137, 0.0293}, {-0.0191, 1.0, 0.0317}, {0.0239, -0.0173, 1.0}};
  int votes = 0;
  for (int d = 0; d < 3; ++d) {
    if ((count_ray(b, x, y, z, D[d][0], D[d][1], D[d][2], err) & 1) == 1) ++votes;
    if (votes >= 2) return true;
    if (d == 1 && votes == 0) return false;
  }
  return votes >= 2;
}

// bvh.ts:265-367 intersectSegment
__device__ double segment(const BvhView& b, double ox, double oy, double oz, double dx, double dy,
                          double dz, double maxT, int* err) {
  if (b.tri_count == 0) return -1;
  const double ix = fabs(dx) > 1e-15 ? 1.0 / dx : (dx >= 0 ? 1e15 : -1e15);
  const double iy = fabs(dy) > 1e-15 ? 1.0 / dy : (dy >= 0 ? 1e15 : -1e15);
  const double iz = fabs(dz) > 1e-15 ? 1.0 / dz : (dz >= 0 ? 1e15 : -1e15);
  double closest = maxT + 1e-7;
  bool found = false;
  int stack[kStack];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const int n = stack[--sp];
    const double* nb = b.nb + (size_t)n * 6;
    const double tx1 = (nb[0] - ox) * ix, tx2 = (nb[3] - ox) * ix;
    double tmin = js_min(tx1, tx2), tmax = js_max(tx1, tx2);
    const double ty1 = (nb[1] - oy) * iy, ty2 = (nb[4] - oy) * iy;
    tmin = js_max(tmin, js_min(ty1, ty2));
    tmax = js_min(tmax, js_max(ty1, ty2));
    const double tz1 = (nb[2] - oz) * iz, tz2 = (nb[5] - oz) * iz;
    tmin = js_max(tmin, js_min(tz1, tz2));
    tmax = js_min(tmax, js_max(tz1, tz2));
    if (tmax < js_max(0, tmin) || tmin > closest) continue;
    const int c = b.cnt[n];
    if (c > 0) {
      const int first = b.lof[n];
      for (int i = first; i < first + c; ++i) {
        const double* T = b.tri + (size_t)b.tidx[i] * 9;
        const double ax = T[0], ay = T[1], az = T[2];
        const double e1x = T[3], e1y = T[4], e1z = T[5];
        const double e2x = T[6], e2y = T[7], e2z = T[8];
        const double px = dy * e2z - dz * e2y;
        const double py = dz * e2x - dx * e2z;
        const double pz = dx * e2y - dy * e2x;
        const double det = e1x * px + e1y * py + e1z * pz;
        if (fabs(det) < 1e-13) continue;
        const double inv = 1.0 / det;
        const double tx = ox - ax, ty = oy - ay, tz = oz - az;
        const double u = (tx * px + ty * py + tz * pz) * inv;
        if (u < -1e-7 || u > 1.0 + 1e-7) continue;
        const double qx = ty * e1z - tz * e1y;
        const double qy = tz * e1x - tx * e1z;
        const double qz = tx * e1y - ty * e1x;
        const double v = (dx * qx + dy * qy + dz * qz) * inv;
        if (v < -1e-7 || u + v > 1.0 + 1e-7) continue;
        const double t = (e2x * qx + e2y * qy + e2z * qz) * inv;
        if (t > 1e-7 && t <= closest) {
          closest = t;
          found = true;
        }
      }
    } else {
      if (sp + 2 > kStack) { atomicOr(err, VOX_ERR_STACK); return -1; }
      const int l = b.lof[n];
      stack[sp++] = l + 1;
      stack[sp++] = l;
    }
  }
  return found ? js_min(maxT, closest) : -1;
}

struct Lattice {
  int nx, ny, nz;
  double h, ox, oy, oz;
  int w[6];  // mesh window minIx, maxIx, minIy, maxIy, minIz, maxIz
};

// STEP 1, voxelizer.ts:127-173.  One thread per (iy, iz) of the window.
__global__ void scan_fill_kernel(BvhView b, Lattice L, uint8_t* flags,
                                 unsigned long long* solid_count, int* err) {
  const int wy = L.w[3] - L.w[2] + 1, wz = L.w[5] - L.w[4] + 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)wy * wz) return;
  const int iy = L.w[2] + (int)(t % wy), iz = L.w[4] + (int)(t / wy);
  const double z = L.oz + (iz + 0.5) * L.h;
  const double y = L.oy + (iy + 0.5) * L.h;
  double hits[kMaxHits];
  const int hc = scanline_hits(b, y, z, hits, err);
  if (hc == 0) return;
  for (int i = 1; i < hc; ++i) {  // ascending numeric sort
    const double key = hits[i];
    int j = i - 1;
    while (j >= 0 && hits[j] > key) { hits[j + 1] = hits[j]; --j; }
    hits[j + 1] = key;
  }
  uint8_t* row = flags + (long long)L.nx * (iy + (long long)L.ny * iz);
  unsigned long long added = 0;
  const int minIx = L.w[0], maxIx = L.w[1];
  if ((hc & 1) == 0) {
    for (int k = 0; k < hc; k += 2) {
      const double xe = hits[k], xx = hits[k + 1];
      if (xx - xe < 1e-7) continue;
      const double s = js_max((double)minIx, ceil((xe - L.ox) / L.h - 0.5));
      const double e = js_min((double)maxIx, floor((xx - L.ox) / L.h - 0.5));
      if (!(s <= e)) continue;
      for (int ix = (int)s; ix <= (int)e; ++ix) {
        if (row[ix] == CELL_FLUID) {
          row[ix] = CELL_SOLID;
          ++added;
        }
      }
    }
  } else {
    for (int ix = minIx; ix <= maxIx; ++ix) {
      const double x = L.ox + (ix + 0.5) * L.h;
      if (x >= hits[0] && x <= hits[hc - 1]) {
        if (point_inside(b, x, y, z, err) && row[ix] == CELL_FLUID) {
          row[ix] = CELL_SOLID;
          ++added;
        }
      }
    }
  }
  if (added) atomicAdd(solid_count, added);
}

// STEP 2, voxelizer.ts:176-212: mark FLUID cells with an in-bounds SOLID neighbour.
__global__ void boundary_mark_kernel(const uint8_t* __restrict__ flags, Lattice L, int sx0, int sy0,
                                     int sz0, int wx, int wy, long long wn,
                                     uint32_t* __restrict__ mark) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= wn) return;
  const int ix = sx0 + (int)(t % wx);
  const long long r = t / wx;
  const int iy = sy0 + (int)(r % wy), iz = sz0 + (int)(r / wy);
  const long long i = ix + (long long)L.nx * (iy + (long long)L.ny * iz);
  uint32_t m = 0;
  if (flags[i] == CELL_FLUID) {
#pragma unroll
    for (int d = 1; d < 19; ++d) {
      const int a = ix + cx_of(d), bb = iy + cy_of(d), c = iz + cz_of(d);
      if (a < 0 || a >= L.nx || bb < 0 || bb >= L.ny || c < 0 || c >= L.nz) continue;
      if (flags[a + (long long)L.nx * (bb + (long long)L.ny * c)] == CELL_SOLID) m = 1;
    }
  }
  mark[t] = m;
}

// Exclusive scan, tiles of 2048 (512 threads x 4 items).
__global__ void scan_tiles_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                  uint32_t* __restrict__ tile_sums, long long n) {
  __shared__ uint32_t s[512];
  const long long base = (long long)blockIdx.x * 2048 + threadIdx.x * 4;
  uint32_t v[4], acc = 0;
  for (int k = 0; k < 4; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0u;
    acc += v[k];
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 1; o < 512; o <<= 1) {  // Hillis-Steele inclusive scan of thread sums
    const uint32_t add = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
    __syncthreads();
    s[threadIdx.x] += add;
    __syncthreads();
  }
  uint32_t run = s[threadIdx.x] - acc;
  for (int k = 0; k < 4; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 511) tile_sums[blockIdx.x] = s[511];
}

__global__ void scan_sums_kernel(uint32_t* sums, long long nt, uint32_t* total) {
  __shared__ uint32_t s[1024];
  uint32_t carry = 0;
  for (long long b0 = 0; b0 < nt; b0 += 1024) {
    const long long i = b0 + threadIdx.x;
    const uint32_t v = i < nt ? sums[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const uint32_t add = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
      __syncthreads();
      s[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < nt) sums[i] = carry + s[threadIdx.x] - v;
    const uint32_t block_total = s[1023];
    __syncthreads();
    carry += block_total;
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_add_kernel(uint32_t* out, const uint32_t* sums, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / 2048];
}

__global__ void boundary_scatter_kernel(uint8_t* flags, Lattice L, int sx0, int sy0, int sz0,
                                        int wx, int wy, long long wn,
                                        const uint32_t* __restrict__ mark,
                                        const uint32_t* __restrict__ pos, int32_t* bcells,
                                        int32_t* bmap) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= wn || !mark[t]) return;
  const int ix = sx0 + (int)(t % wx);
  const long long r = t / wx;
  const int iy = sy0 + (int)(r % wy), iz = sz0 + (int)(r / wy);
  const long long i = ix + (long long)L.nx * (iy + (long long)L.ny * iz);
  const uint32_t b = pos[t];
  flags[i] = CELL_BOUNDARY;
  bcells[b] = (int32_t)i;
  bmap[i] = (int32_t)b;
}

// STEP 3, voxelizer.ts:221-256 (+ computeSubGridLinkFraction :65-80).
__global__ void q_links_kernel(BvhView bv, Lattice L, const uint8_t* __restrict__ flags,
                               const int32_t* __restrict__ bcells, long long B, float* q, int* err) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * 18) return;
  const long long b = t / 18;
  const int d = (int)(t % 18) + 1;
  const long long ci = bcells[b];
  const int ix = (int)(ci % L.nx);
  const long long rem = (ci - ix) / L.nx;
  const int iy = (int)(rem % L.ny);
  const int iz = (int)((rem - iy) / L.ny);
  const int a = ix + cx_of(d), bb = iy + cy_of(d), c = iz + cz_of(d);
  float out = -1.0f;
  if (!(a < 0 || a >= L.nx || bb < 0 || bb >= L.ny || c < 0 || c >= L.nz) &&
      flags[a + (long long)L.nx * (bb + (long long)L.ny * c)] == CELL_SOLID) {
    const double fx = L.ox + (ix + 0.5) * L.h, fy = L.oy + (iy + 0.5) * L.h,
                 fz = L.oz + (iz + 0.5) * L.h;
    const double tq = segment(bv, fx, fy, fz, cx_of(d) * L.h, cy_of(d) * L.h, cz_of(d) * L.h, 1.0, err);
    double qv = 0.5;
    if (tq > 0 && tq <= 1.0) qv = js_max(1e-4, js_min(1.0, tq));
    out = (float)qv;
  }
  q[t] = out;
}

__global__ void min_q_kernel(const float* __restrict__ q, long long B, float* minq) {
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  float m = 1.0f;
  for (int k = 0; k < 18; ++k) {
    const float v = q[b * 18 + k];
    if (v > 0.0f && v < m) m = v;
  }
  minq[b] = m;
}

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
}

}  // namespace

#define VCHECK(x)                                                              \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      *err = std::string("voxelizer: ") + #x + ": " + cudaGetErrorString(e_);  \
      goto fail;                                                               \
    }                                                                          \
  } while (0)

int run_voxelizer(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx,
                  const double* world16, double tunnel_height, int nx, int ny, int nz,
                  cudaStream_t s, DevGrid* g, std::string* err) {
  const auto t0 = std::chrono::steady_clock::now();
  HostBvh hb;
  hb.build(pos, nverts, idx, nidx, world16);
  const long long N = (long long)nx * ny * nz;
  const double h = tunnel_height / ny;
  Lattice L{nx, ny, nz, h, -nx * h * 0.5, -ny * h * 0.5, -nz * h * 0.5, {0, 0, 0, 0, 0, 0}};
  double* d_tri = nullptr;
  double* d_nb = nullptr;
  int32_t *d_lof = nullptr, *d_cnt = nullptr, *d_tidx = nullptr;
  uint32_t *d_mark = nullptr, *d_pos = nullptr, *d_sums = nullptr, *d_total = nullptr;
  unsigned long long* d_solid = nullptr;
  int* d_err = nullptr;
  int rc = -3;
  BvhView bv{};
  long long wn = 0, ntile = 0;
  int sx0 = 0, sy0 = 0, sz0 = 0, wx = 0, wy = 0, wz = 0;
  uint32_t B = 0;
  unsigned long long solid = 0;
  int herr = 0;

  g->nx = nx; g->ny = ny; g->nz = nz; g->N = N;
  g->h = h; g->ox = L.ox; g->oy = L.oy; g->oz = L.oz;
  {
    auto fl = [](double v) { return (int)std::floor(v); };
    auto cl = [](double v) { return (int)std::ceil(v); };
    L.w[0] = std::max(0, fl((hb.bmin[0] - L.ox) / h) - 1);
    L.w[1] = std::min(nx - 1, cl((hb.bmax[0] - L.ox) / h) + 1);
    L.w[2] = std::max(0, fl((hb.bmin[1] - L.oy) / h) - 1);
    L.w[3] = std::min(ny - 1, cl((hb.bmax[1] - L.oy) / h) + 1);
    L.w[4] = std::max(0, fl((hb.bmin[2] - L.oz) / h) - 1);
    L.w[5] = std::min(nz - 1, cl((hb.bmax[2] - L.oz) / h) + 1);
  }
  VCHECK(dalloc(&g->flags, N));
  VCHECK(dalloc(&g->bmap, N));
  VCHECK(cudaMemsetAsync(g->flags, 0, N, s));
  VCHECK(cudaMemsetAsync(g->bmap, 0xff, N * sizeof(int32_t), s));
  VCHECK(dalloc(&d_solid, 1));
  VCHECK(dalloc(&d_err, 1));
  VCHECK(dalloc(&d_total, 1));
  VCHECK(cudaMemsetAsync(d_solid, 0, sizeof(unsigned long long), s));
  VCHECK(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  VCHECK(cudaMemsetAsync(d_total, 0, sizeof(uint32_t), s));
  if (hb.tri_count > 0) {
    VCHECK(dalloc(&d_tri, hb.tri.size()));
    VCHECK(dalloc(&d_nb, hb.nb.size()));
    VCHECK(dalloc(&d_lof, hb.lof.size()));
    VCHECK(dalloc(&d_cnt, hb.cnt.size()));
    VCHECK(dalloc(&d_tidx, hb.tidx.size()));
    VCHECK(cudaMemcpyAsync(d_tri, hb.tri.data(), hb.tri.size() * 8, cudaMemcpyHostToDevice, s));
    VCHECK(cudaMemcpyAsync(d_nb, hb.nb.data(), hb.nb.size() * 8, cudaMemcpyHostToDevice, s));
    VCHECK(cudaMemcpyAsync(d_lof, hb.lof.data(), hb.lof.size() * 4, cudaMemcpyHostToDevice, s));
    VCHECK(cudaMemcpyAsync(d_cnt, hb.cnt.data(), hb.cnt.size() * 4, cudaMemcpyHostToDevice, s));
    VCHECK(cudaMemcpyAsync(d_tidx, hb.tidx.data(), hb.tidx.size() * 4, cudaMemcpyHostToDevice, s));
    bv = BvhView{d_tri, d_nb, d_lof, d_cnt, d_tidx, hb.tri_count,
                 {hb.bmin[0], hb.bmin[1], hb.bmin[2]}, {hb.bmax[0], hb.bmax[1], hb.bmax[2]}};
    // STEP 1 (window may be empty when the mesh lies outside the lattice)
    const long long rows = (long long)(L.w[3] - L.w[2] + 1) * (L.w[5] - L.w[4] + 1);
    if (L.w[0] <= L.w[1] && L.w[2] <= L.w[3] && L.w[4] <= L.w[5] && rows > 0) {
      scan_fill_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(bv, L, g->flags, d_solid, d_err);
      VCHECK(cudaGetLastError());
    }
    // STEP 2
    sx0 = std::max(0, L.w[0] - 1); sy0 = std::max(0, L.w[2] - 1); sz0 = std::max(0, L.w[4] - 1);
    wx = std::min(nx - 1, L.w[1] + 1) - sx0 + 1;
    wy = std::min(ny - 1, L.w[3] + 1) - sy0 + 1;
    wz = std::min(nz - 1, L.w[5] + 1) - sz0 + 1;
    wn = (wx > 0 && wy > 0 && wz > 0) ? (long long)wx * wy * wz : 0;
    if (wn > 0) {
      ntile = (wn + 2047) / 2048;
      VCHECK(dalloc(&d_mark, wn));
      VCHECK(dalloc(&d_pos, wn));
      VCHECK(dalloc(&d_sums, ntile));
      boundary_mark_kernel<<<(unsigned)((wn + 255) / 256), 256, 0, s>>>(g->flags, L, sx0, sy0, sz0, wx, wy, wn, d_mark);
      scan_tiles_kernel<<<(unsigned)ntile, 512, 0, s>>>(d_mark, d_pos, d_sums, wn);
      scan_sums_kernel<<<1, 1024, 0, s>>>(d_sums, ntile, d_total);
      scan_add_kernel<<<(unsigned)((wn + 255) / 256), 256, 0, s>>>(d_pos, d_sums, wn);
      VCHECK(cudaGetLastError());
    }
  }
  VCHECK(cudaMemcpyAsync(&B, d_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  VCHECK(cudaMemcpyAsync(&solid, d_solid, sizeof(solid), cudaMemcpyDeviceToHost, s));
  VCHECK(cudaStreamSynchronize(s));
  g->B = B;
  g->solid = (long long)solid;
  VCHECK(dalloc(&g->bcells, B));
  VCHECK(dalloc(&g->q, (size_t)B * 18));
  VCHECK(dalloc(&g->minq, B));
  if (B > 0) {
    boundary_scatter_kernel<<<(unsigned)((wn + 255) / 256), 256, 0, s>>>(g->flags, L, sx0, sy0, sz0, wx, wy, wn, d_mark, d_pos, g->bcells, g->bmap);
    // STEP 3
    const long long links = (long long)B * 18;
    q_links_kernel<<<(unsigned)((links + 127) / 128), 128, 0, s>>>(bv, L, g->flags, g->bcells, B, g->q, d_err);
    min_q_kernel<<<(unsigned)((B + 255) / 256), 256, 0, s>>>(g->q, B, g->minq);
    VCHECK(cudaGetLastError());
  }
  VCHECK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  VCHECK(cudaStreamSynchronize(s));
  if (herr) {
    *err = (herr & VOX_ERR_STACK) ? "voxelizer: BVH deeper than the 64-entry traversal stack"
                                  : "voxelizer: more than 128 hits on one scanline";
    rc = -4;
    goto fail;
  }
  g->window[0] = L.w[0]; g->window[1] = L.w[1]; g->window[2] = L.w[2];
  g->window[3] = L.w[3]; g->window[4] = L.w[4]; g->window[5] = L.w[5];
  g->vox_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  rc = 0;
fail:
  cudaFree(d_tri); cudaFree(d_nb); cudaFree(d_lof); cudaFree(d_cnt); cudaFree(d_tidx);
  cudaFree(d_mark); cudaFree(d_pos); cudaFree(d_sums); cudaFree(d_total);
  cudaFree(d_solid); cudaFree(d_err);
  return rc;
}

}  // namespace aerosim
