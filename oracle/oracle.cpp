// CPU oracle for the AeroSim solver hot path -- TEST INFRASTRUCTURE ONLY.
//
// This file is a C++17 restatement of the reference's single-threaded TypeScript
// CPU path. It exists so that tests, the smoke check and the benchmark's CPU
// baseline leg can compare the CUDA library against the reference algorithm.
// Nothing in the product (aerosim_b200/, include/) links or calls it.
//
// Restated reference files (paths inside the reference project):
//   src/solver/lbmConstants.ts:10-66,142-152   D3Q19 tables, computeEquilibrium
//   src/geometry/bvh.ts:34-589                 MeshBVH (build, segment, scanline, vote)
//   src/geometry/voxelizer.ts:65-281           computeSubGridLinkFraction, voxelizeMeshToLattice
//   src/solver/lbmCpuReference.ts:76-495       LBMCpuReferenceSolver
//   src/solver/forceIntegrator.ts:57-315       surface area, momentum exchange, coefficients
//   src/geometry/frontalArea.ts:22-179         computeProjectedFrontalArea
//
// Parity pinning: the reference is TypeScript and no JavaScript runtime exists
// on the build or GPU machines, so the reference itself cannot be executed to
// produce golden vectors. This restatement is pinned by the reference's own
// known-answer tests (solid-cell count of the 1 m cube, non-manifold vote,
// analytic-sphere q error, link consistency, zero-inflow force, mass
// conservation, Strouhal band, Cd bands) which the test suite re-runs against it.
//
// Precision rules that mirror the JavaScript semantics exactly:
//   * every scalar is IEEE double, every typed-array store is float;
//   * LBM_WEIGHTS_F32 (float weights promoted to double) in the collision and the
//     force integrator, exact double weights in computeEquilibrium (boundaries);
//   * no floating-point contraction (build with -ffp-contract=off);
//   * Math.min / Math.max propagate NaN (js_min / js_max below).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// lbmConstants.ts:10-48
const int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
const int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};

// lbmConstants.ts:56-63 (LBM_WEIGHTS and its Float32Array copy)
double W64[19];
double W32[19];  // float-rounded weights promoted back to double
struct WeightInit {
  WeightInit() {
    for (int d = 0; d < 19; ++d) {
      W64[d] = d == 0 ? 1.0 / 3.0 : (d <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
      W32[d] = (double)(float)W64[d];
    }
  }
} weight_init;

const uint8_t CELL_FLUID = 0, CELL_SOLID = 1, CELL_BOUNDARY = 2;

inline double js_min(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return NAN;
  return a < b ? a : b;
}
inline double js_max(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return NAN;
  return a > b ? a : b;
}
inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// lbmConstants.ts:142-152 computeEquilibrium (double weights)
inline double feq64(int d, double rho, double ux, double uy, double uz) {
  const double cu = 3.0 * ((double)CX[d] * ux + (double)CY[d] * uy + (double)CZ[d] * uz);
  const double uSq = ux * ux + uy * uy + uz * uz;
  return W64[d] * rho * (1.0 + cu + 0.5 * cu * cu - 1.5 * uSq);
}

// ---------------------------------------------------------------------------
// bvh.ts -- MeshBVH
// ---------------------------------------------------------------------------
struct BVH {
  int tri_count = 0;
  std::vector<double> tri;  // 9 per triangle: A, E1, E2
  std::vector<double> node_bounds;
  std::vector<int32_t> node_left_or_first, node_tri_count, tri_indices;
  double bmin[3] = {INFINITY, INFINITY, INFINITY};
  double bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  int node_ptr = 0;

  // bvh.ts:141-253 buildNode
  void build_node(int node, int first, int count, const std::vector<double>& cen,
                  const std::vector<double>& tb) {
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    double cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = first; i < first + count; ++i) {
      const int t = tri_indices[i];
      for (int a = 0; a < 3; ++a) {
        if (tb[t * 6 + a] < mn[a]) mn[a] = tb[t * 6 + a];
        if (tb[t * 6 + 3 + a] > mx[a]) mx[a] = tb[t * 6 + 3 + a];
      }
      for (int a = 0; a < 3; ++a) {
        const double c = cen[t * 3 + a];
        if (c < cmn[a]) cmn[a] = c;
        if (c > cmx[a]) cmx[a] = c;
      }
    }
    for (int a = 0; a < 3; ++a) {
      node_bounds[node * 6 + a] = mn[a];
      node_bounds[node * 6 + 3 + a] = mx[a];
    }
    if (count <= 4) {
      node_left_or_first[node] = first;
      node_tri_count[node] = count;
      return;
    }
    const double ext[3] = {cmx[0] - cmn[0], cmx[1] - cmn[1], cmx[2] - cmn[2]};
    int axis = 0;
    double split = 0.5 * (cmn[0] + cmx[0]);
    double max_ext = ext[0];
    if (ext[1] > max_ext) { axis = 1; max_ext = ext[1]; split = 0.5 * (cmn[1] + cmx[1]); }
    if (ext[2] > max_ext) { axis = 2; max_ext = ext[2]; split = 0.5 * (cmn[2] + cmx[2]); }
    if (max_ext <= 1e-12) {
      node_left_or_first[node] = first;
      node_tri_count[node] = count;
      return;
    }
    int i = first, j = first + count - 1;
    while (i <= j) {
      const int t = tri_indices[i];
      if (cen[t * 3 + axis] < split) {
        ++i;
      } else {
        std::swap(tri_indices[i], tri_indices[j]);
        --j;
      }
    }
    int left = i - first;
    if (left == 0 || left == count) left = count >> 1;
    const int lc = node_ptr;
    node_ptr += 2;
    node_left_or_first[node] = lc;
    node_tri_count[node] = 0;
    build_node(lc, first, left, cen, tb);
    build_node(lc + 1, first + left, count - left, cen, tb);
  }

  // bvh.ts:34-139 constructor. Positions are float (BufferGeometry), promoted to
  // double; the optional world matrix is column-major like THREE.Matrix4.elements
  // and applied with Vector3.applyMatrix4's perspective divide.
  BVH(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx, const double* m) {
    tri_count = idx ? (int)(nidx / 3) : (int)(nverts / 3);
    tri.assign((size_t)tri_count * 9, 0.0);
    tri_indices.resize(tri_count);
    std::vector<double> cen((size_t)tri_count * 3), tb((size_t)tri_count * 6);
    for (int t = 0; t < tri_count; ++t) {
      tri_indices[t] = t;
      int64_t vi[3];
      for (int k = 0; k < 3; ++k) vi[k] = idx ? idx[t * 3 + k] : (int64_t)t * 3 + k;
      double v[3][3];
      for (int k = 0; k < 3; ++k) {
        double x = pos[vi[k] * 3], y = pos[vi[k] * 3 + 1], z = pos[vi[k] * 3 + 2];
        if (m) {
          const double w = 1.0 / (m[3] * x + m[7] * y + m[11] * z + m[15]);
          const double nx = (m[0] * x + m[4] * y + m[8] * z + m[12]) * w;
          const double ny = (m[1] * x + m[5] * y + m[9] * z + m[13]) * w;
          const double nz = (m[2] * x + m[6] * y + m[10] * z + m[14]) * w;
          x = nx; y = ny; z = nz;
        }
        v[k][0] = x; v[k][1] = y; v[k][2] = z;
      }
      for (int a = 0; a < 3; ++a) {
        tri[t * 9 + a] = v[0][a];
        tri[t * 9 + 3 + a] = v[1][a] - v[0][a];
        tri[t * 9 + 6 + a] = v[2][a] - v[0][a];
        cen[t * 3 + a] = (v[0][a] + v[1][a] + v[2][a]) / 3.0;
        const double lo = js_min(js_min(v[0][a], v[1][a]), v[2][a]);
        const double hi = js_max(js_max(v[0][a], v[1][a]), v[2][a]);
        tb[t * 6 + a] = lo;
        tb[t * 6 + 3 + a] = hi;
        if (lo < bmin[a]) bmin[a] = lo;
        if (hi > bmax[a]) bmax[a] = hi;
      }
    }
    const int max_nodes = std::max(1, tri_count * 2);
    node_bounds.assign((size_t)max_nodes * 6, 0.0);
    node_left_or_first.assign(max_nodes, 0);
    node_tri_count.assign(max_nodes, 0);
    if (tri_count > 0) {
      node_ptr = 1;
      build_node(0, 0, tri_count, cen, tb);
    }
  }

  // bvh.ts:265-367 intersectSegment
  double intersect_segment(double ox, double oy, double oz, double dx, double dy, double dz,
                           double maxT) const {
    if (tri_count == 0) return -1;
    const double idx_ = std::fabs(dx) > 1e-15 ? 1.0 / dx : (dx >= 0 ? 1e15 : -1e15);
    const double idy = std::fabs(dy) > 1e-15 ? 1.0 / dy : (dy >= 0 ? 1e15 : -1e15);
    const double idz = std::fabs(dz) > 1e-15 ? 1.0 / dz : (dz >= 0 ? 1e15 : -1e15);
    double closest = maxT + 1e-7;
    bool found = false;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int n = stack[--sp];
      const double* b = &node_bounds[(size_t)n * 6];
      const double tx1 = (b[0] - ox) * idx_, tx2 = (b[3] - ox) * idx_;
      double tmin = js_min(tx1, tx2), tmax = js_max(tx1, tx2);
      const double ty1 = (b[1] - oy) * idy, ty2 = (b[4] - oy) * idy;
      tmin = js_max(tmin, js_min(ty1, ty2));
      tmax = js_min(tmax, js_max(ty1, ty2));
      const double tz1 = (b[2] - oz) * idz, tz2 = (b[5] - oz) * idz;
      tmin = js_max(tmin, js_min(tz1, tz2));
      tmax = js_min(tmax, js_max(tz1, tz2));
      if (tmax < js_max(0, tmin) || tmin > closest) continue;
      const int cnt = node_tri_count[n];
      if (cnt > 0) {
        const int first = node_left_or_first[n];
        for (int i = first; i < first + cnt; ++i) {
          const double* T = &tri[(size_t)tri_indices[i] * 9];
          const double ax = T[0], ay = T[1], az = T[2];
          const double e1x = T[3], e1y = T[4], e1z = T[5];
          const double e2x = T[6], e2y = T[7], e2z = T[8];
          const double px = dy * e2z - dz * e2y;
          const double py = dz * e2x - dx * e2z;
          const double pz = dx * e2y - dy * e2x;
          const double det = e1x * px + e1y * py + e1z * pz;
          if (std::fabs(det) < 1e-13) continue;
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
        const int l = node_left_or_first[n];
        stack[sp++] = l + 1;
        stack[sp++] = l;
      }
    }
    return found ? js_min(maxT, closest) : -1;
  }

  // bvh.ts:375-457 collectXScanlineHits
  void scanline(double y, double z, std::vector<double>& hits) const {
    hits.clear();
    if (tri_count == 0) return;
    const double py = y + 1.37e-8, pz = z + 2.93e-8;
    if (py < bmin[1] || py > bmax[1] || pz < bmin[2] || pz > bmax[2]) return;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int n = stack[--sp];
      const double* b = &node_bounds[(size_t)n * 6];
      if (py < b[1] || py > b[4] || pz < b[2] || pz > b[5]) continue;
      const int cnt = node_tri_count[n];
      if (cnt > 0) {
        const int first = node_left_or_first[n];
        for (int i = first; i < first + cnt; ++i) {
          const double* T = &tri[(size_t)tri_indices[i] * 9];
          const double ax = T[0], ay = T[1], az = T[2];
          const double e1x = T[3], e1y = T[4], e1z = T[5];
          const double e2x = T[6], e2y = T[7], e2z = T[8];
          const double det = -e1y * e2z + e1z * e2y;
          if (std::fabs(det) < 1e-13) continue;
          const double inv = 1.0 / det;
          const double ty = py - ay, tz = pz - az;
          const double u = (-ty * e2z + tz * e2y) * inv;
          if (u < 0.0 || u > 1.0) continue;
          const double v = (ty * e1z - tz * e1y) * inv;
          if (v < 0.0 || u + v > 1.0) continue;
          hits.push_back(ax + u * e1x + v * e2x);
        }
      } else {
        const int l = node_left_or_first[n];
        stack[sp++] = l + 1;
        stack[sp++] = l;
      }
    }
    if (hits.size() > 1) std::sort(hits.begin(), hits.end());
  }

  // bvh.ts:499-589 countRayIntersections
  int count_ray(double ox, double oy, double oz, double dx, double dy, double dz) const {
    const double idx_ = 1.0 / dx, idy = 1.0 / dy, idz = 1.0 / dz;
    int hit_count = 0;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int n = stack[--sp];
      const double* b = &node_bounds[(size_t)n * 6];
      const double tx1 = (b[0] - ox) * idx_, tx2 = (b[3] - ox) * idx_;
      double tmin = js_min(tx1, tx2), tmax = js_max(tx1, tx2);
      const double ty1 = (b[1] - oy) * idy, ty2 = (b[4] - oy) * idy;
      tmin = js_max(tmin, js_min(ty1, ty2));
      tmax = js_min(tmax, js_max(ty1, ty2));
      const double tz1 = (b[2] - oz) * idz, tz2 = (b[5] - oz) * idz;
      tmin = js_max(tmin, js_min(tz1, tz2));
      tmax = js_min(tmax, js_max(tz1, tz2));
      if (tmax < js_max(0, tmin)) continue;
      const int cnt = node_tri_count[n];
      if (cnt > 0) {
        const int first = node_left_or_first[n];
        for (int i = first; i < first + cnt; ++i) {
          const double* T = &tri[(size_t)tri_indices[i] * 9];
          const double ax = T[0], ay = T[1], az = T[2];
          const double e1x = T[3], e1y = T[4], e1z = T[5];
          const double e2x = T[6], e2y = T[7], e2z = T[8];
          const double px = dy * e2z - dz * e2y;
          const double py = dz * e2x - dx * e2z;
          const double pz = dx * e2y - dy * e2x;
          const double det = e1x * px + e1y * py + e1z * pz;
          if (std::fabs(det) < 1e-13) continue;
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
          if (t > 1e-7) ++hit_count;
        }
      } else {
        const int l = node_left_or_first[n];
        stack[sp++] = l + 1;
        stack[sp++] = l;
      }
    }
    return hit_count;
  }

  // bvh.ts:464-497 isPointInside
  bool is_point_inside(double x, double y, double z) const {
    if (x < bmin[0] || x > bmax[0] || y < bmin[1] || y > bmax[1] || z < bmin[2] || z > bmax[2])
      return false;
    static const double dirs[3][3] = {{1.0, 0.0137, 0.0293}, {-0.0191, 1.0, 0.0317},
                                      {0.0239, -0.0173, 1.0}};
    int votes = 0;
    for (int d = 0; d < 3; ++d) {
      const int h = count_ray(x, y, z, dirs[d][0], dirs[d][1], dirs[d][2]);
      if ((h & 1) == 1) ++votes;
      if (votes >= 2) return true;
      if (d == 1 && votes == 0) return false;
    }
    return votes >= 2;
  }
};

// ---------------------------------------------------------------------------
// voxelizer.ts -- voxelizeMeshToLattice
// ---------------------------------------------------------------------------
struct Voxel {
  int nx, ny, nz;
  double h, ox, oy, oz;
  std::vector<uint8_t> flags;
  std::vector<int32_t> bmap, bcells;
  std::vector<float> q, minq;
  int64_t solid = 0;
  int window[6];  // minIx, maxIx, minIy, maxIy, minIz, maxIz
  double ms = 0;
};

// voxelizer.ts:65-80
double sub_grid_link_fraction(const BVH& b, double fx, double fy, double fz, double vx,
                              double vy, double vz) {
  const double q = b.intersect_segment(fx, fy, fz, vx, vy, vz, 1.0);
  if (q > 0 && q <= 1.0) return js_max(1e-4, js_min(1.0, q));
  return 0.5;
}

Voxel* voxelize(const BVH& bvh, double tun_h, int nx, int ny, int nz) {
  auto t0 = std::chrono::steady_clock::now();
  Voxel* V = new Voxel();
  V->nx = nx; V->ny = ny; V->nz = nz;
  const int64_t N = (int64_t)nx * ny * nz;
  const double h = tun_h / ny;
  const double dx = h, dy = h, dz = h;
  const double ox = -nx * h * 0.5, oy = -ny * h * 0.5, oz = -nz * h * 0.5;
  V->h = h; V->ox = ox; V->oy = oy; V->oz = oz;
  V->flags.assign(N, CELL_FLUID);
  auto fl = [](double v) { return (int)std::floor(v); };
  auto cl = [](double v) { return (int)std::ceil(v); };
  const int minIx = std::max(0, fl((bvh.bmin[0] - ox) / dx) - 1);
  const int maxIx = std::min(nx - 1, cl((bvh.bmax[0] - ox) / dx) + 1);
  const int minIy = std::max(0, fl((bvh.bmin[1] - oy) / dy) - 1);
  const int maxIy = std::min(ny - 1, cl((bvh.bmax[1] - oy) / dy) + 1);
  const int minIz = std::max(0, fl((bvh.bmin[2] - oz) / dz) - 1);
  const int maxIz = std::min(nz - 1, cl((bvh.bmax[2] - oz) / dz) + 1);
  V->window[0] = minIx; V->window[1] = maxIx; V->window[2] = minIy;
  V->window[3] = maxIy; V->window[4] = minIz; V->window[5] = maxIz;
  std::vector<double> hits;
  uint8_t* F = V->flags.data();
  // voxelizer.ts:127-173 STEP 1
  for (int iz = minIz; iz <= maxIz; ++iz) {
    const double z = oz + (iz + 0.5) * dz;
    for (int iy = minIy; iy <= maxIy; ++iy) {
      const double y = oy + (iy + 0.5) * dy;
      bvh.scanline(y, z, hits);
      const int hc = (int)hits.size();
      if (hc == 0) continue;
      const int64_t row = (int64_t)nx * (iy + (int64_t)ny * iz);
      if ((hc & 1) == 0) {
        for (int k = 0; k < hc; k += 2) {
          const double xe = hits[k], xx = hits[k + 1];
          if (xx - xe < 1e-7) continue;
          const double s = std::ceil((xe - ox) / dx - 0.5);
          const double e = std::floor((xx - ox) / dx - 0.5);
          const double si = js_max(minIx, s), ei = js_min(maxIx, e);
          for (int ix = (int)si; ix <= ei; ++ix) {
            if (F[row + ix] == CELL_FLUID) {
              F[row + ix] = CELL_SOLID;
              ++V->solid;
            }
          }
        }
      } else {
        for (int ix = minIx; ix <= maxIx; ++ix) {
          const double x = ox + (ix + 0.5) * dx;
          if (x >= hits[0] && x <= hits[hc - 1]) {
            if (bvh.is_point_inside(x, y, z)) {
              if (F[row + ix] == CELL_FLUID) {
                F[row + ix] = CELL_SOLID;
                ++V->solid;
              }
            }
          }
        }
      }
    }
  }
  // voxelizer.ts:176-212 STEP 2
  const int sx0 = std::max(0, minIx - 1), sx1 = std::min(nx - 1, maxIx + 1);
  const int sy0 = std::max(0, minIy - 1), sy1 = std::min(ny - 1, maxIy + 1);
  const int sz0 = std::max(0, minIz - 1), sz1 = std::min(nz - 1, maxIz + 1);
  for (int iz = sz0; iz <= sz1; ++iz)
    for (int iy = sy0; iy <= sy1; ++iy) {
      const int64_t row = (int64_t)nx * (iy + (int64_t)ny * iz);
      for (int ix = sx0; ix <= sx1; ++ix) {
        const int64_t i = row + ix;
        if (F[i] != CELL_FLUID) continue;
        bool any = false;
        for (int d = 1; d <= 18 && !any; ++d) {
          const int a = ix + CX[d], b = iy + CY[d], c = iz + CZ[d];
          if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
          if (F[a + (int64_t)nx * (b + (int64_t)ny * c)] == CELL_SOLID) any = true;
        }
        if (any) {
          F[i] = CELL_BOUNDARY;
          V->bcells.push_back((int32_t)i);
        }
      }
    }
  const int64_t B = (int64_t)V->bcells.size();
  V->bmap.assign(N, -1);
  V->q.assign(B * 18, -1.0f);
  V->minq.assign(B, 1.0f);
  // voxelizer.ts:221-256 STEP 3
  for (int64_t bi = 0; bi < B; ++bi) {
    const int64_t ci = V->bcells[bi];
    V->bmap[ci] = (int32_t)bi;
    const int ix = (int)(ci % nx);
    const int64_t rem = (ci - ix) / nx;
    const int iy = (int)(rem % ny);
    const int iz = (int)((rem - iy) / ny);
    const double fx = ox + (ix + 0.5) * dx, fy = oy + (iy + 0.5) * dy, fz = oz + (iz + 0.5) * dz;
    double mq = 1.0;
    for (int d = 1; d <= 18; ++d) {
      const int a = ix + CX[d], b = iy + CY[d], c = iz + CZ[d];
      if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
      if (F[a + (int64_t)nx * (b + (int64_t)ny * c)] == CELL_SOLID) {
        const double q = sub_grid_link_fraction(bvh, fx, fy, fz, CX[d] * dx, CY[d] * dy, CZ[d] * dz);
        V->q[bi * 18 + (d - 1)] = (float)q;
        if (q < mq) mq = q;
      }
    }
    V->minq[bi] = (float)mq;
  }
  V->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return V;
}

// ---------------------------------------------------------------------------
// lbmCpuReference.ts -- LBMCpuReferenceSolver
// ---------------------------------------------------------------------------
struct Solver {
  int nx, ny, nz;
  int64_t N;
  double u_inlet, nu, cs;
  bool ground_no_slip;
  int64_t step_index = 0;
  std::vector<float> fsrc, fdst, ux, uy, uz, rho;
  std::vector<uint8_t> flags;
  std::vector<int32_t> bmap;
  std::vector<float> q;
  int64_t rescale_count = 0;

  // lbmCpuReference.ts:114-143
  void reset() {
    step_index = 0;
    rescale_count = 0;
    for (int64_t i = 0; i < N; ++i) {
      const int iy = (int)((i / nx) % ny);
      double u0 = u_inlet;
      if (ground_no_slip) {
        const double yf = (iy + 0.5) / ny;
        u0 = u_inlet * js_min(1.15, 0.35 + 0.8 * std::pow(yf, 0.3));
        if (iy == 0) u0 = 0;
      }
      if (flags[i] == CELL_SOLID) u0 = 0.0;
      ux[i] = (float)u0; uy[i] = 0.0f; uz[i] = 0.0f; rho[i] = 1.0f;
      for (int d = 0; d < 19; ++d) {
        const float e = (float)feq64(d, 1.0, u0, 0.0, 0.0);
        fsrc[d * N + i] = e;
        fdst[d * N + i] = e;
      }
    }
  }

  // lbmCpuReference.ts:158-313 collide + pull-stream for one cell
  void collide_cell(int ix, int iy, int iz, double tau0, double csSq) {
    const int64_t idx = ix + (int64_t)nx * (iy + (int64_t)ny * iz);
    const uint8_t flag = flags[idx];
    if (flag == CELL_SOLID) {
      ux[idx] = 0; uy[idx] = 0; uz[idx] = 0; rho[idx] = 1.0f;
      return;
    }
    float fl[19], fe[19];
    double r = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
    const int b = flag == CELL_BOUNDARY ? bmap[idx] : -1;
    const int64_t qb = b >= 0 ? (int64_t)b * 18 : -1;
    const float* S = fsrc.data();
    for (int d = 0; d < 19; ++d) {
      const int sx = clampi(ix - CX[d], 0, nx - 1);
      const int sy = clampi(iy - CY[d], 0, ny - 1);
      const int sz = clampi(iz - CZ[d], 0, nz - 1);
      const int64_t src = sx + (int64_t)nx * (sy + (int64_t)ny * sz);
      double val;
      if (d > 0 && flags[src] == CELL_SOLID) {
        const int wd = OPP[d];
        const double qv = qb >= 0 ? (double)q[qb + (wd - 1)] : 0.5;
        const double qe = qv > 0.0 ? qv : 0.5;
        const double fo = S[wd * N + idx];
        const int fx = clampi(ix + CX[d], 0, nx - 1);
        const int fy = clampi(iy + CY[d], 0, ny - 1);
        const int fz = clampi(iz + CZ[d], 0, nz - 1);
        const int64_t ff = fx + (int64_t)nx * (fy + (int64_t)ny * fz);
        if (flags[ff] != CELL_SOLID) {
          if (qe < 0.5) {
            const double fon = S[wd * N + ff];
            val = 2.0 * qe * fo + (1.0 - 2.0 * qe) * fon;
          } else {
            const double fic = S[d * N + idx];
            const double inv2q = 1.0 / (2.0 * qe);
            val = inv2q * fo + (1.0 - inv2q) * fic;
          }
        } else {
          val = fo;
        }
      } else {
        val = S[d * N + src];
      }
      fl[d] = (float)val;
      r += val;
      jx += (double)CX[d] * val;
      jy += (double)CY[d] * val;
      jz += (double)CZ[d] * val;
    }
    r = js_max(0.5, js_min(1.8, r));
    const double ir = 1.0 / r;
    jx *= ir; jy *= ir; jz *= ir;
    const double m2 = jx * jx + jy * jy + jz * jz;
    const double mu = 0.22;
    if (m2 > mu * mu) {
      const double s = mu / std::sqrt(m2);
      jx *= s; jy *= s; jz *= s;
    }
    const double uSq = jx * jx + jy * jy + jz * jz;
    double pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
    for (int d = 0; d < 19; ++d) {
      const double cx = CX[d], cy = CY[d], cz = CZ[d];
      const double cu = 3.0 * (cx * jx + cy * jy + cz * jz);
      const double eq = W32[d] * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * uSq);
      fe[d] = (float)eq;
      const double fn = (double)fl[d] - eq;
      pxx += cx * cx * fn;
      pyy += cy * cy * fn;
      pzz += cz * cz * fn;
      pxy += cx * cy * fn;
      pxz += cx * cz * fn;
      pyz += cy * cz * fn;
    }
    const double pn =
        std::sqrt(pxx * pxx + pyy * pyy + pzz * pzz + 2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
    const double tau = 0.5 * (tau0 + std::sqrt(tau0 * tau0 + (18.0 * M_SQRT2 * csSq * pn) / r));
    const double om = 1.0 / js_max(0.5015, js_min(1.95, tau));
    float* D = fdst.data();
    for (int d = 0; d < 19; ++d) {
      const double cx = CX[d], cy = CY[d], cz = CZ[d];
      const double qxx = cx * cx - 1.0 / 3.0, qyy = cy * cy - 1.0 / 3.0, qzz = cz * cz - 1.0 / 3.0;
      const double qxy = cx * cy, qxz = cx * cz, qyz = cy * cz;
      const double f1 = 4.5 * W32[d] *
                        (qxx * pxx + qyy * pyy + qzz * pzz + 2.0 * (qxy * pxy + qxz * pxz + qyz * pyz));
      D[d * N + idx] = (float)((double)fe[d] + (1.0 - om) * f1);
    }
    ux[idx] = (float)jx; uy[idx] = (float)jy; uz[idx] = (float)jz; rho[idx] = (float)r;
  }

  void collide(int threads) {
    const double tau0 = 3.0 * nu + 0.5;
    const double csSq = cs * cs;
#ifdef _OPENMP
#pragma omp parallel for collapse(2) schedule(static) num_threads(threads) if (threads > 1)
#endif
    for (int iz = 0; iz < nz; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) collide_cell(ix, iy, iz, tau0, csSq);
    (void)threads;
  }

  // lbmCpuReference.ts:315-456
  void boundaries() {
    float* D = fdst.data();
    for (int iz = 0; iz < nz; ++iz)
      for (int iy = 0; iy < ny; ++iy) {
        const int64_t row = (int64_t)nx * (iy + (int64_t)ny * iz);
        const int64_t in = row, nxt = row + 1;
        if (flags[in] != CELL_SOLID) {
          double uxi = u_inlet;
          if (ground_no_slip) {
            const double yf = (iy + 0.5) / ny;
            uxi = u_inlet * js_min(1.15, 0.35 + 0.8 * std::pow(yf, 0.3));
          }
          double uyi = 0.0;
          if (step_index < 120)
            uyi = 0.015 * u_inlet * std::sin(step_index * 0.15 + ((double)iy / ny) * M_PI * 2.0);
          const double ri = 0.85 * rho[nxt] + 0.15 * 1.0;
          for (int d = 0; d < 19; ++d) D[d * N + in] = (float)feq64(d, ri, uxi, uyi, 0.0);
          ux[in] = (float)uxi; uy[in] = (float)uyi; uz[in] = 0.0f; rho[in] = (float)ri;
        }
        const int64_t out = row + (nx - 1), prv = out - 1;
        if (flags[out] != CELL_SOLID) {
          const double ro = rho[prv] * 0.85 + 1.0 * 0.15;
          const double uxo = ux[prv], uyo = uy[prv], uzo = uz[prv];
          for (int d = 0; d < 19; ++d) {
            const double fp = D[d * N + prv];
            const double fe = feq64(d, ro, uxo, uyo, uzo);
            D[d * N + out] = (float)(0.75 * fp + 0.25 * fe);
          }
          ux[out] = (float)uxo; uy[out] = (float)uyo; uz[out] = (float)uzo; rho[out] = (float)ro;
        }
      }
    for (int iz = 0; iz < nz; ++iz)
      for (int ix = 1; ix < nx - 1; ++ix) {
        const int64_t bot = ix + (int64_t)nx * (0 + (int64_t)ny * iz);
        if (flags[bot] != CELL_SOLID && flags[bot] != CELL_BOUNDARY) {
          const double uxw = ground_no_slip ? 0.0 : (double)ux[bot];
          const double uzw = ground_no_slip ? 0.0 : (double)uz[bot];
          const double rw = rho[bot];
          for (int d = 0; d < 19; ++d) D[d * N + bot] = (float)feq64(d, rw, uxw, 0.0, uzw);
          ux[bot] = (float)uxw; uy[bot] = 0.0f; uz[bot] = (float)uzw;
        }
        const int64_t top = ix + (int64_t)nx * (ny - 1 + (int64_t)ny * iz);
        if (flags[top] != CELL_SOLID && flags[top] != CELL_BOUNDARY) {
          const double rw = rho[top];
          for (int d = 0; d < 19; ++d)
            D[d * N + top] = (float)feq64(d, rw, ux[top], 0.0, uz[top]);
          uy[top] = 0.0f;
        }
      }
    if (nz > 4) {
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 1; ix < nx - 1; ++ix) {
          for (int side = 0; side < 2; ++side) {
            const int iz = side == 0 ? 0 : nz - 1;
            const int64_t c = ix + (int64_t)nx * (iy + (int64_t)ny * iz);
            if (flags[c] != CELL_SOLID && flags[c] != CELL_BOUNDARY) {
              const double rw = rho[c];
              for (int d = 0; d < 19; ++d) D[d * N + c] = (float)feq64(d, rw, ux[c], uy[c], 0.0);
              uz[c] = 0.0f;
            }
          }
        }
    }
    // Mass rescale, lbmCpuReference.ts:434-455. The double sum of float densities is
    // exact here (every partial sum is a multiple of 2^-25 below 2^53), so the
    // summation order does not change the result.
    double sum = 0.0;
    int64_t cnt = 0;
    for (int64_t i = 0; i < N; ++i)
      if (flags[i] != CELL_SOLID) {
        sum += rho[i];
        ++cnt;
      }
    if (cnt > 0) {
      const double mean = sum / cnt;
      const double corr = 1.0 / mean;
      if (std::fabs(mean - 1.0) > 1e-4) {
        ++rescale_count;
        for (int64_t i = 0; i < N; ++i)
          if (flags[i] != CELL_SOLID) {
            rho[i] = (float)((double)rho[i] * corr);
            for (int d = 0; d < 19; ++d) D[d * N + i] = (float)((double)D[d * N + i] * corr);
          }
      }
    }
  }

  void step(int n, int threads) {
    for (int s = 0; s < n; ++s) {
      collide(threads);
      boundaries();
      std::swap(fsrc, fdst);
      ++step_index;
    }
  }
};

// forceIntegrator.ts:106-216 (plus Mx, My about the domain centre, which the
// reference's GPU shader forces.wgsl:95-102 also reports)
void momentum_exchange(int nx, int ny, int nz, const uint8_t* flags, const int32_t* bcells,
                       const float* q, int64_t B, const float* f, double* out) {
  const int64_t N = (int64_t)nx * ny * nz;
  double fx = 0, fy = 0, fz = 0, mx = 0, my = 0, mz = 0;
  int64_t cut = 0;
  for (int64_t b = 0; b < B; ++b) {
    const int64_t ci = bcells[b];
    const int ix = (int)(ci % nx);
    const int64_t rem = (ci - ix) / nx;
    const int iy = (int)(rem % ny);
    const int iz = (int)((rem - iy) / ny);
    double cfx = 0, cfy = 0, cfz = 0;
    for (int d = 1; d <= 18; ++d) {
      const double qv = q[b * 18 + (d - 1)];
      if (qv > 0.0) {
        const int od = OPP[d];
        const double fo = f[d * N + ci];
        const int a = clampi(ix + CX[od], 0, nx - 1);
        const int bb = clampi(iy + CY[od], 0, ny - 1);
        const int c = clampi(iz + CZ[od], 0, nz - 1);
        const int64_t ff = a + (int64_t)nx * (bb + (int64_t)ny * c);
        double fi = fo;
        if (flags[ff] != 1) {
          if (qv < 0.5) {
            const double fon = f[d * N + ff];
            fi = 2.0 * qv * fo + (1.0 - 2.0 * qv) * fon;
          } else {
            const double fic = f[od * N + ci];
            const double inv2q = 1.0 / (2.0 * qv);
            fi = inv2q * fo + (1.0 - inv2q) * fic;
          }
        }
        const double mom = fo + fi - 2.0 * W32[d];
        cfx += CX[d] * mom;
        cfy += CY[d] * mom;
        cfz += CZ[d] * mom;
        if (d <= 6) ++cut;
      }
    }
    fx += cfx; fy += cfy; fz += cfz;
    const double rx = (ix + 0.5) - 0.5 * nx;
    const double ry = (iy + 0.5) - 0.5 * ny;
    const double rz = (iz + 0.5) - 0.5 * nz;
    mz += rx * cfy - ry * cfx;
    mx += ry * cfz - rz * cfy;
    my += rz * cfx - rx * cfz;
  }
  out[0] = fx; out[1] = fy; out[2] = fz; out[3] = mx; out[4] = my; out[5] = mz;
  out[6] = (double)cut;
}

}  // namespace

extern "C" {

// ---- BVH ------------------------------------------------------------------
void* orc_bvh_create(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx,
                     const double* world16) {
  return new BVH(pos, nverts, idx, nidx, world16);
}
void orc_bvh_free(void* b) { delete (BVH*)b; }
void orc_bvh_bounds(void* b, double* out6) {
  BVH* v = (BVH*)b;
  for (int a = 0; a < 3; ++a) { out6[a] = v->bmin[a]; out6[3 + a] = v->bmax[a]; }
}
int orc_bvh_nodes(void* b, double* bounds, int32_t* lof, int32_t* cnt, int32_t* tri_idx) {
  BVH* v = (BVH*)b;
  const int n = std::max(1, v->tri_count * 2);
  if (bounds) std::memcpy(bounds, v->node_bounds.data(), sizeof(double) * 6 * n);
  if (lof) std::memcpy(lof, v->node_left_or_first.data(), sizeof(int32_t) * n);
  if (cnt) std::memcpy(cnt, v->node_tri_count.data(), sizeof(int32_t) * n);
  if (tri_idx) std::memcpy(tri_idx, v->tri_indices.data(), sizeof(int32_t) * v->tri_count);
  return v->node_ptr;
}
double orc_bvh_intersect_segment(void* b, double ox, double oy, double oz, double dx, double dy,
                                 double dz, double maxT) {
  return ((BVH*)b)->intersect_segment(ox, oy, oz, dx, dy, dz, maxT);
}
int orc_bvh_is_point_inside(void* b, double x, double y, double z) {
  return ((BVH*)b)->is_point_inside(x, y, z) ? 1 : 0;
}
int orc_bvh_scanline(void* b, double y, double z, double* out, int cap) {
  std::vector<double> h;
  ((BVH*)b)->scanline(y, z, h);
  for (int i = 0; i < (int)h.size() && i < cap; ++i) out[i] = h[i];
  return (int)h.size();
}

// ---- voxelizer ------------------------------------------------------------
void* orc_voxelize(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx,
                   const double* world16, double tunnel_height, int nx, int ny, int nz) {
  BVH bvh(pos, nverts, idx, nidx, world16);
  return voxelize(bvh, tunnel_height, nx, ny, nz);
}
void orc_voxel_free(void* v) { delete (Voxel*)v; }
// counts: [solid, boundary]; geom: [h, ox, oy, oz, ms]; window: 6 ints
void orc_voxel_info(void* v, int64_t* counts, double* geom, int32_t* window) {
  Voxel* V = (Voxel*)v;
  counts[0] = V->solid;
  counts[1] = (int64_t)V->bcells.size();
  geom[0] = V->h; geom[1] = V->ox; geom[2] = V->oy; geom[3] = V->oz; geom[4] = V->ms;
  for (int i = 0; i < 6; ++i) window[i] = V->window[i];
}
void orc_voxel_get(void* v, uint8_t* flags, int32_t* bmap, int32_t* bcells, float* q,
                   float* minq) {
  Voxel* V = (Voxel*)v;
  if (flags) std::memcpy(flags, V->flags.data(), V->flags.size());
  if (bmap) std::memcpy(bmap, V->bmap.data(), V->bmap.size() * 4);
  if (bcells) std::memcpy(bcells, V->bcells.data(), V->bcells.size() * 4);
  if (q) std::memcpy(q, V->q.data(), V->q.size() * 4);
  if (minq) std::memcpy(minq, V->minq.data(), V->minq.size() * 4);
}

// ---- solver ---------------------------------------------------------------
void* orc_solver_create(int nx, int ny, int nz, const uint8_t* flags, const int32_t* bmap,
                        const float* q, int64_t B, double u_inlet, double nu, double cs,
                        int ground_no_slip) {
  Solver* S = new Solver();
  S->nx = nx; S->ny = ny; S->nz = nz;
  S->N = (int64_t)nx * ny * nz;
  S->u_inlet = u_inlet; S->nu = nu; S->cs = cs; S->ground_no_slip = ground_no_slip != 0;
  S->flags.assign(flags, flags + S->N);
  S->bmap.assign(bmap, bmap + S->N);
  S->q.assign(q, q + B * 18);
  S->fsrc.assign(19 * S->N, 0.0f);
  S->fdst.assign(19 * S->N, 0.0f);
  S->ux.assign(S->N, 0.0f); S->uy.assign(S->N, 0.0f);
  S->uz.assign(S->N, 0.0f); S->rho.assign(S->N, 0.0f);
  S->reset();
  return S;
}
void orc_solver_free(void* s) { delete (Solver*)s; }
void orc_solver_set_params(void* s, double u_inlet, double nu, double cs, int gns) {
  Solver* S = (Solver*)s;
  S->u_inlet = u_inlet; S->nu = nu; S->cs = cs; S->ground_no_slip = gns != 0;
}
void orc_solver_reset(void* s) { ((Solver*)s)->reset(); }
void orc_solver_step(void* s, int n, int threads) { ((Solver*)s)->step(n, threads); }
int64_t orc_solver_step_index(void* s) { return ((Solver*)s)->step_index; }
int64_t orc_solver_rescale_count(void* s) { return ((Solver*)s)->rescale_count; }
void orc_solver_get_f(void* s, float* out, int which) {
  Solver* S = (Solver*)s;
  const std::vector<float>& v = which == 0 ? S->fsrc : S->fdst;
  std::memcpy(out, v.data(), v.size() * 4);
}
void orc_solver_set_f(void* s, const float* in) {
  Solver* S = (Solver*)s;
  std::memcpy(S->fsrc.data(), in, S->fsrc.size() * 4);
}
void orc_solver_get_macro(void* s, float* ux, float* uy, float* uz, float* rho) {
  Solver* S = (Solver*)s;
  std::memcpy(ux, S->ux.data(), S->N * 4);
  std::memcpy(uy, S->uy.data(), S->N * 4);
  std::memcpy(uz, S->uz.data(), S->N * 4);
  std::memcpy(rho, S->rho.data(), S->N * 4);
}
// lbmCpuReference.ts:461-495. out: total, mean, max_speed, has_nan
void orc_solver_mass_stats(void* s, double* out) {
  Solver* S = (Solver*)s;
  double total = 0, maxs = 0;
  int64_t cnt = 0;
  int nan = 0;
  for (int64_t i = 0; i < S->N; ++i) {
    if (S->flags[i] == CELL_SOLID) continue;
    const double r = S->rho[i], u = S->ux[i], v = S->uy[i], w = S->uz[i];
    if (std::isnan(r) || std::isnan(u) || std::isnan(v) || std::isnan(w)) {
      nan = 1;
      break;
    }
    total += r;
    ++cnt;
    const double sp = std::sqrt(u * u + v * v + w * w);
    if (sp > maxs) maxs = sp;
  }
  out[0] = total;
  out[1] = cnt > 0 ? total / cnt : 1.0;
  out[2] = maxs;
  out[3] = nan;
}

// ---- forces ---------------------------------------------------------------
// out: fx, fy, fz, mx, my, mz, cut_face_links
void orc_momentum_exchange(int nx, int ny, int nz, const uint8_t* flags, const int32_t* bcells,
                           const float* q, int64_t B, const float* f, double* out) {
  momentum_exchange(nx, ny, nz, flags, bcells, q, B, f, out);
}
// forceIntegrator.ts:240-315. out: cd_raw, cd, cl, cm, xcp
void orc_force_coefficients(double fx, double fy, double mz, double dx, double u_inlet,
                            double frontal_area, double char_len, double tunnel_w,
                            double tunnel_h, double* out) {
  const double cell_area = dx * dx;
  const double q_lat = js_max(1e-9, 0.5 * 1.0 * u_inlet * u_inlet);
  const double a_ref = js_max(1e-4, frontal_area / cell_area);
  const double l_ref = js_max(1.0, char_len / dx);
  const double cd_raw = fx / (q_lat * a_ref);
  const double cl = fy / (q_lat * a_ref);
  const double cm = mz / (q_lat * a_ref * l_ref);
  const double t_area = js_max(1e-4, tunnel_w * tunnel_h);
  const double br = js_min(0.40, frontal_area / t_area);
  const double mf = 1.0 + 2.5 * js_max(0.0, cd_raw) * br;
  out[0] = cd_raw;
  out[1] = cd_raw / mf;
  out[2] = cl;
  out[3] = cm;
  out[4] = std::fabs(fy) > 1e-5
               ? js_max(-char_len * 0.5, js_min(char_len * 0.5, -(mz / fy) * dx))
               : 0.0;
}

// frontalArea.ts:22-179 computeProjectedFrontalArea
double orc_frontal_area(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx,
                        const double* m, int res) {
  if (nverts < 3) return 0;
  const int64_t T = idx ? nidx / 3 : nverts / 3;
  if (T == 0) return 0;
  std::vector<double> py(nverts), pz(nverts);
  double mny = INFINITY, mxy = -INFINITY, mnz = INFINITY, mxz = -INFINITY;
  for (int64_t i = 0; i < nverts; ++i) {
    double x = pos[i * 3], y = pos[i * 3 + 1], z = pos[i * 3 + 2];
    if (m) {
      const double w = 1.0 / (m[3] * x + m[7] * y + m[11] * z + m[15]);
      const double yy = (m[1] * x + m[5] * y + m[9] * z + m[13]) * w;
      const double zz = (m[2] * x + m[6] * y + m[10] * z + m[14]) * w;
      y = yy; z = zz;
    }
    py[i] = y; pz[i] = z;
    if (y < mny) mny = y;
    if (y > mxy) mxy = y;
    if (z < mnz) mnz = z;
    if (z > mxz) mxz = z;
  }
  const double sy = mxy - mny, sz = mxz - mnz;
  if (sy <= 1e-9 || sz <= 1e-9) return 0;
  const int ny = res, nz = res;
  std::vector<uint16_t> mask((size_t)ny * nz, 0);
  const double icy = ny / sy, icz = nz / sz;
  const double off[4] = {0.125, 0.375, 0.625, 0.875};
  for (int64_t t = 0; t < T; ++t) {
    int64_t i0, i1, i2;
    if (idx) { i0 = idx[t * 3]; i1 = idx[t * 3 + 1]; i2 = idx[t * 3 + 2]; }
    else { i0 = t * 3; i1 = t * 3 + 1; i2 = t * 3 + 2; }
    const double z0 = (pz[i0] - mnz) * icz, y0 = (py[i0] - mny) * icy;
    const double z1 = (pz[i1] - mnz) * icz, y1 = (py[i1] - mny) * icy;
    const double z2 = (pz[i2] - mnz) * icz, y2 = (py[i2] - mny) * icy;
    const double a2 = (z1 - z0) * (y2 - y0) - (y1 - y0) * (z2 - z0);
    if (std::fabs(a2) < 1e-11) continue;
    double az = z0, ay = y0, bz = z1, by = y1, cz = z2, cy = y2;
    if (a2 < 0) { bz = z2; by = y2; cz = z1; cy = y1; }
    const int tz0 = (int)js_max(0, std::floor(js_min(js_min(az, bz), cz)));
    const int tz1 = (int)js_min(nz - 1, std::floor(js_max(js_max(az, bz), cz)));
    const int ty0 = (int)js_max(0, std::floor(js_min(js_min(ay, by), cy)));
    const int ty1 = (int)js_min(ny - 1, std::floor(js_max(js_max(ay, by), cy)));
    const double dz01 = bz - az, dy01 = by - ay, dz12 = cz - bz, dy12 = cy - by;
    const double dz20 = az - cz, dy20 = ay - cy;
    for (int iy = ty0; iy <= ty1; ++iy)
      for (int iz = tz0; iz <= tz1; ++iz) {
        uint16_t mk = mask[(size_t)iy * nz + iz];
        if (mk == 0xffff) continue;
        int bit = 1;
        for (int a = 0; a < 4; ++a) {
          const double yy = iy + off[a];
          for (int c = 0; c < 4; ++c) {
            if ((mk & bit) == 0) {
              const double zz = iz + off[c];
              const double e0 = dz01 * (yy - ay) - dy01 * (zz - az);
              if (e0 >= -1e-9) {
                const double e1 = dz12 * (yy - by) - dy12 * (zz - bz);
                if (e1 >= -1e-9) {
                  const double e2 = dz20 * (yy - cy) - dy20 * (zz - cz);
                  if (e2 >= -1e-9) mk |= bit;
                }
              }
            }
            bit <<= 1;
          }
        }
        mask[(size_t)iy * nz + iz] = mk;
      }
  }
  int64_t cov = 0;
  for (uint16_t v : mask) cov += __builtin_popcount(v);
  return ((double)cov / ((double)ny * nz * 16)) * (sy * sz);
}

// forceIntegrator.ts:57-99 computeTrueMeshSurfaceArea
double orc_surface_area(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx,
                        const double* m) {
  const int64_t T = idx ? nidx / 3 : nverts / 3;
  double total = 0;
  for (int64_t t = 0; t < T; ++t) {
    double v[3][3];
    for (int k = 0; k < 3; ++k) {
      const int64_t vi = idx ? idx[t * 3 + k] : t * 3 + k;
      double x = pos[vi * 3], y = pos[vi * 3 + 1], z = pos[vi * 3 + 2];
      if (m) {
        const double w = 1.0 / (m[3] * x + m[7] * y + m[11] * z + m[15]);
        const double a = (m[0] * x + m[4] * y + m[8] * z + m[12]) * w;
        const double b = (m[1] * x + m[5] * y + m[9] * z + m[13]) * w;
        const double c = (m[2] * x + m[6] * y + m[10] * z + m[14]) * w;
        x = a; y = b; z = c;
      }
      v[k][0] = x; v[k][1] = y; v[k][2] = z;
    }
    const double e1[3] = {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]};
    const double e2[3] = {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]};
    const double cx = e1[1] * e2[2] - e1[2] * e2[1];
    const double cy = e1[2] * e2[0] - e1[0] * e2[2];
    const double cz = e1[0] * e2[1] - e1[1] * e2[0];
    total += 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
  }
  return total;
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ---- slice image: sampleCFDColormap + extractSliceRGBA, lbmCpuReference.ts:23-46, 499-596
static void cfd_colormap(double tv, double rgb[3]) {
  const double t = js_max(0.0, js_min(1.0, tv));
  if (t < 0.25) {
    const double u = t * 4.0;
    rgb[0] = 0.08 + (0.06 - 0.08) * u; rgb[1] = 0.22 + (0.72 - 0.22) * u; rgb[2] = 0.75 + (0.88 - 0.75) * u;
  } else if (t < 0.5) {
    const double u = (t - 0.25) * 4.0;
    rgb[0] = 0.06 + (0.12 - 0.06) * u; rgb[1] = 0.72 + (0.82 - 0.72) * u; rgb[2] = 0.88 + (0.38 - 0.88) * u;
  } else if (t < 0.75) {
    const double u = (t - 0.5) * 4.0;
    rgb[0] = 0.12 + (0.98 - 0.12) * u; rgb[1] = 0.82 + (0.62 - 0.82) * u; rgb[2] = 0.38 + (0.08 - 0.38) * u;
  } else {
    const double u = (t - 0.75) * 4.0;
    rgb[0] = 0.98 + (0.94 - 0.98) * u; rgb[1] = 0.62 + (0.16 - 0.62) * u; rgb[2] = 0.08 + (0.18 - 0.08) * u;
  }
}
// Math.round: the nearest integer, halves toward +infinity
static double js_round(double x) { return std::floor(x + 0.5); }

void orc_colormap(double t, double* rgb) { cfd_colormap(t, rgb); }

// axis 0 = x, 1 = y, 2 = z; mode 0 = velocity, 1 = vorticity, 2 = pressure.
// rgba: width * height * 4 bytes (width, height as the reference forms them).
void orc_extract_slice(void* s, int axis, double frac, int mode, uint8_t* rgba, int* w_out, int* h_out) {
  const Solver* S = (const Solver*)s;
  const int nx = S->nx, ny = S->ny, nz = S->nz;
  int width = nx, height = ny;
  if (axis == 1) { width = nx; height = nz; }
  else if (axis == 0) { width = nz; height = ny; }
  *w_out = width;
  *h_out = height;
  if (!rgba) return;
  const double uref = js_max(1e-4, S->u_inlet);
  const int fz = (int)js_min(nz - 1, js_max(0, std::floor(frac * nz)));
  const int fy = (int)js_min(ny - 1, js_max(0, std::floor(frac * ny)));
  const int fx = (int)js_min(nx - 1, js_max(0, std::floor(frac * nx)));
  const float *ux = S->ux.data(), *uy = S->uy.data(), *uz = S->uz.data(), *rho = S->rho.data();
  for (int v = 0; v < height; ++v)
    for (int u = 0; u < width; ++u) {
      int ix = u, iy = v, iz = fz;
      if (axis == 1) { ix = u; iy = fy; iz = v; }
      else if (axis == 0) { ix = fx; iy = v; iz = u; }
      const int64_t idx = ix + (int64_t)nx * (iy + (int64_t)ny * iz);
      uint8_t* px = rgba + ((int64_t)v * width + u) * 4;
      if (S->flags[idx] == CELL_SOLID) { px[0] = px[1] = px[2] = px[3] = 0; continue; }
      double sn = 0.5, alpha = 215;
      if (mode == 0) {
        const double sp = std::sqrt((double)ux[idx] * ux[idx] + (double)uy[idx] * uy[idx] + (double)uz[idx] * uz[idx]);
        sn = js_min(1.0, js_max(0.0, sp / (uref * 1.55)));
      } else if (mode == 1) {
        const int ixP = (int)js_min(nx - 1, ix + 1), ixM = (int)js_max(0, ix - 1);
        const int iyP = (int)js_min(ny - 1, iy + 1), iyM = (int)js_max(0, iy - 1);
        const int izP = (int)js_min(nz - 1, iz + 1), izM = (int)js_max(0, iz - 1);
        auto at = [&](int x, int y, int z) { return x + (int64_t)nx * (y + (int64_t)ny * z); };
        const double wx = 0.5 * ((double)uz[at(ix, iyP, iz)] - uz[at(ix, iyM, iz)]) -
                          0.5 * ((double)uy[at(ix, iy, izP)] - uy[at(ix, iy, izM)]);
        const double wy = 0.5 * ((double)ux[at(ix, iy, izP)] - ux[at(ix, iy, izM)]) -
                          0.5 * ((double)uz[at(ixP, iy, iz)] - uz[at(ixM, iy, iz)]);
        const double wz = 0.5 * ((double)uy[at(ixP, iy, iz)] - uy[at(ixM, iy, iz)]) -
                          0.5 * ((double)ux[at(ix, iyP, iz)] - ux[at(ix, iyM, iz)]);
        const double vm = std::sqrt(wx * wx + wy * wy + wz * wz);
        const double vn = js_min(1.0, vm / (uref * 0.42));
        sn = 0.35 + 0.65 * vn;
        alpha = js_round(70 + 175 * vn);
      } else {
        const double cp = (((double)rho[idx] - 1.0) / 3.0) / (0.5 * uref * uref);
        sn = js_min(1.0, js_max(0.0, (cp + 1.1) / 2.1));
      }
      double rgb[3];
      cfd_colormap(sn, rgb);
      px[0] = (uint8_t)(int)js_round(rgb[0] * 255);
      px[1] = (uint8_t)(int)js_round(rgb[1] * 255);
      px[2] = (uint8_t)(int)js_round(rgb[2] * 255);
      px[3] = (uint8_t)(int)alpha;
    }
}

// ---- Q-criterion and vorticity, src/render/vortexIso.ts:22-122 (computeQCriterion).
// flags may be null; outputs: q[N], om[N], omv[3N] (float, 0 at solid cells), maxima.
void orc_q_criterion(int nx, int ny, int nz, double dx, const float* ux, const float* uy, const float* uz,
                     const uint8_t* flags, float* q, float* om, float* omv, double* max_q, double* max_om) {
  double mq = 1e-6, mo = 1e-6;
  const double inv2dx = 1.0 / (2.0 * dx);
  auto at = [&](int x, int y, int z) { return x + (int64_t)nx * (y + (int64_t)ny * z); };
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const int64_t i = at(ix, iy, iz);
        if (flags && flags[i] == 1) continue;
        const int xp = (int)js_max(0, ix - 1), xn = (int)js_min(nx - 1, ix + 1);
        const int yp = (int)js_max(0, iy - 1), yn = (int)js_min(ny - 1, iy + 1);
        const int zp = (int)js_max(0, iz - 1), zn = (int)js_min(nz - 1, iz + 1);
        const double sx = xn > xp ? 1.0 / ((xn - xp) * dx) : inv2dx;
        const double sy = yn > yp ? 1.0 / ((yn - yp) * dx) : inv2dx;
        const double sz = zn > zp ? 1.0 / ((zn - zp) * dx) : inv2dx;
        const double a = ((double)ux[at(xn, iy, iz)] - ux[at(xp, iy, iz)]) * sx;
        const double b = ((double)ux[at(ix, yn, iz)] - ux[at(ix, yp, iz)]) * sy;
        const double c = ((double)ux[at(ix, iy, zn)] - ux[at(ix, iy, zp)]) * sz;
        const double d = ((double)uy[at(xn, iy, iz)] - uy[at(xp, iy, iz)]) * sx;
        const double e = ((double)uy[at(ix, yn, iz)] - uy[at(ix, yp, iz)]) * sy;
        const double f = ((double)uy[at(ix, iy, zn)] - uy[at(ix, iy, zp)]) * sz;
        const double g = ((double)uz[at(xn, iy, iz)] - uz[at(xp, iy, iz)]) * sx;
        const double h = ((double)uz[at(ix, yn, iz)] - uz[at(ix, yp, iz)]) * sy;
        const double k = ((double)uz[at(ix, iy, zn)] - uz[at(ix, iy, zp)]) * sz;
        const double S12 = 0.5 * (b + d), S13 = 0.5 * (c + g), S23 = 0.5 * (f + h);
        const double nS = a * a + e * e + k * k + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
        const double O12 = 0.5 * (b - d), O13 = 0.5 * (c - g), O23 = 0.5 * (f - h);
        const double nO = 2.0 * (O12 * O12 + O13 * O13 + O23 * O23);
        const double qv = 0.5 * (nO - nS);
        q[i] = (float)qv;
        if (qv > mq) mq = qv;
        const double ox = h - f, oy = c - g, oz = d - b;
        const double m = std::sqrt(ox * ox + oy * oy + oz * oz);
        omv[3 * i] = (float)ox; omv[3 * i + 1] = (float)oy; omv[3 * i + 2] = (float)oz;
        om[i] = (float)m;
        if (m > mo) mo = m;
      }
  *max_q = mq;
  *max_om = mo;
}

}  // extern "C"
