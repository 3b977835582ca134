// Geometry inputs of the force coefficients: the STL reader, the millimetre
// auto-scale, the mesh statistics (src/geometry/stlLoader.ts) and the projected
// frontal area A_ref as a CUDA raster (src/geometry/frontalArea.ts:22-179).
//
// The reference runs these once per geometry on the browser's main thread with
// three.js 0.170.0 (package-lock.json), which is not part of the reference tree;
// the pieces of it that decide the numbers are restated here from its published
// source: BufferAttribute.applyMatrix4 / Vector3.applyMatrix4 (the w-divided affine
// map), Box3.setFromBufferAttribute / getCenter / getSize, BufferGeometry.translate /
// scale (which recompute an existing bounding box in place), MathUtils.degToRad,
// Quaternion.setFromEuler ('XYZ') and Matrix4.compose.
//
// Compiled with -fmad=false: the raster's edge functions and the projected
// coordinates round exactly like the host raster (aerosim_frontal_area), so both
// return the same area bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "aerosim.h"
#include "common.cuh"
#include "engine_internal.h"

namespace aerosim {
namespace {

// ---- three.js arithmetic --------------------------------------------------

// Vector3.applyMatrix4: (e0 x + e4 y + e8 z + e12) / (e3 x + e7 y + e11 z + e15), ...
__host__ __device__ inline void apply_matrix4(const double* e, double& x, double& y, double& z) {
  const double w = 1.0 / (e[3] * x + e[7] * y + e[11] * z + e[15]);
  const double tx = (e[0] * x + e[4] * y + e[8] * z + e[12]) * w;
  const double ty = (e[1] * x + e[5] * y + e[9] * z + e[13]) * w;
  const double tz = (e[2] * x + e[6] * y + e[10] * z + e[14]) * w;
  x = tx; y = ty; z = tz;
}

// BufferAttribute.applyMatrix4 on float32 positions: each result is stored as float32.
void apply_matrix4_f32(const double* e, float* pos, int64_t nv) {
  for (int64_t i = 0; i < nv; ++i) {
    double x = pos[i * 3], y = pos[i * 3 + 1], z = pos[i * 3 + 2];
    apply_matrix4(e, x, y, z);
    pos[i * 3] = (float)x; pos[i * 3 + 1] = (float)y; pos[i * 3 + 2] = (float)z;
  }
}

// Box3.setFromBufferAttribute: Math.min / Math.max over the float32 positions.
void bounding_box(const float* pos, int64_t nv, double mn[3], double mx[3]) {
  for (int k = 0; k < 3; ++k) { mn[k] = INFINITY; mx[k] = -INFINITY; }
  for (int64_t i = 0; i < nv; ++i)
    for (int k = 0; k < 3; ++k) {
      mn[k] = js_min(mn[k], (double)pos[i * 3 + k]);
      mx[k] = js_max(mx[k], (double)pos[i * 3 + k]);
    }
}

// Matrix4.compose(position, Quaternion.setFromEuler(Euler(rx, ry, rz, 'XYZ')), scale)
// with the angles from MathUtils.degToRad (degrees * (Math.PI / 180)).
void compose_model_matrix(const aerosim_model_transform& t, double* te) {
  const double deg2rad = M_PI / 180.0;
  const double rx = t.rotation_deg[0] * deg2rad, ry = t.rotation_deg[1] * deg2rad,
               rz = t.rotation_deg[2] * deg2rad;
  const double c1 = std::cos(rx / 2), c2 = std::cos(ry / 2), c3 = std::cos(rz / 2);
  const double s1 = std::sin(rx / 2), s2 = std::sin(ry / 2), s3 = std::sin(rz / 2);
  const double qx = s1 * c2 * c3 + c1 * s2 * s3;
  const double qy = c1 * s2 * c3 - s1 * c2 * s3;
  const double qz = c1 * c2 * s3 + s1 * s2 * c3;
  const double qw = c1 * c2 * c3 - s1 * s2 * s3;
  const double x2 = qx + qx, y2 = qy + qy, z2 = qz + qz;
  const double xx = qx * x2, xy = qx * y2, xz = qx * z2;
  const double yy = qy * y2, yz = qy * z2, zz = qz * z2;
  const double wx = qw * x2, wy = qw * y2, wz = qw * z2;
  const double sx = t.scale[0], sy = t.scale[1], sz = t.scale[2];
  te[0] = (1 - (yy + zz)) * sx; te[1] = (xy + wz) * sx;       te[2] = (xz - wy) * sx;        te[3] = 0;
  te[4] = (xy - wz) * sy;       te[5] = (1 - (xx + zz)) * sy; te[6] = (yz + wx) * sy;        te[7] = 0;
  te[8] = (xz + wy) * sz;       te[9] = (yz - wx) * sz;       te[10] = (1 - (xx + yy)) * sz; te[11] = 0;
  te[12] = t.position[0];       te[13] = t.position[1];       te[14] = t.position[2];        te[15] = 1;
}

// Math.round: nearest integer, halves toward +infinity; -0 folded into +0 because the
// reference compares the rounded values through their decimal strings (`${-0}` is "0").
inline double js_round(double v) {
  double r = std::floor(v);
  if (v - r >= 0.5) r += 1.0;
  return r + 0.0;
}

// ---- STL parsing ----------------------------------------------------------

// Byte length of a JavaScript `\s` character (WhiteSpace or LineTerminator) encoded
// in UTF-8 at p, or 0.
inline int js_space_len(const uint8_t* p, const uint8_t* end) {
  const uint8_t c = p[0];
  if (c == ' ' || (c >= 0x09 && c <= 0x0d)) return 1;
  const int64_t n = end - p;
  if (c == 0xc2 && n >= 2 && p[1] == 0xa0) return 2;                              // U+00A0
  if (c == 0xe1 && n >= 3 && p[1] == 0x9a && p[2] == 0x80) return 3;               // U+1680
  if (c == 0xe2 && n >= 3 && p[1] == 0x80 &&
      (p[2] <= 0x8a || p[2] == 0xa8 || p[2] == 0xa9 || p[2] == 0xaf) && p[2] >= 0x80) return 3;  // U+2000-200A, 2028, 2029, 202F
  if (c == 0xe2 && n >= 3 && p[1] == 0x81 && p[2] == 0x9f) return 3;               // U+205F
  if (c == 0xe3 && n >= 3 && p[1] == 0x80 && p[2] == 0x80) return 3;               // U+3000
  if (c == 0xef && n >= 3 && p[1] == 0xbb && p[2] == 0xbf) return 3;               // U+FEFF
  return 0;
}

inline bool is_digit(uint8_t c) { return c >= '0' && c <= '9'; }

// Longest match at p of the number pattern [+-]?\d*\.?\d+(?:[eE][+-]?\d+)?, the token
// the reference's vertex regex captures (stlLoader.ts:79).  Returns its end, or null.
// Every shorter match ends on a character of the longest one, so a number followed by
// \s+ matches exactly when the longest match is followed by whitespace.
const uint8_t* match_number(const uint8_t* p, const uint8_t* end) {
  const uint8_t* q = p;
  if (q < end && (*q == '+' || *q == '-')) ++q;
  const uint8_t* d0 = q;
  while (q < end && is_digit(*q)) ++q;
  const uint8_t* int_end = q;
  const uint8_t* m = nullptr;
  if (q < end && *q == '.' && q + 1 < end && is_digit(q[1])) {  // \d*\.\d+
    q += 1;
    while (q < end && is_digit(*q)) ++q;
    m = q;
  } else if (int_end > d0) {  // \d+ (a '.' not followed by a digit is not part of it)
    m = int_end;
  }
  if (!m) return nullptr;
  if (m < end && (*m == 'e' || *m == 'E')) {  // optional exponent, all or nothing
    const uint8_t* e = m + 1;
    if (e < end && (*e == '+' || *e == '-')) ++e;
    const uint8_t* ed = e;
    while (e < end && is_digit(*e)) ++e;
    if (e > ed) m = e;
  }
  return m;
}

double parse_number(const uint8_t* a, const uint8_t* b) {
  std::string s(reinterpret_cast<const char*>(a), (size_t)(b - a));
  return std::strtod(s.c_str(), nullptr);  // correctly rounded, like parseFloat
}

// parseAsciiSTL, stlLoader.ts:77-95: every match of
// /vertex\s+(NUM)\s+(NUM)\s+(NUM)/g, parseFloat'ed and stored as float32.
int parse_ascii(const uint8_t* text, int64_t n, std::vector<float>* out) {
  static const char kVertex[] = "vertex";
  const uint8_t* end = text + n;
  const uint8_t* p = text;
  out->clear();
  while (end - p >= 6) {
    if (std::memcmp(p, kVertex, 6) != 0) { ++p; continue; }
    const uint8_t* q = p + 6;
    double v[3];
    bool ok = true;
    for (int k = 0; k < 3 && ok; ++k) {
      int sp = 0, nsp = 0;
      while (q < end && (sp = js_space_len(q, end)) > 0) { q += sp; ++nsp; }
      if (nsp == 0) { ok = false; break; }
      const uint8_t* e = match_number(q, end);
      if (!e) { ok = false; break; }
      if (k < 2 && (e >= end || js_space_len(e, end) == 0)) { ok = false; break; }
      v[k] = parse_number(q, e);
      q = e;
    }
    if (!ok) { ++p; continue; }
    for (int k = 0; k < 3; ++k) out->push_back((float)v[k]);
    p = q;  // the global regex resumes after the match
  }
  if (out->size() < 9 || out->size() % 9 != 0) {
    set_global_error("ASCII STL file contains no valid triangles.");
    return AEROSIM_ERR_FORMAT;
  }
  return AEROSIM_OK;
}

// TextDecoder drops a leading UTF-8 byte-order mark; String.trimStart drops leading
// WhiteSpace / LineTerminator characters.  True when what is left of the first 256
// bytes starts with "solid" in any letter case.
bool header_says_solid(const uint8_t* b, int64_t n) {
  const uint8_t* end = b + std::min<int64_t>(256, n);
  const uint8_t* p = b;
  if (end - p >= 3 && p[0] == 0xef && p[1] == 0xbb && p[2] == 0xbf) p += 3;
  int sp;
  while (p < end && (sp = js_space_len(p, end)) > 0) p += sp;
  static const char kSolid[] = "solid";
  if (end - p < 5) return false;
  for (int i = 0; i < 5; ++i)
    if ((p[i] | 0x20) != (uint8_t)kSolid[i]) return false;
  return true;
}

bool contains(const uint8_t* b, int64_t n, const char* word) {
  const size_t w = std::strlen(word);
  if ((size_t)n < w) return false;
  return std::search(b, b + n, word, word + w) != b + n;
}

uint32_t read_u32le(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// parseBinarySTL, stlLoader.ts:40-75: 50-byte facets after the 84-byte header, the
// three vertices of each at bytes 12..47 (the facet normal and attribute word skipped).
void parse_binary(const uint8_t* b, uint32_t faces, std::vector<float>* out) {
  out->resize((size_t)faces * 9);
  for (uint32_t i = 0; i < faces; ++i) {
    const uint8_t* f = b + 84 + (size_t)i * 50 + 12;
    for (int k = 0; k < 9; ++k) {
      const uint32_t bits = read_u32le(f + 4 * k);
      float v;
      std::memcpy(&v, &bits, 4);
      (*out)[(size_t)i * 9 + k] = v;
    }
  }
}

// ---- frontal-area raster on the GPU ---------------------------------------

struct Mat16 {
  double e[16];
  int has;
};

struct RasterStatus {
  unsigned long long box[4];  // order keys of min y, max y, min z, max z
  unsigned long long covered; // covered sub-samples
  int bad_index;
};

// Monotone map of a double onto unsigned 64-bit integers (atomicMin / atomicMax).
__host__ __device__ inline unsigned long long order_key(double v) {
  unsigned long long b;
  memcpy(&b, &v, 8);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double from_order_key(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  memcpy(&v, &b, 8);
  return v;
}

constexpr int kRasterThreads = 256;

// Projects every vertex to (y, z) through the world matrix and reduces the Y-Z
// bounding box (frontalArea.ts: the projected coordinates and their extent).
__global__ void __launch_bounds__(kRasterThreads) frontal_project_kernel(
    const float* __restrict__ pos, int64_t nv, const Mat16 m, double* __restrict__ py,
    double* __restrict__ pz, RasterStatus* st) {
  unsigned long long kmin_y = ~0ull, kmax_y = 0, kmin_z = ~0ull, kmax_z = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
    double x = pos[i * 3], y = pos[i * 3 + 1], z = pos[i * 3 + 2];
    if (m.has) apply_matrix4(m.e, x, y, z);
    py[i] = y; pz[i] = z;
    const unsigned long long ky = order_key(y), kz = order_key(z);
    kmin_y = min(kmin_y, ky); kmax_y = max(kmax_y, ky);
    kmin_z = min(kmin_z, kz); kmax_z = max(kmax_z, kz);
  }
  for (int o = 16; o > 0; o >>= 1) {
    kmin_y = min(kmin_y, __shfl_xor_sync(0xffffffffu, kmin_y, o));
    kmax_y = max(kmax_y, __shfl_xor_sync(0xffffffffu, kmax_y, o));
    kmin_z = min(kmin_z, __shfl_xor_sync(0xffffffffu, kmin_z, o));
    kmax_z = max(kmax_z, __shfl_xor_sync(0xffffffffu, kmax_z, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&st->box[0], kmin_y); atomicMax(&st->box[1], kmax_y);
    atomicMin(&st->box[2], kmin_z); atomicMax(&st->box[3], kmax_z);
  }
}

// One warp per triangle: the lanes walk the triangle's pixel box and OR the 4x4
// sub-sample coverage bits of each pixel into `cover` (computeProjectedFrontalArea's
// supersampled raster; coverage is order-independent, so the result equals the
// serial raster's).
__global__ void __launch_bounds__(kRasterThreads) frontal_raster_kernel(
    const double* __restrict__ py, const double* __restrict__ pz, int64_t nv,
    const int32_t* __restrict__ idx, int64_t T, int res, unsigned* __restrict__ cover, RasterStatus* st) {
  const double y0 = from_order_key(st->box[0]), y1 = from_order_key(st->box[1]);
  const double z0 = from_order_key(st->box[2]), z1 = from_order_key(st->box[3]);
  const double span_y = y1 - y0, span_z = z1 - z0;
  if (span_y <= 1e-9 || span_z <= 1e-9) return;
  const double sy = res / span_y, sz = res / span_z;
  const double sub[4] = {0.125, 0.375, 0.625, 0.875};
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; t < T; t += warps) {
    int64_t v[3];
    bool bad = false;
    for (int k = 0; k < 3; ++k) {
      v[k] = idx ? idx[t * 3 + k] : t * 3 + k;
      bad |= v[k] < 0 || v[k] >= nv;
    }
    if (bad) {
      if (lane == 0) atomicExch(&st->bad_index, 1);
      continue;
    }
    double Z[3], Y[3];
    for (int k = 0; k < 3; ++k) {
      Z[k] = (pz[v[k]] - z0) * sz;
      Y[k] = (py[v[k]] - y0) * sy;
    }
    const double area2 = (Z[1] - Z[0]) * (Y[2] - Y[0]) - (Y[1] - Y[0]) * (Z[2] - Z[0]);
    if (fabs(area2) < 1e-11) continue;
    if (area2 < 0) {
      double s = Z[1]; Z[1] = Z[2]; Z[2] = s;
      s = Y[1]; Y[1] = Y[2]; Y[2] = s;
    }
    const int iz0 = (int)js_max(0, floor(js_min(js_min(Z[0], Z[1]), Z[2])));
    const int iz1 = (int)js_min(res - 1, floor(js_max(js_max(Z[0], Z[1]), Z[2])));
    const int iy0 = (int)js_max(0, floor(js_min(js_min(Y[0], Y[1]), Y[2])));
    const int iy1 = (int)js_min(res - 1, floor(js_max(js_max(Y[0], Y[1]), Y[2])));
    if (iz1 < iz0 || iy1 < iy0) continue;
    double ez[3], ey[3];
    for (int k = 0; k < 3; ++k) {
      ez[k] = Z[(k + 1) % 3] - Z[k];
      ey[k] = Y[(k + 1) % 3] - Y[k];
    }
    const int wz = iz1 - iz0 + 1;
    const int64_t pixels = (int64_t)(iy1 - iy0 + 1) * wz;
    for (int64_t p = lane; p < pixels; p += 32) {
      const int iy = iy0 + (int)(p / wz), iz = iz0 + (int)(p % wz);
      unsigned mask = 0;
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
          const double Py = iy + sub[a], Pz = iz + sub[b];
          bool in = true;
          for (int k = 0; k < 3 && in; ++k) in = ez[k] * (Py - Y[k]) - ey[k] * (Pz - Z[k]) >= -1e-9;
          if (in) mask |= 1u << (a * 4 + b);
        }
      if (mask) atomicOr(&cover[(int64_t)iy * res + iz], mask);
    }
  }
}

__global__ void __launch_bounds__(kRasterThreads) frontal_count_kernel(const unsigned* __restrict__ cover,
                                                                       int64_t n, RasterStatus* st) {
  unsigned long long c = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    c += __popc(cover[i]);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&st->covered, c);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    cudaSetDevice(d);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int cuda_fail(const char* what, cudaError_t e) {
  set_global_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? AEROSIM_ERR_NOMEM : AEROSIM_ERR_CUDA;
}

int frontal_area_cuda(int device, const float* pos, int64_t nv, const int32_t* idx, int64_t ni,
                      const double* world16, int res, double* out) {
  *out = 0.0;
  if (nv < 3) return AEROSIM_OK;
  const int64_t T = idx ? ni / 3 : nv / 3;
  if (T == 0) return AEROSIM_OK;
  int n_dev = 0;
  cudaError_t e = cudaGetDeviceCount(&n_dev);
  if (e != cudaSuccess || n_dev == 0) return cuda_fail("aerosim_frontal_area_cuda: no CUDA device", e);
  if (device < 0 || device >= n_dev) {
    set_global_error("aerosim_frontal_area_cuda: bad device ordinal");
    return AEROSIM_ERR_ARG;
  }
  DeviceGuard guard(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaStream_t s = nullptr;
  if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail("cudaStreamCreate", e);
  const int64_t cover_n = (int64_t)res * res;
  const size_t bytes_pos = (size_t)nv * 12, bytes_idx = idx ? (size_t)T * 12 : 0;
  const size_t bytes_pyz = (size_t)nv * 8, bytes_cover = (size_t)cover_n * 4;
  char* base = nullptr;
  auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t total = align(sizeof(RasterStatus)) + align(bytes_pos) + align(bytes_idx) + 2 * align(bytes_pyz) +
                       align(bytes_cover);
  e = cudaMallocAsync((void**)&base, total, s);
  int rc = AEROSIM_OK;
  if (e != cudaSuccess) {
    rc = cuda_fail("aerosim_frontal_area_cuda: device allocation", e);
  } else {
    size_t off = 0;
    auto take = [&](size_t b) { char* p = base + off; off += align(b); return p; };
    RasterStatus* d_st = (RasterStatus*)take(sizeof(RasterStatus));
    float* d_pos = (float*)take(bytes_pos);
    int32_t* d_idx = idx ? (int32_t*)take(bytes_idx) : nullptr;
    double* d_py = (double*)take(bytes_pyz);
    double* d_pz = (double*)take(bytes_pyz);
    unsigned* d_cover = (unsigned*)take(bytes_cover);
    RasterStatus init{};
    init.box[0] = init.box[2] = ~0ull;
    Mat16 m{};
    if (world16) {
      std::memcpy(m.e, world16, sizeof(m.e));
      m.has = 1;
    }
    RasterStatus st{};
    const int grid_v = (int)std::max<int64_t>(1, std::min<int64_t>((nv + kRasterThreads - 1) / kRasterThreads, 8LL * sms));
    const int grid_t = (int)std::max<int64_t>(1, std::min<int64_t>((T * 32 + kRasterThreads - 1) / kRasterThreads, 16LL * sms));
    const int grid_c = (int)std::max<int64_t>(1, std::min<int64_t>((cover_n + kRasterThreads - 1) / kRasterThreads, 4LL * sms));
    if ((e = cudaMemcpyAsync(d_st, &init, sizeof(init), cudaMemcpyHostToDevice, s)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d_pos, pos, bytes_pos, cudaMemcpyHostToDevice, s)) == cudaSuccess &&
        (!idx || (e = cudaMemcpyAsync(d_idx, idx, bytes_idx, cudaMemcpyHostToDevice, s)) == cudaSuccess) &&
        (e = cudaMemsetAsync(d_cover, 0, bytes_cover, s)) == cudaSuccess) {
      frontal_project_kernel<<<grid_v, kRasterThreads, 0, s>>>(d_pos, nv, m, d_py, d_pz, d_st);
      frontal_raster_kernel<<<grid_t, kRasterThreads, 0, s>>>(d_py, d_pz, nv, d_idx, T, res, d_cover, d_st);
      frontal_count_kernel<<<grid_c, kRasterThreads, 0, s>>>(d_cover, cover_n, d_st);
      if ((e = cudaGetLastError()) == cudaSuccess)
        e = cudaMemcpyAsync(&st, d_st, sizeof(st), cudaMemcpyDeviceToHost, s);
    }
    cudaError_t ef = cudaFreeAsync(base, s);
    cudaError_t es = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = ef != cudaSuccess ? ef : es;
    if (e != cudaSuccess) {
      rc = cuda_fail("aerosim_frontal_area_cuda", e);
    } else if (st.bad_index) {
      set_global_error("aerosim_frontal_area_cuda: triangle index out of range");
      rc = AEROSIM_ERR_ARG;
    } else {
      const double span_y = from_order_key(st.box[1]) - from_order_key(st.box[0]);
      const double span_z = from_order_key(st.box[3]) - from_order_key(st.box[2]);
      if (span_y > 1e-9 && span_z > 1e-9)
        *out = ((double)st.covered / ((double)res * res * 16)) * (span_y * span_z);
    }
  }
  cudaStreamDestroy(s);
  return rc;
}

// ---- mesh statistics ------------------------------------------------------

struct KeyHash {
  size_t operator()(const std::array<uint64_t, 3>& k) const {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (uint64_t v : k) h = (h ^ v) * 0xff51afd7ed558ccdull + (h >> 29);
    return (size_t)h;
  }
};

}  // namespace
}  // namespace aerosim

using namespace aerosim;

extern "C" {

int aerosim_parse_stl(const uint8_t* bytes, int64_t byte_count, float* positions, int64_t capacity_vertices,
                      int64_t* vertex_count, int32_t* format) {
  if (!vertex_count || byte_count < 0 || (byte_count > 0 && !bytes)) {
    set_global_error("aerosim_parse_stl: bad arguments");
    return AEROSIM_ERR_ARG;
  }
  std::vector<float> v;
  int fmt = AEROSIM_STL_ASCII;
  int rc = AEROSIM_OK;
  if (byte_count < 84) {
    rc = parse_ascii(bytes, byte_count, &v);
  } else {
    const uint32_t faces = read_u32le(bytes + 80);
    const uint64_t expected = 84 + (uint64_t)faces * 50;
    if (expected == (uint64_t)byte_count) {
      fmt = AEROSIM_STL_BINARY;
      parse_binary(bytes, faces, &v);
    } else if (header_says_solid(bytes, byte_count) && contains(bytes, byte_count, "facet") &&
               contains(bytes, byte_count, "vertex")) {
      rc = parse_ascii(bytes, byte_count, &v);
    } else if (expected <= (uint64_t)byte_count && faces > 0) {
      fmt = AEROSIM_STL_BINARY;
      parse_binary(bytes, faces, &v);
    } else {
      set_global_error("Invalid or corrupted STL file.");
      rc = AEROSIM_ERR_FORMAT;
    }
  }
  if (rc != AEROSIM_OK) return rc;
  *vertex_count = (int64_t)(v.size() / 3);
  if (format) *format = fmt;
  if (!positions) return AEROSIM_OK;
  if (capacity_vertices < *vertex_count) {
    set_global_error("aerosim_parse_stl: positions buffer too small");
    return AEROSIM_ERR_ARG;
  }
  std::memcpy(positions, v.data(), v.size() * sizeof(float));
  return AEROSIM_OK;
}

int aerosim_normalize_and_center(float* positions, int64_t vertex_count, int32_t* auto_scaled_from_mm) {
  if (vertex_count < 0 || (vertex_count > 0 && !positions)) {
    set_global_error("aerosim_normalize_and_center: bad arguments");
    return AEROSIM_ERR_ARG;
  }
  if (auto_scaled_from_mm) *auto_scaled_from_mm = 0;
  if (vertex_count == 0) return AEROSIM_OK;  // Box3 is empty: center and size are zero
  double mn[3], mx[3];
  bounding_box(positions, vertex_count, mn, mx);
  double t[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  for (int k = 0; k < 3; ++k) t[12 + k] = -((mn[k] + mx[k]) * 0.5);  // Box3.getCenter
  apply_matrix4_f32(t, positions, vertex_count);
  // translate() recomputed the same Box3 object, so the size is the centred box's.
  bounding_box(positions, vertex_count, mn, mx);
  const double max_dim = js_max(js_max(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
  if (max_dim > 10.0) {
    const double s = max_dim > 50 ? 0.001 : 1.0 / max_dim;
    const double sc[16] = {s, 0, 0, 0, 0, s, 0, 0, 0, 0, s, 0, 0, 0, 0, 1};
    apply_matrix4_f32(sc, positions, vertex_count);
    if (auto_scaled_from_mm) *auto_scaled_from_mm = 1;
  }
  return AEROSIM_OK;
}

int aerosim_model_matrix(const aerosim_model_transform* transform, double* world16) {
  if (!transform || !world16) {
    set_global_error("aerosim_model_matrix: bad arguments");
    return AEROSIM_ERR_ARG;
  }
  compose_model_matrix(*transform, world16);
  return AEROSIM_OK;
}

int aerosim_frontal_area_cuda(int32_t device, const float* positions, int64_t vertex_count, const int32_t* indices,
                              int64_t index_count, const double* world16, int32_t grid_resolution, double* out) {
  if (!out || grid_resolution <= 0 || grid_resolution > 16384 || vertex_count < 0 ||
      (vertex_count > 0 && !positions) || index_count < 0 || (index_count > 0 && !indices)) {
    set_global_error("aerosim_frontal_area_cuda: bad arguments");
    return AEROSIM_ERR_ARG;
  }
  return frontal_area_cuda(device, positions, vertex_count, indices, index_count, world16, grid_resolution, out);
}

int aerosim_compute_mesh_stats(const float* positions, int64_t vertex_count, const int32_t* indices, int64_t index_count,
                       const aerosim_model_transform* transform, int32_t device, aerosim_mesh_stats* out) {
  if (!out || !transform || vertex_count < 0 || (vertex_count > 0 && !positions) || index_count < 0 ||
      (index_count > 0 && !indices)) {
    set_global_error("aerosim_compute_mesh_stats: bad arguments");
    return AEROSIM_ERR_ARG;
  }
  *out = aerosim_mesh_stats{};
  const int64_t T = indices ? index_count / 3 : vertex_count / 3;
  double m[16];
  compose_model_matrix(*transform, m);
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  double s6 = 0.0;
  const bool edges = T <= 100000;
  std::unordered_map<std::array<uint64_t, 3>, int32_t, KeyHash> ids;
  std::unordered_map<uint64_t, int32_t> edge_counts;
  if (edges) {
    ids.reserve((size_t)T * 2);
    edge_counts.reserve((size_t)T * 3);
  }
  auto vertex_id = [&](const double* p) {
    std::array<uint64_t, 3> k;
    for (int c = 0; c < 3; ++c) {
      const double r = js_round(p[c] * 1e5);
      std::memcpy(&k[c], &r, 8);
    }
    auto it = ids.emplace(k, (int32_t)ids.size());
    return it.first->second;
  };
  auto add_edge = [&](int32_t a, int32_t b) {
    if (a == b) return;
    const uint64_t key = a < b ? ((uint64_t)a << 32 | (uint32_t)b) : ((uint64_t)b << 32 | (uint32_t)a);
    ++edge_counts[key];
  };
  for (int64_t t = 0; t < T; ++t) {
    double v[3][3];
    for (int k = 0; k < 3; ++k) {
      const int64_t i = indices ? indices[t * 3 + k] : t * 3 + k;
      if (i < 0 || i >= vertex_count) {
        set_global_error("aerosim_compute_mesh_stats: triangle index out of range");
        return AEROSIM_ERR_ARG;
      }
      for (int c = 0; c < 3; ++c) v[k][c] = positions[i * 3 + c];
    }
    if (edges) {
      const int32_t k0 = vertex_id(v[0]), k1 = vertex_id(v[1]), k2 = vertex_id(v[2]);
      add_edge(k0, k1);
      add_edge(k1, k2);
      add_edge(k2, k0);
    }
    for (int k = 0; k < 3; ++k) {
      apply_matrix4(m, v[k][0], v[k][1], v[k][2]);
      for (int c = 0; c < 3; ++c) {
        mn[c] = js_min(mn[c], v[k][c]);
        mx[c] = js_max(mx[c], v[k][c]);
      }
    }
    s6 += v[0][0] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]) + v[0][1] * (v[1][2] * v[2][0] - v[1][0] * v[2][2]) +
          v[0][2] * (v[1][0] * v[2][1] - v[1][1] * v[2][0]);
  }
  int64_t open = 0;
  for (const auto& kv : edge_counts) open += kv.second != 2;
  double area = 0.0;
  const int rc = device >= 0 ? frontal_area_cuda(device, positions, vertex_count, indices, index_count, m, 512, &area)
                             : aerosim_frontal_area(positions, vertex_count, indices, index_count, m, 512, &area);
  if (rc != AEROSIM_OK) return rc;
  const double sx = js_max(0, mx[0] - mn[0]), sy = js_max(0, mx[1] - mn[1]), sz = js_max(0, mx[2] - mn[2]);
  out->triangle_count = T;
  out->vertex_count = vertex_count;
  out->open_edge_count = open;
  out->is_watertight = open == 0 && T > 0;
  out->bounding_box_size[0] = sx;
  out->bounding_box_size[1] = sy;
  out->bounding_box_size[2] = sz;
  out->characteristic_length = js_max(1e-4, sx);
  out->frontal_area = area;
  out->volume = std::fabs(s6) / 6.0;
  return AEROSIM_OK;
}

}  // extern "C"
