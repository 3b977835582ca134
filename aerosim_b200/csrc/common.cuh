// Shared device definitions: the D3Q19 lattice, population storage codecs and
// NaN-propagating min/max with JavaScript's Math.min / Math.max semantics.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

namespace aerosim {

// D3Q19 velocity set and opposite table, src/solver/lbmConstants.ts:10-48
// (same ordering: rest, 6 faces, 12 edges).
__host__ __device__ constexpr int cx_of(int d) {
  return (d == 1 || d == 7 || d == 9 || d == 11 || d == 13) ? 1
       : (d == 2 || d == 8 || d == 10 || d == 12 || d == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cy_of(int d) {
  return (d == 3 || d == 7 || d == 10 || d == 15 || d == 17) ? 1
       : (d == 4 || d == 8 || d == 9 || d == 16 || d == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cz_of(int d) {
  return (d == 5 || d == 11 || d == 14 || d == 15 || d == 18) ? 1
       : (d == 6 || d == 12 || d == 13 || d == 16 || d == 17) ? -1 : 0;
}
__host__ __device__ constexpr int opp_of(int d) { return d == 0 ? 0 : ((d & 1) ? d + 1 : d - 1); }

// Exact double weights 1/3, 1/18, 1/36 (LBM_WEIGHTS) ...
__host__ __device__ constexpr double w64_of(int d) {
  return d == 0 ? 1.0 / 3.0 : (d <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
}
// ... and the float copy promoted to double (LBM_WEIGHTS_F32), used by the
// reference's collision and force integrator.
__host__ __device__ constexpr double w32_of(int d) { return (double)(float)w64_of(d); }
__host__ __device__ constexpr float wf_of(int d) { return (float)w64_of(d); }

constexpr uint8_t CELL_FLUID = 0, CELL_SOLID = 1, CELL_BOUNDARY = 2;
// Cell class byte used by the solver kernels: the low 2 bits are the reference
// flag; CLS_NEAR marks a non-solid cell with at least one SOLID clamped pull source.
constexpr uint8_t CLS_FLAG_MASK = 3, CLS_NEAR = 4;

// Math.min / Math.max: NaN if either operand is NaN.
__host__ __device__ inline double js_min(double a, double b) {
  return (a != a || b != b) ? a + b : (a < b ? a : b);
}
__host__ __device__ inline double js_max(double a, double b) {
  return (a != a || b != b) ? a + b : (a > b ? a : b);
}

// FP16 storage scale: (f - w) * 2^15 keeps the deviations of a near-equilibrium
// flow inside half's normal range (6.1e-5 .. 65504) with its full 11-bit mantissa.
constexpr float F16S_SCALE = 32768.0f;
constexpr float F16S_INV_SCALE = 1.0f / 32768.0f;

// Population storage codecs.  All six expose the same interface in terms of the
// deviation h = f - w_d from the rest weight (the form the FP32 collision works in)
// and of the full value f (the form the FP64 paths work in):
//   h_of(raw, d), raw_of_h(h, d)  -- float deviation
//   f_of(raw, d), raw_of_f(f, d)  -- double value
// d is a loop index of fully unrolled loops, so w_d folds to a constant.
// kRawMoments marks the codecs of stored deviations, the ones the FP32-arithmetic
// kernels run on: those take the stored values as they are (raw()) and apply the storage
// scale kRawScale and the pending mean-density rescale to the collision's ten moments
// instead of to the 19 values (a full f would lose its small moments to cancellation
// against the rest weights).
struct StoreF32 {
  using T = float;
  // FP32-collision output in the storage domain: value = kOutScale * h + kOutW * w_d
  static constexpr float kOutScale = 1.0f, kOutW = 1.0f;
  static constexpr bool kCompensate = false;
  static constexpr bool kRawMoments = false;
  static constexpr float kRawScale = 1.0f;
  __device__ __forceinline__ static float raw(T v) { return v; }
  __device__ __forceinline__ static T store(float v) { return v; }
  __device__ __forceinline__ static float h_of(T v, int d) { return v - wf_of(d); }
  __device__ __forceinline__ static T raw_of_h(float h, int d) { return wf_of(d) + h; }
  __device__ __forceinline__ static double f_of(T v, int) { return (double)v; }
  __device__ __forceinline__ static T raw_of_f(double f, int) { return (float)f; }
};
// FP32 storage of the deviation f - w_d, for the FP32-arithmetic kernels: the collision
// takes the stored deviations as they are and decodes its ten moments (kRawMoments), and
// the deviations keep float's full relative precision (storing f = w_d + h rounds h to
// the ulp of w_d).  The bit-parity mode keeps StoreF32, the reference's own values.
struct StoreF32S {
  using T = float;
  static constexpr float kOutScale = 1.0f, kOutW = 0.0f;
  static constexpr bool kCompensate = false;
  static constexpr bool kRawMoments = true;
  static constexpr float kRawScale = 1.0f;
  __device__ __forceinline__ static float raw(T v) { return v; }
  __device__ __forceinline__ static T store(float v) { return v; }
  __device__ __forceinline__ static float h_of(T v, int) { return v; }
  __device__ __forceinline__ static T raw_of_h(float h, int) { return h; }
  __device__ __forceinline__ static double f_of(T v, int d) { return (double)wf_of(d) + (double)v; }
  __device__ __forceinline__ static T raw_of_f(double f, int d) { return (float)(f - (double)wf_of(d)); }
};
struct StoreF64 {
  using T = double;
  static constexpr float kOutScale = 1.0f, kOutW = 1.0f;
  static constexpr bool kCompensate = false;
  static constexpr bool kRawMoments = false;
  static constexpr float kRawScale = 1.0f;
  __device__ __forceinline__ static float raw(T v) { return (float)v; }
  __device__ __forceinline__ static T store(float v) { return (double)v; }
  __device__ __forceinline__ static float h_of(T v, int d) { return (float)(v - w64_of(d)); }
  __device__ __forceinline__ static T raw_of_h(float h, int d) { return w64_of(d) + (double)h; }
  __device__ __forceinline__ static double f_of(T v, int) { return v; }
  __device__ __forceinline__ static T raw_of_f(double f, int) { return f; }
};
struct StoreF16S {
  using T = __half;
  static constexpr float kOutScale = F16S_SCALE, kOutW = 0.0f;
  static constexpr bool kCompensate = false;
  static constexpr bool kRawMoments = true;
  static constexpr float kRawScale = F16S_INV_SCALE;
  __device__ __forceinline__ static float raw(T v) { return __half2float(v); }
  __device__ __forceinline__ static T store(float v) { return __float2half_rn(v); }
  __device__ __forceinline__ static float h_of(T v, int) { return __half2float(v) * F16S_INV_SCALE; }
  __device__ __forceinline__ static T raw_of_h(float h, int) { return __float2half_rn(h * F16S_SCALE); }
  __device__ __forceinline__ static double f_of(T v, int d) { return (double)wf_of(d) + (double)h_of(v, d); }
  __device__ __forceinline__ static T raw_of_f(double f, int d) { return raw_of_h((float)(f - (double)wf_of(d)), d); }
};
struct StoreBF16S {
  using T = __nv_bfloat16;
  static constexpr float kOutScale = 1.0f, kOutW = 0.0f;
  static constexpr bool kCompensate = false;
  static constexpr bool kRawMoments = true;
  static constexpr float kRawScale = 1.0f;
  __device__ __forceinline__ static float raw(T v) { return __bfloat162float(v); }
  __device__ __forceinline__ static T store(float v) { return __float2bfloat16_rn(v); }
  __device__ __forceinline__ static float h_of(T v, int) { return __bfloat162float(v); }
  __device__ __forceinline__ static T raw_of_h(float h, int) { return __float2bfloat16_rn(h); }
  __device__ __forceinline__ static double f_of(T v, int d) { return (double)wf_of(d) + (double)h_of(v, d); }
  __device__ __forceinline__ static T raw_of_f(double f, int d) { return raw_of_h((float)(f - (double)wf_of(d)), d); }
};
// FP16 shifted storage with mass-compensated rounding: the values are those of StoreF16S,
// but wherever a step kernel stores a cell it rounds the 18 moving populations first and
// gives the rest population what their rounded values leave of the cell's deviation sum
// (compensate_cell and its lane form below, and the pair path of pair_segment), i.e. the
// rest population absorbs their rounding errors before it rounds itself.  The stored
// deviations of a cell then sum to the computed ones up to the single rounding of f_0,
// whose half-precision ulp is 4-8 times finer than the moving populations' near
// equilibrium (|f_0 - w_0| is of the order of 1.5 w_0 u^2, |f_d - w_d| of 3 w_d |c_d . u|),
// where the uncompensated error grows like the square root of 18 roundings.  Initial,
// written and rescaled fields round per value, like StoreF16S.
struct StoreF16C : StoreF16S {
  static constexpr bool kCompensate = true;
};

// Mass-compensated rounding of one cell's 19 values v (storage domain, direction order):
// the rounding errors of directions 1..18 move into direction 0.  No-op for the codecs
// without kCompensate.
template <class S>
__device__ __forceinline__ void compensate_cell(float (&v)[19]) {
  if constexpr (S::kCompensate) {
    float e = 0.0f;
#pragma unroll
    for (int d = 1; d < 19; ++d) e += v[d] - S::raw(S::store(v[d]));
    v[0] += e;
  }
}
// The same for a cell written lane-transposed (lane d < 19 holds direction d); every lane
// of the warp calls it.
template <class S>
__device__ __forceinline__ float compensate_lanes(float v, int lane) {
  if constexpr (S::kCompensate) {
    float e = (lane >= 1 && lane < 19) ? v - S::raw(S::store(v)) : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if (lane == 0) v += e;
  }
  return v;
}

// Storage order of the directions inside a row block ("slots"): directions that pull
// from the same source row (same c_y, c_z) are adjacent, so one bulk copy brings all
// of them.  Groups: (0,0): 0 1 2 | (1,0): 3 7 10 | (-1,0): 4 8 9 | (0,1): 5 11 14 |
// (0,-1): 6 12 13 | (1,1): 15 | (-1,-1): 16 | (1,-1): 17 | (-1,1): 18.
__host__ __device__ constexpr int slot_of(int d) {
  return d <= 3 ? d : d == 4 ? 6 : d == 5 ? 9 : d == 6 ? 12 : d == 7 ? 4 : d == 8 ? 7 : d == 9 ? 8
       : d == 10 ? 5 : d == 11 ? 10 : d == 12 ? 13 : d == 13 ? 14 : d == 14 ? 11 : d;
}
constexpr int kGroups = 9;
__host__ __device__ constexpr int group_first(int g) { return g < 5 ? 3 * g : 10 + g; }
__host__ __device__ constexpr int group_count(int g) { return g < 5 ? 3 : 1; }
__host__ __device__ constexpr int group_cy(int g) {
  return g == 1 || g == 5 || g == 7 ? 1 : g == 2 || g == 6 || g == 8 ? -1 : 0;
}
__host__ __device__ constexpr int group_cz(int g) {
  return g == 3 || g == 5 || g == 8 ? 1 : g == 4 || g == 6 || g == 7 ? -1 : 0;
}

// Population memory layout.  Element (d, x, row) of a lattice with rows = ny * nz
// x-rows lives at  row * rstride + slot(d) * dstride + x.
//   solver (grouped = 1): row blocks -- the 19 direction rows of one x-row are
//     contiguous, dstride = pitch, rstride = 19 * pitch, pitch = nx rounded up to 32
//     (so each row starts on a 16-byte boundary and the 3-row groups are one copy);
//   reference order (grouped = 0): SoA f[d * N + cell] as the reference stores it,
//     dstride = plane = N, rstride = pitch = nx.
// The cell-class array of the solver has one byte per cell with the same pitch.
struct Layout {
  long long plane;    // elements per direction over the lattice (19 * plane in all)
  long long rstride;  // elements between consecutive x-rows of one direction
  long long dstride;  // elements between consecutive slots of one x-row
  int pitch;          // elements per x-row
  int nx, ny, nz;
  int grouped;
  __host__ __device__ int slot(int d) const { return grouped ? slot_of(d) : d; }
  __host__ __device__ long long at(int d, long long cell) const {
    const long long r = cell / nx;
    return r * rstride + (long long)slot(d) * dstride + (cell - r * nx);
  }
  __host__ __device__ long long cls_at(long long cell) const {
    const long long r = cell / nx;
    return r * pitch + (cell - r * nx);
  }
  // the same two by x-row (iy + ny * iz) and x
  __host__ __device__ long long at_row(int d, long long row, int x) const {
    return row * rstride + (long long)slot(d) * dstride + x;
  }
  __host__ __device__ long long cls_at_row(long long row, int x) const { return row * pitch + x; }
};

__host__ inline Layout make_layout(int nx, int ny, int nz) {
  Layout L;
  L.nx = nx; L.ny = ny; L.nz = nz;
  L.pitch = (nx + 31) / 32 * 32;
  L.plane = (long long)ny * nz * L.pitch;
  L.dstride = L.pitch;
  L.rstride = 19LL * L.pitch;
  L.grouped = 1;
  return L;
}

// The reference's own SoA order (dense, unpadded).
__host__ inline Layout make_reference_layout(int nx, int ny, int nz) {
  Layout L;
  L.nx = nx; L.ny = ny; L.nz = nz;
  L.pitch = nx;
  L.plane = (long long)nx * ny * nz;
  L.dstride = L.plane;
  L.rstride = nx;
  L.grouped = 0;
  return L;
}

// Device-resident solver state shared across steps.  Slot [s & 1] belongs to step s.
struct StepState {
  unsigned long long rho_sum[2];   // fixed-point sum of post-boundary densities
  unsigned int ticket[2];          // CTA completion counters (last-CTA finalisation)
  unsigned int next_item[2];       // next work item of step s handed to a CTA (dynamic deal)
  int apply[2];                    // 1 if step s triggered the mean-density rescale
  double corr[2];                  // 1 / meanRho of step s
  double cumulative_rescale;       // product of applied corrections
  long long rescale_count;
  int nan_seen;                    // a non-finite density reached the rescale sum
  int error;                       // kernel-reported error code (0 = none)
};

}  // namespace aerosim
