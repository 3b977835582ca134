// D3Q19 solver kernels for sm_100a: fused pull-stream + Bouzidi + regularized
// collision + Smagorinsky + domain boundary conditions + mean-density rescale,
// the FP64 momentum-exchange force reduction, initialisation and readback.
//
// The kernels restate src/solver/lbmCpuReference.ts (the reference's CPU solver,
// which the WGSL shaders only approximate) for the GPU:
//   * one CTA owns complete x-rows, so the inlet (ix = 0) and outlet (ix = nx-1)
//     of a row read the density / populations of ix = 1 and ix = nx-2 through shared
//     memory inside the same launch -- the reference's phase order (collide, then
//     inlet/outlet, then walls, lbmCpuReference.ts:323-429) without a second pass;
//   * wall conditions depend only on the cell's own post-collision moments, so they
//     are applied in registers after the outlet has captured the pre-wall values;
//   * the mean-density rescale (:431-455) is a grid-wide reduction: densities are
//     summed as exact 2^-25 fixed-point integers, the last CTA forms 1/meanRho and the
//     conditional rescale is folded into the next step's population loads.  The
//     float-valued sum of the reference is exact in double, so this reproduces it
//     bit for bit;
//   * one launch per time step; all per-step traffic is the 19 population reads, the
//     19 writes and one class byte per cell.
#pragma once
#include "common.cuh"

namespace aerosim {

enum { MODE_FAST = 0, MODE_MIRROR = 1, MODE_F64 = 2 };

// Resident CTAs per SM the FP32 step kernel is register-budgeted for.
#ifndef AEROSIM_FAST_MIN_BLOCKS
#define AEROSIM_FAST_MIN_BLOCKS 2
#endif

struct NearLink;

struct StepArgs {
  const void* fsrc;
  void* fdst;
  const uint8_t* cls;     // pitched cell classes
  const int32_t* bmap;    // dense boundaryIndexMap
  const float* q;
  float* mux;             // dense macro outputs
  float* muy;
  float* muz;
  float* mrho;
  const double* abl;      // [ny] Math.min(1.15, 0.35 + 0.8 * yFrac^0.3)
  const double* sin_tab;  // [120 * ny] sin(step * 0.15 + (iy / ny) * PI * 2)
  StepState* st;
  Layout L;
  long long fluid_count;  // non-solid cells
  const int32_t* near_cells;  // cells with a solid pull source, x faces excluded
  long long n_near;
  const NearLink* links;      // [19][n_near] link table of the near-wall cells
  int stages;             // depth of the shared-memory ring
  int step_index;
  int write_macro;
  int ground_no_slip;
  double u_inlet, tau0, k_smag;  // k_smag = 18 * SQRT2 * Cs^2
};

struct ForceArgs {
  const void* f;
  const uint8_t* cls;
  const int32_t* bcells;
  const float* q;
  const StepState* st;
  double* partials;       // [gridDim.x * 8]
  unsigned int* ticket;
  double* out;            // [8]: fx fy fz mx my mz cut_face_links blocks
  Layout L;
  long long B;
  int prev_slot;          // state slot of the step that produced f (-1: none)
};

template <class T>
struct MacroOf { using type = float; };
template <>
struct MacroOf<double> { using type = double; };

// Fixed-point weight of a density in the rescale sum.  A float density in
// [0.25, 2) is an exact multiple of 2^-25; double densities use 2^-36.
__device__ __forceinline__ long long rho_fixed(float r) { return (long long)__float2int_rn(r * 33554432.0f); }
__device__ __forceinline__ long long rho_fixed(double r) { return llrint(r * 68719476736.0); }
__device__ __forceinline__ double rho_unfixed(long long s, float) { return (double)s * (1.0 / 33554432.0); }
__device__ __forceinline__ double rho_unfixed(long long s, double) { return (double)s * (1.0 / 68719476736.0); }

// computeEquilibrium (lbmConstants.ts:142-152) with the exact double weights,
// evaluated literally: W * rho * (1 + cu + 0.5 cu cu - 1.5 uSq).
__device__ __forceinline__ double feq64(int d, double rho, double ux, double uy, double uz) {
  const double cu = 3.0 * ((double)cx_of(d) * ux + (double)cy_of(d) * uy + (double)cz_of(d) * uz);
  const double uSq = ux * ux + uy * uy + uz * uz;
  return w64_of(d) * rho * (1.0 + cu + 0.5 * cu * cu - 1.5 * uSq);
}

// c_d . u with the zero components left out (d is a constant after unrolling).
__device__ __forceinline__ float dotc(int d, float x, float y, float z) {
  const int a = cx_of(d), b = cy_of(d), c = cz_of(d);
  float s = a ? (a > 0 ? x : -x) : (b ? (b > 0 ? y : -y) : (c ? (c > 0 ? z : -z) : 0.0f));
  if (a && b) s += b > 0 ? y : -y;
  if ((a || b) && c) s += c > 0 ? z : -z;
  return s;
}

// FP32 equilibrium deviation feq_d - w_d for the fast path.
__device__ __forceinline__ float heq32(int d, float rho, float ux, float uy, float uz) {
  const float cu = 3.0f * dotc(d, ux, uy, uz);
  const float uSq = ux * ux + uy * uy + uz * uz;
  return wf_of(d) * ((rho - 1.0f) + rho * (cu + 0.5f * cu * cu - 1.5f * uSq));
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }



// ---------------------------------------------------------------------------
// Collision kernels for one cell.  In: pulled values v[19] (already rescaled).
// Out: post-collision values in v[19] (double modes: the value to store, fast mode:
// the deviation h = f - w) and the moments (rho, u) with the reference's clamps.
// ---------------------------------------------------------------------------

// Double modes, lbmCpuReference.ts:226-309, evaluated in the reference's order.
// MIRROR additionally rounds fLocal and feq to float exactly where the reference
// stores them in Float32Arrays and uses the float-rounded weights.
template <bool MIRROR>
__device__ __forceinline__ void collide_f64(double (&v)[19], double& r, double& ux, double& uy,
                                            double& uz, double tau0, double k_smag) {
  double fl[19];
  r = 0.0; ux = 0.0; uy = 0.0; uz = 0.0;
  // Terms with a zero lattice component only add a signed zero to these sums, which
  // leaves every value the reference can produce unchanged, so they are skipped.
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    fl[d] = MIRROR ? (double)(float)v[d] : v[d];
    r += v[d];
    if (cx_of(d)) ux += (double)cx_of(d) * v[d];
    if (cy_of(d)) uy += (double)cy_of(d) * v[d];
    if (cz_of(d)) uz += (double)cz_of(d) * v[d];
  }
  r = js_max(0.5, js_min(1.8, r));
  const double ir = 1.0 / r;
  ux *= ir; uy *= ir; uz *= ir;
  const double m2 = ux * ux + uy * uy + uz * uz;
  if (m2 > 0.22 * 0.22) {
    const double s = 0.22 / sqrt(m2);
    ux *= s; uy *= s; uz *= s;
  }
  const double uSq = ux * ux + uy * uy + uz * uz;
  double pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
  double fe[19];
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    const double cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
    const double cu = 3.0 * (cx * ux + cy * uy + cz * uz);
    const double eq = w32_of(d) * r * (1.0 + cu + 0.5 * cu * cu - 1.5 * uSq);
    fe[d] = MIRROR ? (double)(float)eq : eq;
    const double fn = fl[d] - eq;
    if (cx_of(d)) pxx += cx * cx * fn;
    if (cy_of(d)) pyy += cy * cy * fn;
    if (cz_of(d)) pzz += cz * cz * fn;
    if (cx_of(d) * cy_of(d)) pxy += cx * cy * fn;
    if (cx_of(d) * cz_of(d)) pxz += cx * cz * fn;
    if (cy_of(d) * cz_of(d)) pyz += cy * cz * fn;
  }
  const double pn = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + 2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
  const double tau = 0.5 * (tau0 + sqrt(tau0 * tau0 + (k_smag * pn) / r));
  const double om = 1.0 / js_max(0.5015, js_min(1.95, tau));
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    const double cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
    const double qxx = cx * cx - 1.0 / 3.0, qyy = cy * cy - 1.0 / 3.0, qzz = cz * cz - 1.0 / 3.0;
    const double qxy = cx * cy, qxz = cx * cz, qyz = cy * cz;
    const double f1 = 4.5 * w32_of(d) *
                      (qxx * pxx + qyy * pyy + qzz * pzz + 2.0 * (qxy * pxy + qxz * pxz + qyz * pyz));
    v[d] = fe[d] + (1.0 - om) * f1;
  }
}

// FP32 path on deviations h_d = f_d - w_d, organised by the 9 opposite pairs
// (2p+1, 2p+2) of D3Q19 so that no multiplication by a zero lattice component is
// left for the compiler (IEEE semantics forbid folding 0 * x):
//   pair sums s_p = h_a + h_b give rho - 1 and the second moments,
//   pair differences t_p = h_a - h_b give the momentum;
//   Pi^neq = sum cc h - (rho - 1)/3 I - rho u u  (= the reference's sum cc (f - feq));
//   post-collision h_a,b = E_p +- O_p with the even part
//   E = w (rho - 1 - 1.5 rho u^2 + 4.5 rho (c.u)^2 + (1 - omega) 4.5 Q:Pi) and the odd
//   part O = 3 w rho (c.u), Q:Pi = c.Pi.c - tr(Pi) / 3.
// Pairs: 0 (+-x), 1 (+-y), 2 (+-z), 3 +-(x+y), 4 +-(x-y), 5 +-(x+z), 6 +-(x-z),
// 7 +-(y+z), 8 +-(y-z), matching lbmConstants.ts:10-32.
__device__ __forceinline__ float frcp(float x) { return __frcp_rn(x); }

__device__ __forceinline__ void collide_f32(float (&h)[19], float& r, float& ux, float& uy,
                                            float& uz, float tau0, float k_smag) {
  float s[9], t[9];
#pragma unroll
  for (int p = 0; p < 9; ++p) {
    s[p] = h[2 * p + 1] + h[2 * p + 2];
    t[p] = h[2 * p + 1] - h[2 * p + 2];
  }
  const float dr = h[0] + ((s[0] + s[1]) + (s[2] + s[3]) + ((s[4] + s[5]) + (s[6] + s[7])) + s[8]);
  const float jx = (t[0] + t[3]) + (t[4] + t[5]) + t[6];
  const float jy = (t[1] + t[3]) - t[4] + (t[7] + t[8]);
  const float jz = (t[2] + t[5]) - t[6] + (t[7] - t[8]);
  const float sxx = (s[0] + s[3]) + (s[4] + s[5]) + s[6];
  const float syy = (s[1] + s[3]) + (s[4] + s[7]) + s[8];
  const float szz = (s[2] + s[5]) + (s[6] + s[7]) + s[8];
  const float sxy = s[3] - s[4], sxz = s[5] - s[6], syz = s[7] - s[8];

  r = fmaxf(0.5f, fminf(1.8f, 1.0f + dr));
  if (dr != dr) r = dr;  // keep NaN visible like Math.min / Math.max
  const float ir = frcp(r);
  ux = jx * ir; uy = jy * ir; uz = jz * ir;
  float uSq = ux * ux + uy * uy + uz * uz;
  if (uSq > 0.0484f) {  // Mach limiter |u| <= 0.22
    const float sc = 0.22f * rsqrtf(uSq);
    ux *= sc; uy *= sc; uz *= sc;
    uSq = ux * ux + uy * uy + uz * uz;
  }
  const float drc = r - 1.0f;
  const float d3 = drc * (1.0f / 3.0f);
  const float rux = r * ux, ruy = r * uy, ruz = r * uz;
  const float pxx = fmaf(-rux, ux, sxx - d3);
  const float pyy = fmaf(-ruy, uy, syy - d3);
  const float pzz = fmaf(-ruz, uz, szz - d3);
  const float pxy = fmaf(-rux, uy, sxy);
  const float pxz = fmaf(-rux, uz, sxz);
  const float pyz = fmaf(-ruy, uz, syz);
  const float off = pxy * pxy + pxz * pxz + pyz * pyz;
  const float pn = sqrtf(pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * off);
  const float tau = 0.5f * (tau0 + sqrtf(fmaf(tau0, tau0, k_smag * pn * ir)));
  const float om = frcp(fmaxf(0.5015f, fminf(1.95f, tau)));
  const float g = (1.0f - om) * 4.5f;
  const float tr3 = (pxx + pyy + pzz) * (1.0f / 3.0f);
  const float A = fmaf(-1.5f * r, uSq, drc);
  constexpr float w0 = 1.0f / 3.0f, w1 = 1.0f / 18.0f, w2 = 1.0f / 36.0f;
  // rest population
  h[0] = w0 * fmaf(-g, tr3, A);
  // faces: Q:Pi = P_aa - tr/3
  const float k1 = w1 * 4.5f * r, o1 = w1 * 3.0f * r, g1 = w1 * g, a1 = w1 * A;
  const float qx = pxx - tr3, qy = pyy - tr3, qz = pzz - tr3;
  const float cuf[3] = {ux, uy, uz};
  const float qf[3] = {qx, qy, qz};
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const float E = fmaf(k1, cuf[p] * cuf[p], fmaf(g1, qf[p], a1));
    const float O = o1 * cuf[p];
    h[2 * p + 1] = E + O;
    h[2 * p + 2] = E - O;
  }
  // edges: Q:Pi = P_aa + P_bb - tr/3 +- 2 P_ab
  const float k2 = w2 * 4.5f * r, o2 = w2 * 3.0f * r, g2 = w2 * g, a2 = w2 * A;
  const float bxy = pxx + pyy - tr3, bxz = pxx + pzz - tr3, byz = pyy + pzz - tr3;
  const float cue[6] = {ux + uy, ux - uy, ux + uz, ux - uz, uy + uz, uy - uz};
  const float qe[6] = {fmaf(2.0f, pxy, bxy), fmaf(-2.0f, pxy, bxy), fmaf(2.0f, pxz, bxz),
                       fmaf(-2.0f, pxz, bxz), fmaf(2.0f, pyz, byz), fmaf(-2.0f, pyz, byz)};
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const float E = fmaf(k2, cue[p] * cue[p], fmaf(g2, qe[p], a2));
    const float O = o2 * cue[p];
    h[2 * p + 7] = E + O;
    h[2 * p + 8] = E - O;
  }
}

// ---------------------------------------------------------------------------
// 1-D bulk-copy (TMA) and mbarrier helpers: global -> shared row copies whose
// completion is counted in bytes on a shared-memory mbarrier.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait: gives up after `limit` polls (each poll suspends the thread briefly).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
constexpr int kWaitLimit = 1 << 22;
constexpr int kConsumerWarps = 8;                      // warps 0..7: x-rows
constexpr int kProducerWarp = kConsumerWarps;          // warp 8: bulk copies
constexpr int kHelperWarp = kConsumerWarps + 1;        // warp 9: near-wall cells
constexpr int kStepThreads = (kConsumerWarps + 2) * 32;
enum { STEP_ERR_PIPELINE_TIMEOUT = 1 };

// Thread -> cell mapping of a row: cell ix = slot - shift with slot = lane + 32 * warp
// + tx_span * chunk.  shift = 1 when nx = 1 (mod 32) keeps the cell pairs (0, 1) and
// (nx-2, nx-1) inside one warp, so the inlet and outlet exchange stays warp-local.
__host__ __device__ inline int row_shift(int nx) { return (nx % 32 == 1) ? 1 : 0; }
__host__ __device__ inline int row_span(int nx) {  // threads along x (multiple of 32, <= 256)
  const int t = (nx + row_shift(nx) + 31) / 32 * 32;
  return t > kConsumerWarps * 32 ? kConsumerWarps * 32 : t;
}
__host__ __device__ inline int rows_per_item(int nx) { return (kConsumerWarps * 32) / row_span(nx); }

// Dynamic shared memory of the step kernel: `stages` slots, each holding the 19
// source row segments and the class bytes of the item's destination rows, plus a
// full and an empty mbarrier per slot.
__host__ __device__ inline size_t step_stage_bytes(const Layout& L, size_t elem) {
  return (size_t)rows_per_item(L.nx) * (19 * (size_t)L.pitch * elem + (size_t)L.pitch);
}
// Guard bytes around the slots: the x-face cells read (and discard) one element
// before the first row or past the end of a row.
constexpr size_t kSmemGuard = 64;
__host__ __device__ inline size_t step_smem_bytes(const Layout& L, int stages, size_t elem) {
  return kSmemGuard + (size_t)stages * step_stage_bytes(L, elem) + kSmemGuard + 16 * (size_t)stages + 16 +
         2 * (size_t)L.ny * sizeof(double) + (size_t)stages * rows_per_item(L.nx) * sizeof(int2);
}

// ---------------------------------------------------------------------------
// One launch per time step, main_kernel: a persistent CTA of 8 consumer warps, a
// producer warp and a helper warp.  The producer streams x-rows into the shared
// ring with bulk copies; the consumers walk the rows: pull, collide, wall
// conditions (:375-429), inlet and outlet (:323-373), store.  Meanwhile the helper
// warp takes the CTA's share of the near-wall cells (Bouzidi, :196-221; one lane
// per cell from a link table built with the voxel grid).  A near-wall cell at
// ix = 1 or nx-2 carries its row's inlet or outlet, which need its post-collision
// values.  The last CTA takes the step's mean-density rescale decision (:431-455).
// ---------------------------------------------------------------------------

// Near-wall link table: the value pulled along direction d is  A * p1 + B * p2  with
// p1, p2 populations at element offsets o1, o2 (rescaled like every load):
//   plain        f_d(src)                          A = 1,       B = 0       src = clamp(x - c_d)
//   q < 0.5      2q f_w(x) + (1 - 2q) f_w(ff)      A = 2q,      B = 1 - 2q  w = opp(d), ff = clamp(x + c_d)
//   q >= 0.5     f_w(x) / 2q + (1 - 1/2q) f_d(x)   A = 1/2q,    B = 1 - 1/2q
//   ff solid     f_w(x)                            A = 1,       B = 0
// A and B are formed exactly as the reference forms them (lbmCpuReference.ts:211-220),
// so A * p1 + B * p2 evaluates the same expression; with B = 0 it returns p1.
struct NearLink {
  uint32_t o1, o2;  // element offsets of p1, p2 (plane * direction + row * pitch + x)
  uint32_t d1, d2;  // their directions (the shifted codecs decode with w_d)
  double A, B;
};

// Shared-memory inlet tables appended after the ring: ux_in[ny], uy_in[ny].
__host__ __device__ inline size_t step_inlet_bytes(const Layout& L) { return 2 * (size_t)L.ny * sizeof(double); }

template <class S, int MODE>
__device__ __forceinline__ void wall_feq(typename std::conditional<MODE == MODE_FAST, float, double>::type (&v)[19],
                                         double r, double x, double y, double z) {
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    if constexpr (MODE == MODE_FAST) v[d] = heq32(d, (float)r, (float)x, (float)y, (float)z);
    else v[d] = feq64(d, r, x, y, z);
  }
}

// One near-wall cell: every pulled value from the link table (all loads issued up
// front), collision, the deferred inlet / outlet of its row (ix = 1 or nx-2, from its
// values before any wall condition), the wall condition when it applies, stores.
// Returns the fixed-point density added to the step's sum; sets *nan on a NaN.
template <class S, int MODE>
__device__ __forceinline__ long long near_cell(const StepArgs& a, long long t, double corr,
                                               const double* s_uxi, const double* s_uyi, int* nan) {
  using T = typename S::T;
  using Real = typename std::conditional<MODE == MODE_FAST, float, double>::type;
  using Mac = typename MacroOf<T>::type;
  const Layout L = a.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz, pitch = L.pitch;
  const long long plane = L.plane;
  const T* __restrict__ fs = static_cast<const T*>(a.fsrc);
  T* __restrict__ fd = static_cast<T*>(a.fdst);
  long long add = 0;
  const long long cell = a.near_cells[t];
  const int ix = (int)(cell % nx);
  const long long row = cell / nx;
  const int iy = (int)(row % ny), iz = (int)(row / ny);
  const long long pop_row = row * pitch;
  const int flag = a.cls[pop_row + ix] & CLS_FLAG_MASK;
  const bool wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));
  auto resc = [&](double f) -> double {
    if constexpr (MODE == MODE_MIRROR) return (double)(float)(f * corr);
    else return f * corr;
  };
  Real v[19];
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    const NearLink lk = a.links[(long long)d * a.n_near + t];
    const double p1 = S::f_of(fs[lk.o1], (int)lk.d1);
    const double p2 = S::f_of(fs[lk.o2], (int)lk.d2);
    const double val = lk.A * resc(p1) + lk.B * resc(p2);
    if constexpr (MODE == MODE_FAST) v[d] = (float)(val - (double)wf_of(d));
    else v[d] = val;
  }
  Mac mr, mx, my, mz;
  {
    Real r, ux, uy, uz;
    if constexpr (MODE == MODE_FAST) collide_f32(v, r, ux, uy, uz, (float)a.tau0, (float)a.k_smag);
    else collide_f64<MODE == MODE_MIRROR>(v, r, ux, uy, uz, a.tau0, a.k_smag);
    mr = (Mac)r; mx = (Mac)ux; my = (Mac)uy; mz = (Mac)uz;
  }
  if (ix == 1 && (a.cls[pop_row] & CLS_FLAG_MASK) != CELL_SOLID) {
    // deferred inlet (:328-352)
    const long long ic = row * nx;
    const double uxi = s_uxi[iy], uyi = s_uyi[iy];
    const double ri = MODE == MODE_FAST ? (double)(0.85f * (float)mr + 0.15f) : 0.85 * (double)mr + 0.15 * 1.0;
    T* out = fd + pop_row;
#pragma unroll
    for (int d = 0; d < 19; ++d) {
      if constexpr (MODE == MODE_FAST) out[d * plane] = S::raw_of_h(heq32(d, (float)ri, (float)uxi, (float)uyi, 0.f), d);
      else out[d * plane] = S::raw_of_f(feq64(d, ri, uxi, uyi, 0.0), d);
    }
    if (a.write_macro) {
      a.mux[ic] = (float)uxi; a.muy[ic] = (float)uyi; a.muz[ic] = 0.0f; a.mrho[ic] = (float)(Mac)ri;
    }
    add += rho_fixed((Mac)ri);
  }
  if (ix == nx - 2 && (a.cls[pop_row + nx - 1] & CLS_FLAG_MASK) != CELL_SOLID) {
    // deferred outlet (:354-371)
    const long long oc = row * nx + nx - 1;
    T* out = fd + pop_row + nx - 1;
    Mac ro;
    if constexpr (MODE == MODE_FAST) {
      const float r2 = (float)mr * 0.85f + 0.15f;
#pragma unroll
      for (int d = 0; d < 19; ++d)
        out[d * plane] = S::raw_of_h(0.75f * v[d] + 0.25f * heq32(d, r2, (float)mx, (float)my, (float)mz), d);
      ro = (Mac)r2;
    } else {
      const double r2 = (double)mr * 0.85 + 1.0 * 0.15;
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        const double stored = S::f_of(S::raw_of_f(v[d], d), d);
        out[d * plane] = S::raw_of_f(0.75 * stored + 0.25 * feq64(d, r2, (double)mx, (double)my, (double)mz), d);
      }
      ro = (Mac)r2;
    }
    if (a.write_macro) {
      a.mux[oc] = (float)mx; a.muy[oc] = (float)my; a.muz[oc] = (float)mz; a.mrho[oc] = (float)ro;
    }
    add += rho_fixed(ro);
  }
  if (wall_row && flag == CELL_FLUID) {
    if (iy == 0) {
      if (a.ground_no_slip) { mx = (Mac)0; mz = (Mac)0; }
      my = (Mac)0;
    }
    if (iy == ny - 1) my = (Mac)0;
    if (nz > 4 && (iz == 0 || iz == nz - 1)) mz = (Mac)0;
    wall_feq<S, MODE>(v, (double)mr, (double)mx, (double)my, (double)mz);
  }
  T* out = fd + pop_row + ix;
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    if constexpr (MODE == MODE_FAST) out[d * plane] = S::raw_of_h(v[d], d);
    else out[d * plane] = S::raw_of_f(v[d], d);
  }
  if (a.write_macro) {
    a.mux[cell] = (float)mx; a.muy[cell] = (float)my; a.muz[cell] = (float)mz; a.mrho[cell] = (float)mr;
  }
  if (mr == mr) add += rho_fixed(mr);
  else *nan = 1;
  return add;
}

template <class S, int MODE>
__global__ void __launch_bounds__(kStepThreads, MODE == MODE_FAST ? AEROSIM_FAST_MIN_BLOCKS : 1)
    main_kernel(const StepArgs a) {
  using T = typename S::T;
  using Real = typename std::conditional<MODE == MODE_FAST, float, double>::type;
  using Mac = typename MacroOf<T>::type;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ long long red[kConsumerWarps + 2];
  __shared__ int nan_flag;

  const Layout L = a.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz, pitch = L.pitch;
  const long long plane = L.plane;
  const int S_ = a.stages;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int shift = row_shift(nx), span = row_span(nx), RY = rows_per_item(nx);
  const int wpr = span / 32;
  const long long rows = (long long)ny * nz;
  const long long n_items = (rows + RY - 1) / RY;
  const int my_count = blockIdx.x < n_items ? (int)((n_items - 1 - blockIdx.x) / gridDim.x + 1) : 0;

  T* spop = reinterpret_cast<T*>(smem_raw + kSmemGuard);
  uint8_t* scls = smem_raw + kSmemGuard + (size_t)S_ * RY * 19 * pitch * sizeof(T);
  uint64_t* full = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(scls + (size_t)S_ * RY * pitch + kSmemGuard) + 7) & ~uintptr_t(7));
  uint64_t* empty = full + S_;
  double* s_uxi = reinterpret_cast<double*>(empty + S_);
  double* s_uyi = s_uxi + ny;
  int2* s_row = reinterpret_cast<int2*>(s_uyi + ny);  // [S_][RY] (iy, iz) of the slot's rows

  const T* __restrict__ fs = static_cast<const T*>(a.fsrc);
  T* __restrict__ fd = static_cast<T*>(a.fdst);

  if (threadIdx.x == 0) {
    for (int s = 0; s < S_; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    nan_flag = 0;
    mbar_fence_init();
  }
  // inlet velocity per iy (:334-342), evaluated once per CTA
  for (int i = threadIdx.x; i < ny; i += blockDim.x) {
    double uxi = a.u_inlet;
    if (a.ground_no_slip) uxi = a.u_inlet * a.abl[i];
    double uyi = 0.0;
    if (a.step_index < 120) uyi = 0.015 * a.u_inlet * a.sin_tab[(long long)a.step_index * ny + i];
    s_uxi[i] = uxi;
    s_uyi[i] = uyi;
  }
  __syncthreads();

  long long my_sum = 0;
  bool failed = false;

  if (warp == kHelperWarp) {
    // ---------------- helper warp: this CTA's share of the near-wall cells ----------------
    const int pslot = (a.step_index + 1) & 1;
    const double corr = a.st->apply[pslot] ? a.st->corr[pslot] : 1.0;
    int my_nan = 0;
    for (long long t = (long long)blockIdx.x * 32 + lane; t < a.n_near; t += (long long)gridDim.x * 32)
      my_sum += near_cell<S, MODE>(a, t, corr, s_uxi, s_uyi, &my_nan);
    if (__any_sync(0xffffffffu, my_nan) && lane == 0) nan_flag = 1;
  } else if (warp == kProducerWarp) {
    // ---------------- producer warp ----------------
    if (lane == 0) {
      const uint32_t row_bytes = (uint32_t)(pitch * sizeof(T));
      int issued = 0;
      for (int j = 0; j < my_count; ++j) {
        const int s = j % S_;
        if (j >= S_ && !mbar_wait(&empty[s], (uint32_t)(((j / S_) - 1) & 1), kWaitLimit)) {
          failed = true;
          break;
        }
        const long long r0 = (blockIdx.x + (long long)j * gridDim.x) * RY;
        const int nr = (int)(rows - r0 < RY ? rows - r0 : RY);
        // row coordinates for the consumers, published by the arrive below
        for (int yy = 0; yy < nr; ++yy) {
          const int r = (int)(r0 + yy);
          s_row[s * RY + yy] = make_int2(r % ny, r / ny);
        }
        mbar_arrive_expect_tx(&full[s], (uint32_t)nr * (19u * row_bytes + (uint32_t)pitch));
        for (int yy = 0; yy < nr; ++yy) {
          const int2 yz = s_row[s * RY + yy];
          const int iy = yz.x, iz = yz.y;
          const long long r = r0 + yy;
          T* dst = spop + ((size_t)s * RY + yy) * 19 * pitch;
#pragma unroll
          for (int d = 0; d < 19; ++d) {
            const long long sr =
                clampi(iy - cy_of(d), 0, ny - 1) + (long long)ny * clampi(iz - cz_of(d), 0, nz - 1);
            bulk_load(dst + (size_t)d * pitch, fs + d * plane + sr * pitch, row_bytes, &full[s]);
          }
          bulk_load(scls + ((size_t)s * RY + yy) * pitch, a.cls + r * pitch, (uint32_t)pitch, &full[s]);
        }
        issued = j + 1;
      }
      if (failed) atomicOr(&a.st->error, STEP_ERR_PIPELINE_TIMEOUT);
      // No copy may still be in flight when the CTA exits: wait (bounded) for the
      // last phase issued into every slot; completed phases return at once.
      for (int s = 0; s < S_ && s < issued; ++s) {
        const int last = s + ((issued - 1 - s) / S_) * S_;
        mbar_wait(&full[s], (uint32_t)((last / S_) & 1), kWaitLimit);
      }
    }
  } else {
    // ---------------- consumer warps ----------------
    const int pslot = (a.step_index + 1) & 1;  // pending rescale of the previous step
    const int apply = a.st->apply[pslot];
    const double corr = apply ? a.st->corr[pslot] : 1.0;
    const float corrf = (float)corr;
    const float corrf_s = corrf * F16S_INV_SCALE;
    const int ry = warp / wpr;
    const int nchunks = (nx + shift + span - 1) / span;
    int my_nan = 0;

    for (int j = 0; j < my_count; ++j) {
      const int s = j % S_;
      if (!mbar_wait(&full[s], (uint32_t)((j / S_) & 1), kWaitLimit)) {
        failed = true;
        break;
      }
      // The row-end warps carry the inlet and outlet: rotate the segment each warp
      // takes from item to item so that extra work is spread over all warps.
      const int seg = (warp % wpr + j) % wpr;
      const int xslot0 = seg * 32 + lane;
      const long long row = (blockIdx.x + (long long)j * gridDim.x) * RY + ry;
      const bool row_ok = row < rows;
      int iy = 0, iz = 0;
      if (row_ok) {
        const int2 yz = s_row[s * RY + ry];
        iy = yz.x;
        iz = yz.y;
      }
      const T* sp = spop + ((size_t)s * RY + ry) * 19 * pitch;
      const uint8_t* sc = scls + ((size_t)s * RY + ry) * pitch;
      const bool wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));
      const long long dense_row = row * nx;
      const long long pop_row = row * pitch;

      for (int c = 0; c < nchunks; ++c) {
        const int ix = xslot0 + c * span - shift;
        const bool active = row_ok && ix >= 0 && ix < nx;
        const int lx = (ix >= 0 && ix < nx) ? ix : 1;  // lanes outside the row read cell 1
        const uint8_t cl = sc[lx];
        const int flag = cl & CLS_FLAG_MASK;
        const bool solid = !active || flag == CELL_SOLID;
        const bool xface = (ix == 0 || ix == nx - 1);
        const bool near = (cl & CLS_NEAR) != 0;
        Real v[19];
        // ---- pull-stream (lbmCpuReference.ts:189-231) from the staged rows.  Every
        // lane loads and collides; x faces, near-wall cells and solids overwrite or
        // discard the result. ----
#pragma unroll
        for (int d = 0; d < 19; ++d) {
          const T raw = sp[d * pitch + lx - cx_of(d)];
          if constexpr (MODE == MODE_FAST) v[d] = S::h_scaled(raw, d, corrf, corrf_s);
          else if constexpr (MODE == MODE_MIRROR) v[d] = (double)(float)(S::f_of(raw, d) * corr);
          else v[d] = S::f_of(raw, d) * corr;
        }
        if (c == nchunks - 1) {  // every value of this slot is in registers: release it
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[s]);
        }
        Mac mr, mx, my, mz;
        {
          Real r, ux, uy, uz;
          if constexpr (MODE == MODE_FAST) collide_f32(v, r, ux, uy, uz, (float)a.tau0, (float)a.k_smag);
          else collide_f64<MODE == MODE_MIRROR>(v, r, ux, uy, uz, a.tau0, a.k_smag);
          mr = (Mac)r; mx = (Mac)ux; my = (Mac)uy; mz = (Mac)uz;
        }
        bool done = active && !solid && !xface && !near;  // this lane stores its cell

        // ---- inlet / outlet (:323-373), inside the warp that holds the row end ----
        const int cell_lo = c * span + seg * 32 - shift;  // cell of lane 0
        if (row_ok && cell_lo <= 0 && 1 <= cell_lo + 31) {
          const int src = 1 - cell_lo;
          // rho at ix = 1 is 1 for a solid (:177); a near-wall ix = 1 defers the inlet
          const double rho1 = __shfl_sync(0xffffffffu, solid ? 1.0 : (double)mr, src);
          const int defer = __shfl_sync(0xffffffffu, (int)(near && !solid), src);
          if (ix == 0 && !solid && !defer) {
            const double uxi = s_uxi[iy], uyi = s_uyi[iy];
            if constexpr (MODE == MODE_FAST) {
              const float ri = 0.85f * (float)rho1 + 0.15f;
#pragma unroll
              for (int d = 0; d < 19; ++d) v[d] = heq32(d, ri, (float)uxi, (float)uyi, 0.f);
              mr = (Mac)ri;
            } else {
              const double ri = 0.85 * rho1 + 0.15 * 1.0;
#pragma unroll
              for (int d = 0; d < 19; ++d) v[d] = feq64(d, ri, uxi, uyi, 0.0);
              mr = (Mac)ri;
            }
            mx = (Mac)uxi; my = (Mac)uyi; mz = (Mac)0;
            done = true;
          }
        }
        if (row_ok && cell_lo <= nx - 2 && nx - 1 <= cell_lo + 31) {
          const int src = nx - 2 - cell_lo;
          const int defer = __shfl_sync(0xffffffffu, (int)(near && !solid), src);
          if (!defer) {
            // the outlet reads fDst at nx-2 before the walls (:363): the stored value,
            // or for a solid cell whatever fDst holds there (never written)
            Real send[19];
            const bool stale = (ix == nx - 2) && solid;
#pragma unroll
            for (int d = 0; d < 19; ++d) {
              if (stale) {
                const double f = S::f_of(fd[d * plane + pop_row + ix], d);
                send[d] = MODE == MODE_FAST ? (Real)(f - (double)wf_of(d)) : (Real)f;
              } else if constexpr (MODE == MODE_FAST) {
                send[d] = v[d];
              } else {
                send[d] = S::f_of(S::raw_of_f(v[d], d), d);
              }
            }
            const double m0 = __shfl_sync(0xffffffffu, stale ? 1.0 : (double)mr, src);
            const double m1 = __shfl_sync(0xffffffffu, stale ? 0.0 : (double)mx, src);
            const double m2 = __shfl_sync(0xffffffffu, stale ? 0.0 : (double)my, src);
            const double m3 = __shfl_sync(0xffffffffu, stale ? 0.0 : (double)mz, src);
#pragma unroll
            for (int d = 0; d < 19; ++d) send[d] = __shfl_sync(0xffffffffu, send[d], src);
            if (ix == nx - 1 && !solid) {
              if constexpr (MODE == MODE_FAST) {
                const float ro = (float)m0 * 0.85f + 0.15f;
#pragma unroll
                for (int d = 0; d < 19; ++d)
                  v[d] = 0.75f * send[d] + 0.25f * heq32(d, ro, (float)m1, (float)m2, (float)m3);
                mr = (Mac)ro;
              } else {
                const double ro = m0 * 0.85 + 1.0 * 0.15;
#pragma unroll
                for (int d = 0; d < 19; ++d) v[d] = 0.75 * send[d] + 0.25 * feq64(d, ro, m1, m2, m3);
                mr = (Mac)ro;
              }
              mx = (Mac)m1; my = (Mac)m2; mz = (Mac)m3;
              done = true;
            }
          }
        }
        // ---- wall conditions (:375-429): own moments, floor, ceiling, then sides ----
        if (wall_row) {
          if (done && !xface && flag == CELL_FLUID) {
            if (iy == 0) {
              if (a.ground_no_slip) { mx = (Mac)0; mz = (Mac)0; }
              my = (Mac)0;
            }
            if (iy == ny - 1) my = (Mac)0;
            if (nz > 4 && (iz == 0 || iz == nz - 1)) mz = (Mac)0;
            wall_feq<S, MODE>(v, (double)mr, (double)mx, (double)my, (double)mz);
          }
        }
        if (done) {
          T* out = fd + pop_row + ix;
#pragma unroll
          for (int d = 0; d < 19; ++d) {
            if constexpr (MODE == MODE_FAST) out[d * plane] = S::raw_of_h(v[d], d);
            else out[d * plane] = S::raw_of_f(v[d], d);
          }
          if (mr == mr) my_sum += rho_fixed(mr);
          else my_nan = 1;
        }
        if (a.write_macro) {
          const long long di = dense_row + ix;
          if (active && solid) {  // solid macro (:173-179)
            a.mux[di] = 0.0f; a.muy[di] = 0.0f; a.muz[di] = 0.0f; a.mrho[di] = 1.0f;
          } else if (done) {
            a.mux[di] = (float)mx; a.muy[di] = (float)my; a.muz[di] = (float)mz; a.mrho[di] = (float)mr;
          }
        }
      }
    }
    if (__any_sync(0xffffffffu, my_nan) && lane == 0) nan_flag = 1;
    if (failed && lane == 0) atomicOr(&a.st->error, STEP_ERR_PIPELINE_TIMEOUT);
  }

#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_sum += __shfl_down_sync(0xffffffffu, my_sum, o);
  if (lane == 0) red[warp] = my_sum;
  __syncthreads();
  const int slot = a.step_index & 1;
  __shared__ int is_last;
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w < kConsumerWarps + 2; ++w) s += red[w];
    if (nan_flag) a.st->nan_seen = 1;
    if (s) atomicAdd(&a.st->rho_sum[slot], (unsigned long long)s);
    __threadfence();
    const unsigned int tk = atomicAdd(&a.st->ticket[slot], 1u);
    is_last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  // ---- mean-density rescale (:431-455): the last CTA takes the decision ----
  if (is_last && threadIdx.x == 0) {
    __threadfence();
    const long long total = (long long)atomicAdd(&a.st->rho_sum[slot], 0ull);
    int ap = 0;
    double cr = 1.0;
    if (a.fluid_count > 0) {
      const double mean = rho_unfixed(total, Mac(0)) / (double)a.fluid_count;
      cr = 1.0 / mean;
      ap = fabs(mean - 1.0) > 1e-4 ? 1 : 0;
    }
    a.st->corr[slot] = cr;
    a.st->apply[slot] = ap;
    if (ap) {
      a.st->cumulative_rescale *= cr;
      a.st->rescale_count += 1;
    }
    // accumulators of the next step start from zero
    a.st->rho_sum[slot ^ 1] = 0ull;
    a.st->ticket[slot ^ 1] = 0u;
  }
}

// ---------------------------------------------------------------------------
// Momentum exchange, forceIntegrator.ts:159-216, FP64 accumulation.
// One thread per boundary cell; per-cell sums in the reference's link order, then a
// deterministic tree across cells (warp shuffle -> CTA -> last CTA in block order).
// ---------------------------------------------------------------------------
template <class S, int MODE>
__global__ void __launch_bounds__(256) forces_kernel(const ForceArgs a) {
  using T = typename S::T;
  __shared__ double red[8][8];
  __shared__ bool is_last;
  const T* __restrict__ f = static_cast<const T*>(a.f);
  const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int apply = a.prev_slot >= 0 ? a.st->apply[a.prev_slot] : 0;
  const double corr = apply ? a.st->corr[a.prev_slot] : 1.0;
  auto pop = [&](int d, long long i) -> double {
    const double v = S::f_of(f[a.L.at(d, i)], d);
    if constexpr (MODE == MODE_MIRROR) return (double)(float)(v * corr);
    else return v * corr;
  };
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (b < a.B) {
    const long long ci = a.bcells[b];
    const int nx = a.L.nx, ny = a.L.ny, nz = a.L.nz;
    const int ix = (int)(ci % nx);
    const long long rem = (ci - ix) / nx;
    const int iy = (int)(rem % ny);
    const int iz = (int)((rem - iy) / ny);
    double cfx = 0.0, cfy = 0.0, cfz = 0.0;
    double cut = 0.0;
#pragma unroll
    for (int d = 1; d < 19; ++d) {
      const double qv = (double)a.q[b * 18 + (d - 1)];
      if (qv > 0.0) {
        const int od = opp_of(d);
        const double fo = pop(d, ci);
        const int ax = clampi(ix + cx_of(od), 0, nx - 1);
        const int ay = clampi(iy + cy_of(od), 0, ny - 1);
        const int az = clampi(iz + cz_of(od), 0, nz - 1);
        const long long ff = ax + (long long)nx * (ay + (long long)ny * az);
        double fi = fo;
        if ((a.cls[a.L.cls_at(ff)] & CLS_FLAG_MASK) != 1) {
          if (qv < 0.5) {
            const double fon = pop(d, ff);
            fi = 2.0 * qv * fo + (1.0 - 2.0 * qv) * fon;
          } else {
            const double fic = pop(od, ci);
            const double inv2q = 1.0 / (2.0 * qv);
            fi = inv2q * fo + (1.0 - inv2q) * fic;
          }
        }
        const double mom = fo + fi - 2.0 * w32_of(d);
        cfx += (double)cx_of(d) * mom;
        cfy += (double)cy_of(d) * mom;
        cfz += (double)cz_of(d) * mom;
        if (d <= 6) cut += 1.0;
      }
    }
    const double rx = (ix + 0.5) - 0.5 * nx;
    const double ry = (iy + 0.5) - 0.5 * ny;
    const double rz = (iz + 0.5) - 0.5 * nz;
    acc[0] = cfx; acc[1] = cfy; acc[2] = cfz;
    acc[3] = ry * cfz - rz * cfy;
    acc[4] = rz * cfx - rx * cfz;
    acc[5] = rx * cfy - ry * cfx;
    acc[6] = cut;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 7; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
    if (lane == 0) red[warp][k] = acc[k];
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    a.partials[(long long)blockIdx.x * 8 + threadIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int t = atomicAdd(a.ticket, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    if (threadIdx.x < 7) {
      double s = 0.0;
      for (unsigned int blk = 0; blk < gridDim.x; ++blk) {
        s += *(volatile double*)&a.partials[(long long)blk * 8 + threadIdx.x];
      }
      a.out[threadIdx.x] = s;
    }
    if (threadIdx.x == 0) {
      a.out[7] = (double)gridDim.x;
      *a.ticket = 0u;
    }
  }
}

}  // namespace aerosim
