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
#include "sgs_mlp.cuh"
#include "sgs_umma.cuh"
#include "lbm_pair.cuh"

namespace aerosim {

enum { MODE_FAST = 0, MODE_MIRROR = 1, MODE_F64 = 2 };

// Resident CTAs per SM the step kernel is register-budgeted for.  FP32 storage gains
// from a third CTA (more warps in flight per SM: 131 -> 121 us per step measured at
// 256x128x128, with some spilling at 64 registers); the 16-bit storage kernels issue
// more instructions per cell and lose more to spills at that budget, so they keep two.
// With the learned closure the tensor-core MLP needs registers: two CTAs.
// MLP: 0 Smagorinsky, 1 the closure as warp-level mma.sync tiles, 2 the closure as
// 128-cell tcgen05 tiles (groups of four consumer warps, TMEM accumulators).
enum { MLP_NONE = 0, MLP_WARP = 1, MLP_TCGEN05 = 2 };
// Two cells per thread (CPT = 2) hold twice the values: two CTAs for every storage.
template <class S, int MODE, int MLP = MLP_NONE, int CPT = 1>
constexpr int step_min_blocks() {
  return MODE != MODE_FAST ? 1 : ((MLP || CPT == 2) ? 2 : (sizeof(typename S::T) == 4 ? 3 : 2));
}
// Row groups per work item of the step kernel: a work item holds item_groups x
// rows_per_item(nx) x-rows and every consumer warp takes its segment of each group, so
// the slot wait and release and the row setup are paid once per item.  The 16-bit
// storage kernels take items of about 1024 cells (4 rows of 256 cells: 102.4 -> 85.1 us
// per step at 256x128x128; the group count is StepArgs::item_groups); FP32 keeps one
// group, because its larger ring slots would cost a resident CTA per SM (118.6 -> 127.6
// us with 2 groups).
template <class S, int MODE, int MLP = MLP_NONE>
constexpr bool step_item_grouped() {
  return MODE == MODE_FAST && !MLP && sizeof(typename S::T) == 2;
}

struct NearLink;
struct NearLinkF;

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
  const NearLinkF* links_f;   // [19][n_near] the same, compact, for the FP32-arithmetic kernels
  int stages;             // depth of the shared-memory ring
  int step_index;
  int write_macro;
  int ground_no_slip;
  double u_inlet, tau0, k_smag;  // k_smag = 18 * SQRT2 * Cs^2
  // learned SGS closure (null: Smagorinsky): packed BF16 weight fragments and biases
  // (sgs_mlp.cuh) and the molecular viscosity nu_0 its output is scaled by
  const uint32_t* mlp_frag;
  const float* mlp_bias;
  const uint4* mlp_umma;  // weight image of the tcgen05 path (sgs_umma.cuh), or null
  float mlp_nu0;
  int item_groups;        // row groups per work item (16-bit storage kernels; 1 elsewhere)
  int wait_limit;         // polls of a ring wait before the step gives up (kWaitLimit;
                          //   0 gives up at once: the failure path's test)
  int cells_per_thread;   // consumer cells per thread: 1, or 2 (pair kernels, even nx)
  int dynamic_items;      // 1: CTAs take work items from a device counter (StepState::next_item)
                          //   instead of the static round-robin deal
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
  int* err_out;           // receives the steps' error code, or null
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

// Approximate reciprocal and square root (one MUFU operation each); the FP32 path is
// held to a tolerance against the oracle, not to its rounding.
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// The same regularized collision as collide_f32 written as one second-order Hermite
// expansion, which needs fewer operations per direction:
//   f*_i = w_i [rho + 3 c_i.j + 4.5 Q_i : X],   X = rho u u + (1 - omega) Pi^neq,
// and, with Pi^neq = S - (rho - 1)/3 I - rho u u (S = sum cc h),
//   X = (S - (rho - 1)/3 I) - omega Pi^neq.
// With B = rho - 1 - 1.5 tr X the deviation is h_i = w_i (B + 4.5 c_i c_i : X + 3 c_i.j).
// rho and u are the clamped, Mach-limited values the reference forms its equilibrium
// from (lbmCpuReference.ts:233-262), j = rho u.  The results are written back into
// h[] already in the storage domain of S (kOutScale * h + kOutW * w), the storage's
// scale and rest weight folded into the per-direction constants.
// With MLP the eddy viscosity comes from the learned closure (sgs_mlp.cuh) evaluated
// by the whole warp on the tensor cores: tau = 3 nu_0 (1 + nu_t / nu_0) + 1/2, with the
// Smagorinsky tau as the fallback when the network returns a non-finite value.
struct MlpRefs {
  const uint32_t* frag;  // shared memory
  const float* bias;
  uint32_t* stage;       // the warp's 32 x 8 BF16 staging block
  float nu0;
  float wall_dist;       // this lane's cell
  int lane;
  UmmaGroup* grp;        // the tcgen05 path: this warp's group state
};

template <class S, int MLP = MLP_NONE>
__device__ __forceinline__ void collide_fast(float (&h)[19], float& r, float& ux, float& uy, float& uz,
                                             float tau0, float k_smag, float2 dec, const MlpRefs* m = nullptr) {
  static_assert(S::kRawMoments, "the FP32 collision runs on stored deviations");
  constexpr float OS = S::kOutScale, OW = S::kOutW;
  constexpr float w0 = 1.0f / 3.0f, w1 = 1.0f / 18.0f, w2 = 1.0f / 36.0f;
  float s[9], t[9];
#pragma unroll
  for (int p = 0; p < 9; ++p) {
    s[p] = h[2 * p + 1] + h[2 * p + 2];
    t[p] = h[2 * p + 1] - h[2 * p + 2];
  }
  float dr = h[0] + ((s[0] + s[1]) + (s[2] + s[3]) + ((s[4] + s[5]) + (s[6] + s[7])) + s[8]);
  float jx = (t[0] + t[3]) + (t[4] + t[5]) + t[6];
  float jy = (t[1] + t[3]) - t[4] + (t[7] + t[8]);
  float jz = (t[2] + t[5]) - t[6] + (t[7] - t[8]);
  float sxx = (s[0] + s[3]) + (s[4] + s[5]) + s[6];
  float syy = (s[1] + s[3]) + (s[4] + s[7]) + s[8];
  float szz = (s[2] + s[5]) + (s[6] + s[7]) + s[8];
  float sxy = s[3] - s[4], sxz = s[5] - s[6], syz = s[7] - s[8];
  {
    // h holds raw stored values, h_i = dec.x raw_i + dec.y w_i (dec = storage scale x
    // pending rescale, rescale - 1): with sum w = 1, sum w c = 0, sum w c_a c_a = 1/3
    // and sum w c_a c_b = 0 the ten moments take the decode in ten operations
    const float cw3 = dec.y * (1.0f / 3.0f);
    dr = fmaf(dr, dec.x, dec.y);
    jx *= dec.x; jy *= dec.x; jz *= dec.x;
    sxx = fmaf(sxx, dec.x, cw3); syy = fmaf(syy, dec.x, cw3); szz = fmaf(szz, dec.x, cw3);
    sxy *= dec.x; sxz *= dec.x; syz *= dec.x;
  }

  r = fmaxf(0.5f, fminf(1.8f, 1.0f + dr));
  if (dr != dr) r = dr;  // keep NaN visible like Math.min / Math.max
  const float ir = rcp_approx(r);
  ux = jx * ir; uy = jy * ir; uz = jz * ir;
  const float uSq0 = ux * ux + uy * uy + uz * uz;
  if (uSq0 > 0.0484f) {  // Mach limiter |u| <= 0.22
    const float sc = 0.22f * rsqrtf(uSq0);
    ux *= sc; uy *= sc; uz *= sc;
  }
  const float drc = r - 1.0f;
  const float d3 = drc * (1.0f / 3.0f);
  const float jcx = r * ux, jcy = r * uy, jcz = r * uz;
  const float dxx = sxx - d3, dyy = syy - d3, dzz = szz - d3;
  const float pxx = fmaf(-jcx, ux, dxx), pyy = fmaf(-jcy, uy, dyy), pzz = fmaf(-jcz, uz, dzz);
  const float pxy = fmaf(-jcx, uy, sxy), pxz = fmaf(-jcx, uz, sxz), pyz = fmaf(-jcy, uz, syz);
  const float off = fmaf(pxy, pxy, fmaf(pxz, pxz, pyz * pyz));
  const float pn = sqrt_approx(fmaf(pxx, pxx, fmaf(pyy, pyy, fmaf(pzz, pzz, 2.0f * off))));
  float tau = 0.5f * (tau0 + sqrt_approx(fmaf(tau0, tau0, k_smag * pn * ir)));
  if constexpr (MLP != MLP_NONE) {
    float x[kMlpIn];
    mlp_features(pxx, pyy, pzz, pxy, pxz, pyz, r, tau, m->wall_dist, x);
    float ratio;
    if constexpr (MLP == MLP_TCGEN05) ratio = mlp_nut_umma(x, *m->grp, m->bias);
    else ratio = mlp_nut_warp(x, m->frag, m->bias, m->stage, m->lane);
    const float tm = fmaf(3.0f * m->nu0, 1.0f + ratio, 0.5f);
    if (tm == tm && tm < 1.0e30f) tau = tm;
  }
  const float om = rcp_approx(fmaxf(0.5015f, fminf(1.95f, tau)));
  const float xxx = fmaf(-om, pxx, dxx), xyy = fmaf(-om, pyy, dyy), xzz = fmaf(-om, pzz, dzz);
  const float xxy = fmaf(-om, pxy, sxy), xxz = fmaf(-om, pxz, sxz), xyz = fmaf(-om, pyz, syz);
  const float B = fmaf(-1.5f, (xxx + xyy) + xzz, drc);
  const float b = OW == 0.0f ? OS * B : fmaf(OS, B, OW);
  h[0] = w0 * b;
  // faces +-a: w1 (B + 4.5 X_aa +- 3 j_a)
  const float b1 = w1 * b;
  constexpr float kf = OS * 4.5f * w1, of = OS * 3.0f * w1;
  {
    const float E = fmaf(kf, xxx, b1), O = of * jcx;
    h[1] = E + O; h[2] = E - O;
  }
  {
    const float E = fmaf(kf, xyy, b1), O = of * jcy;
    h[3] = E + O; h[4] = E - O;
  }
  {
    const float E = fmaf(kf, xzz, b1), O = of * jcz;
    h[5] = E + O; h[6] = E - O;
  }
  // edges +-(a +- b): w2 (B + 4.5 (X_aa + X_bb +- 2 X_ab) + 3 (j_a +- j_b))
  const float b2 = w2 * b;
  constexpr float ke = OS * 4.5f * w2, ke2 = OS * 9.0f * w2, oe = OS * 3.0f * w2;
  const float qx = oe * jcx, qy = oe * jcy, qz = oe * jcz;
  {
    const float base = fmaf(ke, xxx + xyy, b2);
    const float Ep = fmaf(ke2, xxy, base), Em = fmaf(-ke2, xxy, base);
    const float Op = qx + qy, Om = qx - qy;
    h[7] = Ep + Op; h[8] = Ep - Op; h[9] = Em + Om; h[10] = Em - Om;
  }
  {
    const float base = fmaf(ke, xxx + xzz, b2);
    const float Ep = fmaf(ke2, xxz, base), Em = fmaf(-ke2, xxz, base);
    const float Op = qx + qz, Om = qx - qz;
    h[11] = Ep + Op; h[12] = Ep - Op; h[13] = Em + Om; h[14] = Em - Om;
  }
  {
    const float base = fmaf(ke, xyy + xzz, b2);
    const float Ep = fmaf(ke2, xyz, base), Em = fmaf(-ke2, xyz, base);
    const float Op = qy + qz, Om = qy - qz;
    h[15] = Ep + Op; h[16] = Ep - Op; h[17] = Em + Om; h[18] = Em - Om;
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

// Thread -> cell mapping of a row.  One cell per thread (cpt = 1): cell ix = slot - shift
// with slot = lane + 32 * warp + tx_span * chunk; shift = 1 when nx = 1 (mod 32) keeps
// the cell pairs (0, 1) and (nx-2, nx-1) inside one warp, so the inlet and outlet
// exchange stays warp-local.  Two cells per thread (cpt = 2, rows of an even cell count):
// thread slot holds cells 2 slot and 2 slot + 1, so each row end sits in one thread with
// the neighbour its boundary condition reads, and no shift is needed.
__host__ __device__ inline int row_shift(int nx, int cpt = 1) { return (cpt == 1 && nx % 32 == 1) ? 1 : 0; }
__host__ __device__ inline int row_span(int nx, int cpt = 1) {  // threads along x (multiple of 32, <= 256)
  const int t = ((nx + row_shift(nx, cpt) + cpt - 1) / cpt + 31) / 32 * 32;
  return t > kConsumerWarps * 32 ? kConsumerWarps * 32 : t;
}
__host__ __device__ inline int rows_per_item(int nx, int cpt = 1) {
  return (kConsumerWarps * 32) / row_span(nx, cpt);
}
// Row groups per work item for about 1024 cells per item (1..4).
__host__ __device__ inline int item_groups_for(int nx, int cpt = 1) {
  const int span = row_span(nx, cpt) * cpt, chunks = (nx + row_shift(nx, cpt) + span - 1) / span;
  const int cells = rows_per_item(nx, cpt) * chunks * span;
  return cells >= 1024 ? 1 : (1024 / cells > 4 ? 4 : 1024 / cells);
}

// Dynamic shared memory of the step kernel, in order: a guard; the ring of `stages`
// slots, each holding RY row blocks (19 slot rows of `pitch` elements, pulled from
// their source rows; groups x RY rows with item row groups); the class bytes of the
// slots' destination rows; a guard; a full and an empty mbarrier per slot; the inlet
// tables ux_in[ny], uy_in[ny]; the row coordinates [stages][groups x RY]; per consumer warp an outlet scratch row of 20
// floats; the per-lane direction table (c_x, c_y, c_z, w; slot) of the row-end cells.
__host__ __device__ inline size_t step_stage_bytes(const Layout& L, size_t elem, int groups = 1, int cpt = 1) {
  return (size_t)rows_per_item(L.nx, cpt) * groups * (19 * (size_t)L.pitch * elem + (size_t)L.pitch);
}
constexpr size_t kSmemGuard = 64;
// With the learned closure (mlp = MLP_WARP or MLP_TCGEN05): its weight fragments, biases
// and per-warp staging blocks; with MLP_TCGEN05 also the tcgen05 operands (sgs_umma.cuh).
__host__ __device__ inline size_t step_smem_bytes(const Layout& L, int stages, size_t elem, int mlp = 0,
                                                   int groups = 1, int cpt = 1) {
  return kSmemGuard + (size_t)stages * step_stage_bytes(L, elem, groups, cpt) + kSmemGuard + 16 +
         16 * (size_t)stages + 2 * (size_t)L.ny * sizeof(double) +
         (size_t)stages * rows_per_item(L.nx, cpt) * groups * sizeof(int2) +
         kConsumerWarps * 24 * sizeof(float) + 16 + 19 * sizeof(float4) + 19 * sizeof(int) +
         (mlp ? (kMlpFragWords * 32 + kMlpBias + 3 + kConsumerWarps * 128) * 4 : 0) +
         (mlp == 2 ? kStepUmmaBytes : 0);
}

// ---------------------------------------------------------------------------
// One launch per time step, main_kernel: a persistent CTA of 8 consumer warps, a
// producer warp and a helper warp.  The producer streams row blocks into the shared
// ring with bulk copies, one copy per group of directions that share a source row;
// the consumers walk the rows: pull, collide, wall conditions (:375-429), inlet and
// outlet (:323-373), store.  Meanwhile the helper warp takes the CTA's share of the
// near-wall cells (Bouzidi, :196-221; one lane per cell from a link table built with
// the voxel grid).  A near-wall cell at ix = 1 or nx-2 carries its row's inlet or
// outlet, which need its post-collision values.  With 16-bit storage and two cells per
// thread the helper warp also takes, from every ring slot, the two pairs of each row
// that hold its ends (end_pair; the consumers leave them out), and a batch of near-wall
// cells after each slot.  The last CTA takes the step's mean-density rescale decision
// (:431-455).
//
// P is the row pitch when it is a compile-time constant (0: L.pitch at run time):
// with a constant pitch every shared-memory load and global store of a cell is an
// immediate offset from one base address.
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
  uint32_t o1, o2;  // element offsets of p1, p2 (Layout::at)
  uint32_t d1, d2;  // their directions (the shifted codecs decode with w_d)
  double A, B;
};
// The compact table of the FP32-arithmetic kernels (16 bytes a link instead of 32): the
// two populations of a link belong to directions d or opp(d), which share the weight
// w_d, and A + B = 1 in every case, so the pulled deviation is
//   f - w_d = c (A h1 + B h2) + (c - 1) w_d,   h = stored deviation, c = pending rescale.
struct NearLinkF {
  uint32_t o1, o2;
  float A, B;
};

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
// fsrc / fdst are the step's population buffers, inlet_u(iy) the inlet velocity
// (double2) of row iy.  Returns the fixed-point density added to the step's sum; sets
// *nan on a NaN.
template <class S, int MODE, int P, class InletFn>
__device__ __forceinline__ long long near_cell(const StepArgs& a, const void* fsrc, void* fdst, int write_macro,
                                               long long t, double corr, InletFn inlet_u, int* nan) {
  using T = typename S::T;
  using Real = typename std::conditional<MODE == MODE_FAST, float, double>::type;
  using Mac = typename MacroOf<T>::type;
  const Layout& L = a.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int pitch = P ? P : L.pitch;
  const T* __restrict__ fs = static_cast<const T*>(fsrc);
  T* __restrict__ fd = static_cast<T*>(fdst);
  long long add = 0;
  const long long cell = a.near_cells[t];
  const int ix = (int)(cell % nx);
  const long long row = cell / nx;
  const int iy = (int)(row % ny), iz = (int)(row / ny);
  const long long cls_row = row * pitch;
  T* const blk = fd + row * 19 * pitch;  // the row block of the destination row
  const int flag = a.cls[cls_row + ix] & CLS_FLAG_MASK;
  const bool wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));
  auto resc = [&](double f) -> double {
    if constexpr (MODE == MODE_MIRROR) return (double)(float)(f * corr);
    else return f * corr;
  };
  Real v[19];
  if constexpr (MODE == MODE_FAST) {
    const float c = (float)corr, cw = c - 1.0f;
#pragma unroll
    for (int d = 0; d < 19; ++d) {
      const NearLinkF lk = a.links_f[(long long)d * a.n_near + t];
      const float h1 = S::h_of(fs[lk.o1], d), h2 = S::h_of(fs[lk.o2], d);
      v[d] = fmaf(c, fmaf(lk.A, h1, lk.B * h2), cw * wf_of(d));
    }
  } else {
#pragma unroll
    for (int d = 0; d < 19; ++d) {
      const NearLink lk = a.links[(long long)d * a.n_near + t];
      const double p1 = S::f_of(fs[lk.o1], (int)lk.d1);
      const double p2 = S::f_of(fs[lk.o2], (int)lk.d2);
      v[d] = lk.A * resc(p1) + lk.B * resc(p2);
    }
  }
  Mac mr, mx, my, mz;
  {
    Real r, ux, uy, uz;
    if constexpr (MODE == MODE_FAST) collide_f32(v, r, ux, uy, uz, (float)a.tau0, (float)a.k_smag);
    else collide_f64<MODE == MODE_MIRROR>(v, r, ux, uy, uz, a.tau0, a.k_smag);
    mr = (Mac)r; mx = (Mac)ux; my = (Mac)uy; mz = (Mac)uz;
  }
  if (ix == 1 && (a.cls[cls_row] & CLS_FLAG_MASK) != CELL_SOLID) {
    // deferred inlet (:328-352)
    const long long ic = row * nx;
    const double2 ui = inlet_u(iy);
    const double uxi = ui.x, uyi = ui.y;
    const double ri = MODE == MODE_FAST ? (double)(0.85f * (float)mr + 0.15f) : 0.85 * (double)mr + 0.15 * 1.0;
    if constexpr (S::kCompensate) {
      float q[19];
#pragma unroll
      for (int d = 0; d < 19; ++d) q[d] = S::kOutScale * heq32(d, (float)ri, (float)uxi, (float)uyi, 0.f);
      compensate_cell<S>(q);
#pragma unroll
      for (int d = 0; d < 19; ++d) blk[slot_of(d) * pitch] = S::store(q[d]);
    } else {
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        if constexpr (MODE == MODE_FAST)
          blk[slot_of(d) * pitch] = S::raw_of_h(heq32(d, (float)ri, (float)uxi, (float)uyi, 0.f), d);
        else blk[slot_of(d) * pitch] = S::raw_of_f(feq64(d, ri, uxi, uyi, 0.0), d);
      }
    }
    if (write_macro) {
      a.mux[ic] = (float)uxi; a.muy[ic] = (float)uyi; a.muz[ic] = 0.0f; a.mrho[ic] = (float)(Mac)ri;
    }
    add += rho_fixed((Mac)ri);
  }
  if (ix == nx - 2 && (a.cls[cls_row + nx - 1] & CLS_FLAG_MASK) != CELL_SOLID) {
    // deferred outlet (:354-371)
    const long long oc = row * nx + nx - 1;
    T* out = blk + nx - 1;
    Mac ro;
    if constexpr (MODE == MODE_FAST) {
      const float r2 = (float)mr * 0.85f + 0.15f;
      if constexpr (S::kCompensate) {
        float q[19];
#pragma unroll
        for (int d = 0; d < 19; ++d)
          q[d] = S::kOutScale * (0.75f * v[d] + 0.25f * heq32(d, r2, (float)mx, (float)my, (float)mz));
        compensate_cell<S>(q);
#pragma unroll
        for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch] = S::store(q[d]);
      } else {
#pragma unroll
        for (int d = 0; d < 19; ++d)
          out[slot_of(d) * pitch] =
              S::raw_of_h(0.75f * v[d] + 0.25f * heq32(d, r2, (float)mx, (float)my, (float)mz), d);
      }
      ro = (Mac)r2;
    } else {
      const double r2 = (double)mr * 0.85 + 1.0 * 0.15;
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        const double stored = S::f_of(S::raw_of_f(v[d], d), d);
        out[slot_of(d) * pitch] =
            S::raw_of_f(0.75 * stored + 0.25 * feq64(d, r2, (double)mx, (double)my, (double)mz), d);
      }
      ro = (Mac)r2;
    }
    if (write_macro) {
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
  T* out = blk + ix;
  if constexpr (S::kCompensate) {
    float q[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) q[d] = S::kOutScale * v[d];
    compensate_cell<S>(q);
#pragma unroll
    for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch] = S::store(q[d]);
  } else {
#pragma unroll
    for (int d = 0; d < 19; ++d) {
      if constexpr (MODE == MODE_FAST) out[slot_of(d) * pitch] = S::raw_of_h(v[d], d);
      else out[slot_of(d) * pitch] = S::raw_of_f(v[d], d);
    }
  }
  if (write_macro) {
    a.mux[cell] = (float)mx; a.muy[cell] = (float)my; a.muz[cell] = (float)mz; a.mrho[cell] = (float)mr;
  }
  if (mr == mr) add += rho_fixed(mr);
  else *nan = 1;
  return add;
}

// Per-lane state of a consumer cell handed to the general path.
struct CellCtx {
  long long row;     // x-row of the warp's segment
  int ix;            // cell index along x (may lie outside the row for idle lanes)
  int iy, iz;
  int cell_lo;       // cell of lane 0
  int flag;
  bool active, near;
};

// Consumer path of the double modes, with the reference's per-cell logic on the
// pulled values v: collision, inlet / outlet (:323-373) inside the warp that holds the
// row end, wall conditions (:375-429), stores.  Returns the fixed-point density added
// to the step's sum.
template <class S, int MODE, int P>
__device__ __forceinline__ long long general_cells(const StepArgs& a, double (&v)[19], const CellCtx cc,
                                                   const double* s_uxi, const double* s_uyi, int* my_nan) {
  using T = typename S::T;
  using Mac = typename MacroOf<T>::type;
  const Layout& L = a.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int pitch = P ? P : L.pitch;
  T* __restrict__ fd = static_cast<T*>(a.fdst);
  const int ix = cc.ix, iy = cc.iy, iz = cc.iz, flag = cc.flag, cell_lo = cc.cell_lo;
  const bool active = cc.active, near = cc.near;
  const bool solid = !active || flag == CELL_SOLID;
  const bool xface = (ix == 0 || ix == nx - 1);
  const bool wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));
  const bool row_ok = cc.row < (long long)ny * nz;
  const bool has_lo = row_ok && cell_lo <= 0 && 1 <= cell_lo + 31;
  const bool has_hi = row_ok && cell_lo <= nx - 2 && nx - 1 <= cell_lo + 31;
  T* const blk = fd + cc.row * 19 * pitch;
  long long add = 0;

  Mac mr, mx, my, mz;
  {
    double r, ux, uy, uz;
    collide_f64<MODE == MODE_MIRROR>(v, r, ux, uy, uz, a.tau0, a.k_smag);
    mr = (Mac)r; mx = (Mac)ux; my = (Mac)uy; mz = (Mac)uz;
  }
  bool done = active && !solid && !xface && !near;  // this lane stores its cell

  // ---- inlet / outlet (:323-373), inside the warp that holds the row end ----
  if (has_lo) {
    const int src = 1 - cell_lo;
    // rho at ix = 1 is 1 for a solid (:177); a near-wall ix = 1 defers the inlet
    const double rho1 = __shfl_sync(0xffffffffu, solid ? 1.0 : (double)mr, src);
    const int defer = __shfl_sync(0xffffffffu, (int)(near && !solid), src);
    if (ix == 0 && !solid && !defer) {
      const double uxi = s_uxi[iy], uyi = s_uyi[iy];
      const double ri = 0.85 * rho1 + 0.15 * 1.0;
#pragma unroll
      for (int d = 0; d < 19; ++d) v[d] = feq64(d, ri, uxi, uyi, 0.0);
      mr = (Mac)ri;
      mx = (Mac)uxi; my = (Mac)uyi; mz = (Mac)0;
      done = true;
    }
  }
  if (has_hi) {
    const int src = nx - 2 - cell_lo;
    const int defer = __shfl_sync(0xffffffffu, (int)(near && !solid), src);
    if (!defer) {
      // the outlet reads fDst at nx-2 before the walls (:363): the stored value,
      // or for a solid cell whatever fDst holds there (never written)
      double send[19];
      const bool stale = (ix == nx - 2) && solid;
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        if (stale) send[d] = S::f_of(blk[slot_of(d) * pitch + ix], d);
        else send[d] = S::f_of(S::raw_of_f(v[d], d), d);
      }
      const double m0 = __shfl_sync(0xffffffffu, stale ? 1.0 : (double)mr, src);
      const double m1 = __shfl_sync(0xffffffffu, stale ? 0.0 : (double)mx, src);
      const double m2 = __shfl_sync(0xffffffffu, stale ? 0.0 : (double)my, src);
      const double m3 = __shfl_sync(0xffffffffu, stale ? 0.0 : (double)mz, src);
#pragma unroll
      for (int d = 0; d < 19; ++d) send[d] = __shfl_sync(0xffffffffu, send[d], src);
      if (ix == nx - 1 && !solid) {
        const double ro = m0 * 0.85 + 1.0 * 0.15;
#pragma unroll
        for (int d = 0; d < 19; ++d) v[d] = 0.75 * send[d] + 0.25 * feq64(d, ro, m1, m2, m3);
        mr = (Mac)ro;
        mx = (Mac)m1; my = (Mac)m2; mz = (Mac)m3;
        done = true;
      }
    }
  }
  // ---- wall conditions (:375-429): own moments, floor, ceiling, then sides ----
  if (wall_row && done && !xface && flag == CELL_FLUID) {
    if (iy == 0) {
      if (a.ground_no_slip) { mx = (Mac)0; mz = (Mac)0; }
      my = (Mac)0;
    }
    if (iy == ny - 1) my = (Mac)0;
    if (nz > 4 && (iz == 0 || iz == nz - 1)) mz = (Mac)0;
    wall_feq<S, MODE>(v, (double)mr, (double)mx, (double)my, (double)mz);
  }
  if (done) {
    T* out = blk + ix;
#pragma unroll
    for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch] = S::raw_of_f(v[d], d);
    if (mr == mr) add += rho_fixed(mr);
    else *my_nan = 1;
  }
  if (a.write_macro) {
    const long long di = cc.row * nx + ix;
    if (active && solid) {  // solid macro (:173-179)
      a.mux[di] = 0.0f; a.muy[di] = 0.0f; a.muz[di] = 0.0f; a.mrho[di] = 1.0f;
    } else if (done) {
      a.mux[di] = (float)mx; a.muy[di] = (float)my; a.muz[di] = (float)mz; a.mrho[di] = (float)mr;
    }
  }
  return add;
}

// The row ends' equilibria round every operation explicitly (FMA forms), so that the
// lane-transposed row ends (a run-time direction per lane) and the helper warp's end
// pairs (end_pair, unrolled directions) give the same bits: in the storage domain
// OS w_d h + OW w_d with h = A + rho (cu + cu^2 / 2), cu = 3 c_d . u and
// A = (rho - 1) - 1.5 rho u^2 shared by the cell's directions.  The run-time dot product
// adds the zero products c_a u_a = +-0 that dotc leaves out, which changes no sum but the
// sign of a zero, and that sign does not reach the result; OS is a power of two, so OS w_d
// is exact either way.
__device__ __forceinline__ float end_A(float rho, float ux, float uy, float uz) {
  const float usq = __fmaf_rn(ux, ux, __fmaf_rn(uy, uy, __fmul_rn(uz, uz)));
  return __fmaf_rn(__fmul_rn(-1.5f, rho), usq, __fsub_rn(rho, 1.0f));
}
template <class S>
__device__ __forceinline__ float end_eq(float dot, float w, float rho, float A) {
  const float cu = __fmul_rn(3.0f, dot);
  const float h = __fmaf_rn(rho, __fmaf_rn(__fmul_rn(0.5f, cu), cu, cu), A);
  return __fmaf_rn(S::kOutScale * w, h, S::kOutW * w);
}
// The dot product c . u of a run-time direction c = (c_x, c_y, c_z, w).
__device__ __forceinline__ float dot_lane(const float4 c, float ux, float uy, float uz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(c.x, ux), __fmul_rn(c.y, uy)), __fmul_rn(c.z, uz));
}
// The row ends' density from their source cell's: 0.85 rho + 0.15 (:336, :358).
__device__ __forceinline__ float end_rho(float r) { return __fmaf_rn(0.85f, r, 0.15f); }
// Outlet value: 0.75 of the source cell's post-collision value plus 0.25 of the
// equilibrium q of its moments (:361-368), both in the storage domain.
__device__ __forceinline__ float outlet_blend(float prev, float q) {
  return __fmaf_rn(0.75f, prev, __fmul_rn(0.25f, q));
}

// compensate_lanes' correction as lane 0 sums it (the butterfly's order), for a cell whose
// 19 values one thread holds: the rounding errors of directions 1..18.
template <class S>
__device__ __forceinline__ float lane_order_errors(const float (&q)[19]) {
  float e[32];
#pragma unroll
  for (int l = 0; l < 32; ++l) e[l] = (l >= 1 && l < 19) ? q[l] - S::raw(S::store(q[l])) : 0.0f;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int l = 0; l < o; ++l) e[l] = e[l] + e[l + o];
  }
  return e[0];
}

// One FP32-arithmetic consumer segment (32 cells of an x-row), shared by the
// single-lattice and the batched step kernel.  v holds the lane's pulled deviations;
// every lane collides its cell; near-wall cells are left to the near-wall pass and
// solids are never written.  The inlet and outlet cells of the row are written
// lane-transposed (lane d writes direction d) from the density of ix = 1 and the
// post-collision, pre-wall values of nx-2 (shuffles and the 20-float row xo); the wall
// rows replace a cell's result by the equilibrium of its moments.  inlet_u(iy) gives
// the inlet velocity (float2) of row iy; m carries the macro outputs.
struct SegGeom {
  long long row;            // x-row of the segment
  int nx, ny, nz, pitch;
  int iy, iz, cell_lo, ix;  // row coordinates, cell of lane 0, this lane's cell
  int flag;
  bool row_ok, active, near, wall_row, ground_no_slip, write_macro;
  uint8_t cl;               // this lane's class byte
};

template <class S, class InletFn, int MLP = MLP_NONE>
__device__ __forceinline__ void fast_segment(float (&v)[19], typename S::T* __restrict__ fd, const SegGeom g,
                                             float tau0, float k_smag, float2 dec, InletFn inlet_u,
                                             const StepArgs& m,
                                             float* xo, const float4* s_dcw, const int* s_dslot, int lane,
                                             long long& my_sum, int& my_nan, const MlpRefs* mlp = nullptr) {
  using T = typename S::T;
  const int nx = g.nx, ny = g.ny, nz = g.nz, pitch = g.pitch, cell_lo = g.cell_lo, ix = g.ix;
  const long long row = g.row;
  T* const blk = fd + row * 19 * pitch;
  const bool own = g.active && g.flag != CELL_SOLID && !g.near && ix != 0 && ix != nx - 1;
  float r, ux, uy, uz;
  if constexpr (MLP != MLP_NONE) {
    MlpRefs mr = *mlp;
    mr.wall_dist = (float)(g.cl >> 3);
    collide_fast<S, MLP>(v, r, ux, uy, uz, tau0, k_smag, dec, &mr);  // v: storage domain
  } else {
    collide_fast<S>(v, r, ux, uy, uz, tau0, k_smag, dec);
  }
  if (g.row_ok && cell_lo <= 0 && 1 <= cell_lo + 31) {
    // inlet (:328-352): density of ix = 1 (1 for a solid, :177); a near-wall ix = 1
    // defers the inlet to the near-wall pass, a solid ix = 0 has none
    const int c0 = __shfl_sync(0xffffffffu, (int)g.cl, -cell_lo);
    const int c1 = __shfl_sync(0xffffffffu, (int)g.cl, 1 - cell_lo);
    const float r1 = __shfl_sync(0xffffffffu, r, 1 - cell_lo);
    const bool solid1 = (c1 & CLS_FLAG_MASK) == CELL_SOLID;
    if ((c0 & CLS_FLAG_MASK) != CELL_SOLID && !((c1 & CLS_NEAR) && !solid1)) {
      const float ri = end_rho(solid1 ? 1.0f : r1);
      const float2 ui = inlet_u(g.iy);
      float q = 0.0f;
      if (lane < 19) {
        const float4 cw = s_dcw[lane];
        q = end_eq<S>(dot_lane(cw, ui.x, ui.y, 0.0f), cw.w, ri, end_A(ri, ui.x, ui.y, 0.0f));
      }
      q = compensate_lanes<S>(q, lane);
      if (lane < 19) blk[s_dslot[lane] * pitch] = S::store(q);
      if (lane == 0) {
        if (ri == ri) my_sum += rho_fixed(ri);
        else my_nan = 1;
        if (g.write_macro) {
          const long long ic = row * nx;
          m.mux[ic] = ui.x; m.muy[ic] = ui.y; m.muz[ic] = 0.0f; m.mrho[ic] = ri;
        }
      }
    }
  }
  if (g.row_ok && cell_lo <= nx - 2 && nx - 1 <= cell_lo + 31) {
    // outlet (:354-371) from the post-collision, pre-wall cell nx-2, or from what fDst
    // holds there when nx-2 is solid; a near-wall nx-2 defers it
    const int src = nx - 2 - cell_lo;
    const int c2 = __shfl_sync(0xffffffffu, (int)g.cl, src);
    const int c3 = __shfl_sync(0xffffffffu, (int)g.cl, src + 1);
    const bool stale = (c2 & CLS_FLAG_MASK) == CELL_SOLID;
    const float r2 = __shfl_sync(0xffffffffu, r, src);
    const float ox = __shfl_sync(0xffffffffu, ux, src);
    const float oy = __shfl_sync(0xffffffffu, uy, src);
    const float oz = __shfl_sync(0xffffffffu, uz, src);
    if ((c3 & CLS_FLAG_MASK) != CELL_SOLID && !((c2 & CLS_NEAR) && !stale)) {
      if (lane == src && !stale) {
#pragma unroll
        for (int d = 0; d < 19; ++d) xo[slot_of(d)] = v[d];
      }
      __syncwarp();
      const float ro = end_rho(stale ? 1.0f : r2);
      const float mx = stale ? 0.0f : ox, my = stale ? 0.0f : oy, mz = stale ? 0.0f : oz;
      float q = 0.0f;
      const int sl = lane < 19 ? s_dslot[lane] : 0;
      if (lane < 19) {
        const float prev = stale ? (float)blk[sl * pitch + nx - 2] : xo[sl];
        const float4 cw = s_dcw[lane];
        q = outlet_blend(prev, end_eq<S>(dot_lane(cw, mx, my, mz), cw.w, ro, end_A(ro, mx, my, mz)));
      }
      q = compensate_lanes<S>(q, lane);
      if (lane < 19) blk[sl * pitch + nx - 1] = S::store(q);
      __syncwarp();
      if (lane == 0) {
        if (ro == ro) my_sum += rho_fixed(ro);
        else my_nan = 1;
        if (g.write_macro) {
          const long long oc = row * nx + nx - 1;
          m.mux[oc] = mx; m.muy[oc] = my; m.muz[oc] = mz; m.mrho[oc] = ro;
        }
      }
    }
  }
  if (g.wall_row) {  // floor, ceiling, then sides (:375-429), fluid cells only
    if (g.iy == 0) {
      if (g.ground_no_slip) { ux = 0.0f; uz = 0.0f; }
      uy = 0.0f;
    }
    if (g.iy == ny - 1) uy = 0.0f;
    if (nz > 4 && (g.iz == 0 || g.iz == nz - 1)) uz = 0.0f;
#pragma unroll
    for (int d = 0; d < 19; ++d) v[d] = fmaf(S::kOutScale, heq32(d, r, ux, uy, uz), S::kOutW * wf_of(d));
  }
  if (own) {
    T* out = blk + ix;
    compensate_cell<S>(v);
#pragma unroll
    for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch] = S::store(v[d]);
    if (r == r) my_sum += rho_fixed(r);
    else my_nan = 1;
  }
  if (g.write_macro && g.active) {
    const long long di = row * nx + ix;
    if (g.flag == CELL_SOLID) {  // solid macro (:173-179)
      m.mux[di] = 0.0f; m.muy[di] = 0.0f; m.muz[di] = 0.0f; m.mrho[di] = 1.0f;
    } else if (own) {
      m.mux[di] = ux; m.muy[di] = uy; m.muz[di] = uz; m.mrho[di] = r;
    }
  }
}

// Packed loads and stores of two adjacent cells (the first at an even element offset, so
// the pair is 4- or 8-byte aligned) in the raw storage domain.
template <class S>
__device__ __forceinline__ float2 load_pair(const typename S::T* p) {
  using T = typename S::T;
  if constexpr (sizeof(T) == 4) {
    return *reinterpret_cast<const float2*>(p);
  } else if constexpr (std::is_same<T, __half>::value) {
    return __half22float2(*reinterpret_cast<const __half2*>(p));
  } else {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
  }
}
template <class S>
__device__ __forceinline__ void store_pair(typename S::T* p, float2 v) {
  using T = typename S::T;
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float2*>(p) = v;
  } else if constexpr (std::is_same<T, __half>::value) {
    *reinterpret_cast<__half2*>(p) = __float22half2_rn(v);
  } else {
    *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(v);
  }
}

// Geometry of a two-cells-per-thread segment: 64 cells of an x-row with an even cell
// count, lane l holding cells x0 = cell_lo + 2 l and x0 + 1.
struct PairGeom {
  long long row;
  int nx, ny, nz, pitch;
  int iy, iz, x0;
  int cell_lo;           // first cell of lane 0
  bool active;           // both cells lie in the row (nx even: x0 < nx implies x0 + 1 < nx)
  bool has_lo, has_hi;   // the segment holds cell 0 / cell nx-1 (warp-uniform)
  bool wall_row, ground_no_slip, write_macro;
  uint8_t c0, c1;        // class bytes of the two cells
};

// The consumer work of a two-cells-per-thread segment: the same per-cell semantics as
// fast_segment (pull values in v, collision, inlet and outlet of the row, wall rows,
// stores, density sum, macro outputs).  The thread that holds cell 0 holds cell 1 too, and
// the thread that holds cell nx-1 holds nx-2, so the boundary conditions' sources
// (lbmCpuReference.ts:323-373) sit with the row end: the outlet's (cell nx-2 after the
// collision, before any wall condition: 19 values and the moments) are parked in the
// warp's scratch row xo[24].  After the cells' own stores the warp holding a row end writes
// it lane-transposed (lane d writes direction d), so the row-end work is one equilibrium
// per lane and not 19 per thread, whether the compiler branches around it or predicates it.
// ENDS = false: the two pairs of the row that hold its ends, (0, 1) and (nx-2, nx-1), are
// left out altogether (no stores, density sums or macros) -- the helper warp computes
// them from the same ring slot (end_pair) -- and the segment carries no row-end code.
template <class S, class InletFn, bool ENDS = true>
__device__ __forceinline__ void pair_segment(float2 (&v)[19], typename S::T* __restrict__ fd, const PairGeom g,
                                             float tau0, float k_smag, float2 dec, InletFn inlet_u,
                                             const StepArgs& m, float* xo, const float4* s_dcw,
                                             const int* s_dslot, int lane, long long& my_sum, int& my_nan) {
  using T = typename S::T;
  constexpr float OS = S::kOutScale, OW = S::kOutW;
  const int nx = g.nx, ny = g.ny, nz = g.nz, pitch = g.pitch, x0 = g.x0;
  const long long row = g.row;
  T* const blk = fd + row * 19 * pitch;
  float2 r, ux, uy, uz;
  collide_fast2<S>(v, r, ux, uy, uz, tau0, k_smag, dec);  // v: storage domain
  const int f0 = g.c0 & CLS_FLAG_MASK, f1 = g.c1 & CLS_FLAG_MASK;
  const bool mine = ENDS || (x0 != 0 && x0 + 2 != nx);  // not a pair of the helper warp
  const bool own0 = mine && g.active && f0 != CELL_SOLID && !(g.c0 & CLS_NEAR) && x0 != 0;
  const bool own1 = mine && g.active && f1 != CELL_SOLID && !(g.c1 & CLS_NEAR) && x0 + 1 != nx - 1;
  if (ENDS && g.has_hi && x0 == nx - 2) {  // the outlet's sources
#pragma unroll
    for (int d = 0; d < 19; ++d) xo[slot_of(d)] = v[d].x;
    xo[19] = r.x; xo[20] = ux.x; xo[21] = uy.x; xo[22] = uz.x;
  }
  if (g.wall_row) {  // floor, ceiling, then sides (:375-429), fluid cells only
    if (g.iy == 0) {
      if (g.ground_no_slip) { ux = f2(0.0f); uz = f2(0.0f); }
      uy = f2(0.0f);
    }
    if (g.iy == ny - 1) uy = f2(0.0f);
    if (nz > 4 && (g.iz == 0 || g.iz == nz - 1)) uz = f2(0.0f);
    heq_pair<S>(v, r, ux, uy, uz);
  }
  T* out = blk + x0;
  // A row end (cell 0 or nx-1) that this warp rewrites below -- the inlet or the outlet,
  // after a __syncwarp that orders the warp's global stores -- takes the pair store with
  // its neighbour, so the lanes of a row-end segment all store pairs instead of
  // diverging into per-cell stores.  Not for a solid row end (never written) nor with a
  // near-wall neighbour (the near-wall pass writes the row end then).
  const bool pair_st = (own0 && own1) || (own1 && x0 == 0 && f0 != CELL_SOLID) ||
                       (own0 && x0 + 1 == nx - 1 && f1 != CELL_SOLID);
  if constexpr (S::kCompensate) {
    // mass-compensated rounding (compensate_cell) of both cells: the moving directions
    // round first, as packed half2 that are kept for the stores, and direction 0 takes
    // what their rounded values leave of the cell's deviation sum.  The collision and the
    // wall equilibrium both conserve the density, so the 19 values sum to
    // kOutScale (r - 1) (kOutW is 0 for the shifted codecs): direction 0 is formed from
    // that sum rather than from its own value plus the rounding errors, which needs no
    // second copy of the 18 values
    static_assert(std::is_same<T, __half>::value && OW == 0.0f, "compensated rounding is a shifted FP16 codec");
    __half2 hv[19];
    float2 sr = f2(0.0f);
#pragma unroll
    for (int d = 1; d < 19; ++d) {
      hv[d] = __float22half2_rn(v[d]);
      sr = f2add(sr, __half22float2(hv[d]));
    }
    hv[0] = __float22half2_rn(f2sub(f2mul(f2(OS), f2sub(r, f2(1.0f))), sr));
    if (pair_st) {
#pragma unroll
      for (int d = 0; d < 19; ++d) *reinterpret_cast<__half2*>(out + slot_of(d) * pitch) = hv[d];
    } else if (own0 || own1) {
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        if (own0) out[slot_of(d) * pitch] = __low2half(hv[d]);
        if (own1) out[slot_of(d) * pitch + 1] = __high2half(hv[d]);
      }
    }
  } else if (pair_st) {
#pragma unroll
    for (int d = 0; d < 19; ++d) store_pair<S>(out + slot_of(d) * pitch, v[d]);
  } else if (own0 || own1) {
#pragma unroll
    for (int d = 0; d < 19; ++d) {
      if (own0) out[slot_of(d) * pitch] = S::store(v[d].x);
      if (own1) out[slot_of(d) * pitch + 1] = S::store(v[d].y);
    }
  }
  if (own0) {
    if (r.x == r.x) my_sum += rho_fixed(r.x);
    else my_nan = 1;
  }
  if (own1) {
    if (r.y == r.y) my_sum += rho_fixed(r.y);
    else my_nan = 1;
  }
  if (g.write_macro && g.active && mine) {
    const long long di = row * nx + x0;
    if (f0 == CELL_SOLID) {  // solid macro (:173-179)
      m.mux[di] = 0.0f; m.muy[di] = 0.0f; m.muz[di] = 0.0f; m.mrho[di] = 1.0f;
    } else if (own0) {
      m.mux[di] = ux.x; m.muy[di] = uy.x; m.muz[di] = uz.x; m.mrho[di] = r.x;
    }
    if (f1 == CELL_SOLID) {
      m.mux[di + 1] = 0.0f; m.muy[di + 1] = 0.0f; m.muz[di + 1] = 0.0f; m.mrho[di + 1] = 1.0f;
    } else if (own1) {
      m.mux[di + 1] = ux.y; m.muy[di + 1] = uy.y; m.muz[di + 1] = uz.y; m.mrho[di + 1] = r.y;
    }
  }
  if constexpr (!ENDS) return;
  if (g.has_lo) {
    // inlet (:328-352) from the density of cell 1 (1 for a solid, :177; the walls leave
    // the density as it is), both held by lane 0; a near-wall cell 1 defers it to the
    // near-wall pass, a solid cell 0 has none
    const int c0 = __shfl_sync(0xffffffffu, (int)g.c0, 0), c1 = __shfl_sync(0xffffffffu, (int)g.c1, 0);
    const float r1 = __shfl_sync(0xffffffffu, r.y, 0);
    const bool solid1 = (c1 & CLS_FLAG_MASK) == CELL_SOLID;
    if ((c0 & CLS_FLAG_MASK) != CELL_SOLID && !((c1 & CLS_NEAR) && !solid1)) {
      const float ri = end_rho(solid1 ? 1.0f : r1);
      const float2 ui = inlet_u(g.iy);
      float q = 0.0f;
      if (lane < 19) {
        const float4 cw = s_dcw[lane];
        q = end_eq<S>(dot_lane(cw, ui.x, ui.y, 0.0f), cw.w, ri, end_A(ri, ui.x, ui.y, 0.0f));
      }
      q = compensate_lanes<S>(q, lane);
      __syncwarp();  // after lane 0's pair store of cells 0 and 1
      if (lane < 19) blk[s_dslot[lane] * pitch] = S::store(q);
      if (lane == 0) {
        if (ri == ri) my_sum += rho_fixed(ri);
        else my_nan = 1;
        if (g.write_macro) {
          const long long ic = row * nx;
          m.mux[ic] = ui.x; m.muy[ic] = ui.y; m.muz[ic] = 0.0f; m.mrho[ic] = ri;
        }
      }
    }
  }
  if (g.has_hi) {
    // outlet (:354-371) from the parked cell nx-2, or from what fDst holds there when
    // nx-2 is solid; a near-wall nx-2 defers it
    const int src = (nx - 2 - g.cell_lo) >> 1;
    const int c2 = __shfl_sync(0xffffffffu, (int)g.c0, src), c3 = __shfl_sync(0xffffffffu, (int)g.c1, src);
    const bool stale = (c2 & CLS_FLAG_MASK) == CELL_SOLID;
    if ((c3 & CLS_FLAG_MASK) != CELL_SOLID && !((c2 & CLS_NEAR) && !stale)) {
      __syncwarp();  // the parked row xo, and the pair store of cells nx-2 and nx-1 before ours
      const float ro = end_rho(stale ? 1.0f : xo[19]);
      const float mx = stale ? 0.0f : xo[20], my = stale ? 0.0f : xo[21], mz = stale ? 0.0f : xo[22];
      float q = 0.0f;
      const int sl = lane < 19 ? s_dslot[lane] : 0;
      if (lane < 19) {
        const float prev = stale ? S::raw(blk[sl * pitch + nx - 2]) : xo[sl];
        const float4 cw = s_dcw[lane];
        q = outlet_blend(prev, end_eq<S>(dot_lane(cw, mx, my, mz), cw.w, ro, end_A(ro, mx, my, mz)));
      }
      q = compensate_lanes<S>(q, lane);
      if (lane < 19) blk[sl * pitch + nx - 1] = S::store(q);
      __syncwarp();  // the scratch row is free for the next segment
      if (lane == 0) {
        if (ro == ro) my_sum += rho_fixed(ro);
        else my_nan = 1;
        if (g.write_macro) {
          const long long oc = row * nx + nx - 1;
          m.mux[oc] = mx; m.muy[oc] = my; m.muz[oc] = mz; m.mrho[oc] = ro;
        }
      }
    }
  }
}

// One component of heq_pair with the same operations, so that a cell's equilibrium
// rounds as it would in the pair form: OS (feq_d - w_d) + OW w_d.
template <class S>
__device__ __forceinline__ float heq_one(int d, float r, float ux, float uy, float uz) {
  constexpr float OS = S::kOutScale, OW = S::kOutW;
  const float u2 = __fmaf_rn(ux, ux, __fmaf_rn(uy, uy, __fmul_rn(uz, uz)));
  const float A = __fmaf_rn(__fmul_rn(-1.5f, r), u2, __fsub_rn(r, 1.0f));
  const float cu = __fmul_rn(3.0f, dotc(d, ux, uy, uz));
  const float h = __fmaf_rn(r, __fmaf_rn(__fmul_rn(0.5f, cu), cu, cu), A);
  return __fmaf_rn(OS * wf_of(d), h, OW * wf_of(d));
}

// A pair of an x-row that holds one of its ends: cells (0, 1) (x0 = 0) or (nx-2, nx-1).
struct EndGeom {
  long long row;
  int nx, ny, nz, pitch;
  int iy, iz, x0;
  bool wall_row, ground_no_slip, write_macro;
  uint8_t c0, c1;  // class bytes of the two cells
};

// The helper warp's share of a two-cells-per-thread step: one lane per row-end pair,
// pulled from the ring slot like a consumer pair, with pair_segment's semantics for
// both cells -- the collision of both, the inlet of cell 0 from the density of cell 1
// (:328-352) or the outlet of cell nx-1 from the post-collision, pre-wall values of
// cell nx-2 (:354-371), the wall condition of the pair's interior cell (:375-429), the
// stores, the density sum and the macro outputs -- with the row end's 19 equilibria
// evaluated in the lane itself.  A near-wall interior cell defers the row end to the
// near-wall pass (near_cell writes both), a solid row end is never written.  Returns
// the fixed-point density added to the step's sum.
template <class S, class InletFn>
__device__ __forceinline__ long long end_pair(float2 (&v)[19], typename S::T* __restrict__ fd, const EndGeom g,
                                              float tau0, float k_smag, float2 dec, InletFn inlet_u,
                                              const StepArgs& m, int& my_nan) {
  using T = typename S::T;
  constexpr float OS = S::kOutScale;
  const int pitch = g.pitch;
  const bool lo = g.x0 == 0;
  T* const out = fd + g.row * 19 * pitch + g.x0;
  float2 r, ux, uy, uz;
  collide_fast2<S>(v, r, ux, uy, uz, tau0, k_smag, dec);  // v: storage domain
  const int f0 = g.c0 & CLS_FLAG_MASK, f1 = g.c1 & CLS_FLAG_MASK;
  // the interior cell (1 or nx-2), unless solid or near-wall
  const bool own = lo ? (f1 != CELL_SOLID && !(g.c1 & CLS_NEAR)) : (f0 != CELL_SOLID && !(g.c0 & CLS_NEAR));
  bool end = false;                              // the row end is written here
  float er = 0.0f, eu = 0.0f, ev = 0.0f, ew = 0.0f;  // its density and velocity
  if (lo) {
    if (f0 != CELL_SOLID && !((g.c1 & CLS_NEAR) && f1 != CELL_SOLID)) {
      er = end_rho(f1 == CELL_SOLID ? 1.0f : r.y);
      const float2 ui = inlet_u(g.iy);
      eu = ui.x;
      ev = ui.y;
      const float A = end_A(er, eu, ev, 0.0f);
#pragma unroll
      for (int d = 0; d < 19; ++d) v[d].x = end_eq<S>(dotc(d, eu, ev, 0.0f), wf_of(d), er, A);
      end = true;
    }
  } else {
    const bool stale = f0 == CELL_SOLID;  // fDst's values of a solid nx-2 (never written)
    if (f1 != CELL_SOLID && !((g.c0 & CLS_NEAR) && !stale)) {
      er = end_rho(stale ? 1.0f : r.x);
      eu = stale ? 0.0f : ux.x;
      ev = stale ? 0.0f : uy.x;
      ew = stale ? 0.0f : uz.x;
      const float A = end_A(er, eu, ev, ew);
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        const float prev = stale ? S::raw(out[slot_of(d) * pitch]) : v[d].x;
        v[d].y = outlet_blend(prev, end_eq<S>(dotc(d, eu, ev, ew), wf_of(d), er, A));
      }
      end = true;
    }
  }
  if (g.wall_row) {  // floor, ceiling, then sides, on the interior cell
    if (g.iy == 0) {
      if (g.ground_no_slip) { ux = f2(0.0f); uz = f2(0.0f); }
      uy = f2(0.0f);
    }
    if (g.iy == g.ny - 1) uy = f2(0.0f);
    if (g.nz > 4 && (g.iz == 0 || g.iz == g.nz - 1)) uz = f2(0.0f);
    if (lo) {
#pragma unroll
      for (int d = 0; d < 19; ++d) v[d].y = heq_one<S>(d, r.y, ux.y, uy.y, uz.y);
    } else {
#pragma unroll
      for (int d = 0; d < 19; ++d) v[d].x = heq_one<S>(d, r.x, ux.x, uy.x, uz.x);
    }
  }
  const bool s0 = lo ? end : own, s1 = lo ? own : end;
  if constexpr (S::kCompensate) {
    // the interior cell's direction 0 from its deviation sum OS (r - 1) as in
    // pair_segment, the row end's from its own value plus the moving directions'
    // rounding errors, summed in compensate_lanes' order
    static_assert(std::is_same<T, __half>::value, "compensated rounding is a shifted FP16 codec");
    float q[19];
#pragma unroll
    for (int d = 0; d < 19; ++d) q[d] = lo ? v[d].x : v[d].y;
    const float q0 = q[0] + lane_order_errors<S>(q);
    __half2 hv[19];
    float2 sr = f2(0.0f);
#pragma unroll
    for (int d = 1; d < 19; ++d) {
      hv[d] = __float22half2_rn(v[d]);
      sr = f2add(sr, __half22float2(hv[d]));
    }
    const float ix = OS * (r.x - 1.0f) - sr.x, iy_ = OS * (r.y - 1.0f) - sr.y;
    hv[0] = __floats2half2_rn(lo ? q0 : ix, lo ? iy_ : q0);
    if (s0 && s1) {
#pragma unroll
      for (int d = 0; d < 19; ++d) *reinterpret_cast<__half2*>(out + slot_of(d) * pitch) = hv[d];
    } else if (s0) {
#pragma unroll
      for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch] = __low2half(hv[d]);
    } else if (s1) {
#pragma unroll
      for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch + 1] = __high2half(hv[d]);
    }
  } else if (s0 && s1) {
#pragma unroll
    for (int d = 0; d < 19; ++d) store_pair<S>(out + slot_of(d) * pitch, v[d]);
  } else if (s0) {
#pragma unroll
    for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch] = S::store(v[d].x);
  } else if (s1) {
#pragma unroll
    for (int d = 0; d < 19; ++d) out[slot_of(d) * pitch + 1] = S::store(v[d].y);
  }
  long long add = 0;
  const float ri = lo ? r.y : r.x;
  if (own) {
    if (ri == ri) add += rho_fixed(ri);
    else my_nan = 1;
  }
  if (end) {
    if (er == er) add += rho_fixed(er);
    else my_nan = 1;
  }
  if (g.write_macro) {
    const long long di = g.row * g.nx + g.x0;
    const float ru = lo ? ux.y : ux.x, rv = lo ? uy.y : uy.x, rw = lo ? uz.y : uz.x;
    if (f0 == CELL_SOLID) {  // solid macro (:173-179)
      m.mux[di] = 0.0f; m.muy[di] = 0.0f; m.muz[di] = 0.0f; m.mrho[di] = 1.0f;
    } else if (s0) {
      m.mux[di] = lo ? eu : ru; m.muy[di] = lo ? ev : rv; m.muz[di] = lo ? ew : rw; m.mrho[di] = lo ? er : ri;
    }
    if (f1 == CELL_SOLID) {
      m.mux[di + 1] = 0.0f; m.muy[di + 1] = 0.0f; m.muz[di + 1] = 0.0f; m.mrho[di + 1] = 1.0f;
    } else if (s1) {
      m.mux[di + 1] = lo ? ru : eu; m.muy[di + 1] = lo ? rv : ev; m.muz[di + 1] = lo ? rw : ew;
      m.mrho[di + 1] = lo ? ri : er;
    }
  }
  return add;
}

// CPT: consumer cells per thread, 1 or 2 (MODE_FAST without the closure, even nx; the
// host chooses, pair_segment does the work).
template <class S, int MODE, int P, int MLP = MLP_NONE, int CPT = 1>
__global__ void __launch_bounds__(kStepThreads, step_min_blocks<S, MODE, MLP, CPT>())
    main_kernel(const __grid_constant__ StepArgs a) {
  static_assert(CPT == 1 || (MODE == MODE_FAST && MLP == MLP_NONE), "two cells per thread: fast mode only");
  using T = typename S::T;
  using Real = typename std::conditional<MODE == MODE_FAST, float, double>::type;
  using Mac = typename MacroOf<T>::type;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ long long red[kConsumerWarps + 2];
  __shared__ int nan_flag;
  __shared__ long long s_first[8];  // dynamic deal: first row of the item in ring slot s (-1: none left)

  const Layout& L = a.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int pitch = P ? P : L.pitch;
  const int S_ = a.stages;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int shift = row_shift(nx, CPT), span = row_span(nx, CPT), RY = rows_per_item(nx, CPT);
  const int wpr = span / 32;
  const long long rows = (long long)ny * nz;
  const int G = step_item_grouped<S, MODE, MLP>() && a.item_groups > 1 ? a.item_groups : 1;
  const int RYG = RY * G;  // rows per work item
  const long long n_items = (rows + RYG - 1) / RYG;
  const int my_count = blockIdx.x < n_items ? (int)((n_items - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  // Odd steps take the items last to first: a step then begins on the rows the step
  // before wrote last, while they are still in L2.  Every cell's update reads only the
  // source lattice and the density sums are fixed-point, so the order changes no result.
  const bool reverse = (a.step_index & 1) != 0;
  const long long item_row0 = (reverse ? n_items - 1 - blockIdx.x : (long long)blockIdx.x) * RYG;
  const long long item_step = reverse ? -(long long)gridDim.x * RYG : (long long)gridDim.x * RYG;

  T* spop = reinterpret_cast<T*>(smem_raw + kSmemGuard);
  uint8_t* scls = smem_raw + kSmemGuard + (size_t)S_ * RYG * 19 * pitch * sizeof(T);
  uint64_t* full = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(scls + (size_t)S_ * RYG * pitch + kSmemGuard) + 7) & ~uintptr_t(7));
  uint64_t* empty = full + S_;
  double* s_uxi = reinterpret_cast<double*>(empty + S_);
  double* s_uyi = s_uxi + ny;
  int2* s_row = reinterpret_cast<int2*>(s_uyi + ny);        // [S_][RYG] (iy, iz) of the slot's rows
  float* s_xo = reinterpret_cast<float*>(s_row + S_ * RYG);  // [kConsumerWarps][24]
  float4* s_dcw = reinterpret_cast<float4*>(
      (reinterpret_cast<uintptr_t>(s_xo + kConsumerWarps * 24) + 15) & ~uintptr_t(15));  // [19]
  int* s_dslot = reinterpret_cast<int*>(s_dcw + 19);                                     // [19]
  // learned closure: weight fragments, biases, one staging block per consumer warp
  uint32_t* s_mfrag = reinterpret_cast<uint32_t*>(s_dslot + 19);                          // [24 * 32]
  float* s_mbias = reinterpret_cast<float*>(s_mfrag + kMlpFragWords * 32);               // [65]
  uint32_t* s_mstage = reinterpret_cast<uint32_t*>(s_mbias + kMlpBias + 3);              // [8][128]
  if constexpr (MLP != MLP_NONE) {
    for (int i = threadIdx.x; i < kMlpFragWords * 32; i += blockDim.x) s_mfrag[i] = a.mlp_frag[i];
    for (int i = threadIdx.x; i < kMlpBias; i += blockDim.x) s_mbias[i] = a.mlp_bias[i];
  }
  // tcgen05 closure: the weight image, per group of four consumer warps its A operands
  // and completion mbarrier, and the TMEM address slot (128-byte aligned region)
  uint8_t* s_umma = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(s_mstage + kConsumerWarps * 128) + 127) & ~uintptr_t(127));
  uint8_t* s_ub = s_umma;                                                   // weight image
  uint8_t* s_ua = s_umma + kUmmaBBytes;                                     // [group] A1, A2
  uint64_t* s_umbar = reinterpret_cast<uint64_t*>(s_ua + kStepUmmaGroups * (kStepUmmaA1 + kStepUmmaA2));
  uint32_t* s_utmem = reinterpret_cast<uint32_t*>(s_umbar + kStepUmmaGroups);

  const T* __restrict__ fs = static_cast<const T*>(a.fsrc);
  T* __restrict__ fd = static_cast<T*>(a.fdst);

  // Consumer warps that own a row segment: RY rows of wpr warps.  When wpr does not
  // divide the 8 consumer warps (row spans of 96, 160, 192, 224 threads) the
  // remaining warps take no rows.
  const int n_cons = RY * wpr;
  // Two cells per thread: the helper warp takes the row-end pairs of every item from the
  // ring (end_pair) and releases each slot with the consumers.
  // (16-bit storage only: the FP32 steps, bound by bandwidth, lose more to the helper's
  // slot releases than they gain: 101.4 -> 106.9 us at 256x128x128.)
  constexpr bool kHelperEnds = CPT == 2 && sizeof(T) == 2;
  // the tcgen05 closure needs all 8 consumer warps busy on every item (two full groups);
  // the host launches it only then, and a lattice where that does not hold steps nothing
  // and reports an error instead of leaving a group barrier short of a warp
  const bool groups_ok = MLP != MLP_TCGEN05 || n_cons == kConsumerWarps;
  const int count = groups_ok ? my_count : 0;
  // Dynamic deal: the producer takes items from the step's counter and publishes each
  // item's first row with its slot; a slot holding -1 tells the consumers that no item is
  // left.  Every cell's update reads only the source lattice, so the deal changes no result.
  const bool dyn = a.dynamic_items && groups_ok;
  const int cur_slot = a.step_index & 1;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S_; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], n_cons + (kHelperEnds ? 1 : 0));
    }
    nan_flag = 0;
    if (!groups_ok) atomicOr(&a.st->error, STEP_ERR_PIPELINE_TIMEOUT);
    mbar_fence_init();
  }
  if constexpr (MLP == MLP_TCGEN05) {
    for (int i = threadIdx.x; i < kUmmaBBytes / 16; i += blockDim.x)
      reinterpret_cast<uint4*>(s_ub)[i] = a.mlp_umma[i];
    if (warp < kConsumerWarps) {  // K padding of this thread's row of the input operand
      const int g = warp >> 2, row = (warp & 3) * 32 + lane;
      *reinterpret_cast<uint4*>(s_ua + g * (kStepUmmaA1 + kStepUmmaA2) + umma_off(row, 8, 16)) =
          make_uint4(0u, 0u, 0u, 0u);
    }
    if (threadIdx.x < kStepUmmaGroups) umma_mbar_init(smem_addr(&s_umbar[threadIdx.x]));
    if (warp == 0) {
      tmem_alloc(smem_addr(s_utmem), kStepUmmaTmemCols);
      tmem_relinquish();
    }
    fence_async_smem();
    tc_fence_before();
  }
  if (threadIdx.x < 19) {  // direction table of the lane-transposed row ends
    const int d = threadIdx.x;
    const int px = (1 << 1) | (1 << 7) | (1 << 9) | (1 << 11) | (1 << 13);
    const int mx_ = (1 << 2) | (1 << 8) | (1 << 10) | (1 << 12) | (1 << 14);
    const int py = (1 << 3) | (1 << 7) | (1 << 10) | (1 << 15) | (1 << 17);
    const int my_ = (1 << 4) | (1 << 8) | (1 << 9) | (1 << 16) | (1 << 18);
    const int pz = (1 << 5) | (1 << 11) | (1 << 14) | (1 << 15) | (1 << 18);
    const int mz_ = (1 << 6) | (1 << 12) | (1 << 13) | (1 << 16) | (1 << 17);
    const float w = d == 0 ? 1.0f / 3.0f : (d <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f);
    s_dcw[d] = make_float4((float)(((px >> d) & 1) - ((mx_ >> d) & 1)), (float)(((py >> d) & 1) - ((my_ >> d) & 1)),
                           (float)(((pz >> d) & 1) - ((mz_ >> d) & 1)), w);
    int sl = d;
#pragma unroll
    for (int e = 0; e < 19; ++e)
      if (e == d) sl = slot_of(e);
    s_dslot[d] = sl;
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
  if constexpr (MLP == MLP_TCGEN05) tc_fence_after();
  // Programmatic dependent launch: this CTA may have started while the previous kernel
  // of the stream was still finishing.  Everything above wrote only shared memory and
  // read only inputs the host copied in; wait for that kernel to complete and flush
  // before reading its results or overwriting what it reads.  Then let the next step's
  // CTAs be scheduled as this grid's CTAs exit (all of this grid is resident already).
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  long long my_sum = 0;
  bool failed = false;

  if (warp == kHelperWarp) {
    // ---------------- helper warp: this CTA's share of the near-wall cells ----------------
    // (two cells per thread: and the row-end pairs of every item, one batch of near-wall
    // cells after each item's pairs)
    const int pslot = (a.step_index + 1) & 1;
    const double corr = a.st->apply[pslot] ? a.st->corr[pslot] : 1.0;
    int my_nan = 0;
    auto inlet_d = [&](int y) { return make_double2(s_uxi[y], s_uyi[y]); };
    long long t = (long long)blockIdx.x * 32 + lane;
    const long long t_step = (long long)gridDim.x * 32;
    if constexpr (kHelperEnds) {
      const float corrf = (float)corr;
      const float2 dec = make_float2(corrf * S::kRawScale, corrf - 1.0f);
      auto inlet_f = [&](int y) { return make_float2((float)s_uxi[y], (float)s_uyi[y]); };
      int s = 0;
      uint32_t ph = 0;
      long long r0 = item_row0;
      for (int j = 0; dyn || j < count; ++j, r0 += item_step) {
        const bool ok = mbar_wait(&full[s], ph, a.wait_limit);
        if (!__any_sync(0xffffffffu, ok)) {
          failed = true;
          break;
        }
        if (dyn) {  // the item the producer took for this slot
          const long long first = s_first[s];
          if (first < 0) break;
          r0 = first;
        }
        const int nr = (int)(rows - r0 < RYG ? rows - r0 : RYG);
        for (int e0 = 0; e0 < 2 * nr; e0 += 32) {  // lane e: row e / 2 of the item, end e % 2
          const int e = e0 + lane;
          const bool act = e < 2 * nr;
          const int yy = act ? e >> 1 : 0;
          const int x0 = act && (e & 1) ? nx - 2 : 0;
          const T* sp = spop + (size_t)(s * RYG + yy) * 19 * pitch + x0;
          float2 v[19];
#pragma unroll
          for (int d = 0; d < 19; ++d) {
            const T* q = sp + slot_of(d) * pitch;
            if (cx_of(d) == 0) v[d] = load_pair<S>(q);
            else v[d] = make_float2(S::raw(q[-cx_of(d)]), S::raw(q[1 - cx_of(d)]));
          }
          const uint32_t cls2 = *reinterpret_cast<const uint16_t*>(scls + (size_t)(s * RYG + yy) * pitch + x0);
          const int2 yz = s_row[s * RYG + yy];
          if (e0 + 32 >= 2 * nr) {  // the item's last pull: release the slot
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
          }
          if (act) {
            EndGeom g;
            g.row = r0 + yy; g.nx = nx; g.ny = ny; g.nz = nz; g.pitch = pitch;
            g.iy = yz.x; g.iz = yz.y; g.x0 = x0;
            g.wall_row = yz.x == 0 || yz.x == ny - 1 || (nz > 4 && (yz.y == 0 || yz.y == nz - 1));
            g.ground_no_slip = a.ground_no_slip; g.write_macro = a.write_macro;
            g.c0 = (uint8_t)(cls2 & 0xffu);
            g.c1 = (uint8_t)(cls2 >> 8);
            my_sum += end_pair<S>(v, fd, g, (float)a.tau0, (float)a.k_smag, dec, inlet_f, a, my_nan);
          }
        }
        if (t < a.n_near) {
          my_sum += near_cell<S, MODE, P>(a, a.fsrc, a.fdst, a.write_macro, t, corr, inlet_d, &my_nan);
          t += t_step;
        }
        if (++s == S_) { s = 0; ph ^= 1u; }
      }
    }
    for (; t < a.n_near; t += t_step)
      my_sum += near_cell<S, MODE, P>(a, a.fsrc, a.fdst, a.write_macro, t, corr, inlet_d, &my_nan);
    if (__any_sync(0xffffffffu, my_nan) && lane == 0) nan_flag = 1;
    if (failed && lane == 0) atomicOr(&a.st->error, STEP_ERR_PIPELINE_TIMEOUT);
  } else if (warp == kProducerWarp) {
    // ---------------- producer warp: lanes issue the copies of an item in parallel ----------------
    const uint32_t slot_bytes = (uint32_t)(pitch * sizeof(T));
    int issued = 0;
    int end_slot = -1;  // the slot that took the dynamic deal's end mark
    int s = 0;
    uint32_t ph = 0;  // parity of the slot's current fill
    long long r0 = item_row0;  // first row of this CTA's j-th item
    for (int j = 0;; ++j, r0 += item_step) {
      long long k = 0;  // dynamic deal: this fill's item (-1: none left)
      if (dyn) {
        if (lane == 0) k = (long long)atomicAdd(&a.st->next_item[cur_slot], 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= n_items) k = -1;
        else r0 = (reverse ? n_items - 1 - k : k) * RYG;
      } else if (j >= count) {
        break;
      }
      if (j >= S_) {  // the slot's previous fill must have been consumed
        const bool ok = mbar_wait(&empty[s], ph ^ 1u, a.wait_limit);
        if (!__any_sync(0xffffffffu, ok)) {
          failed = true;
          break;
        }
      }
      if (dyn && k < 0) {  // no items left: the consumers leave when they reach this slot
        if (lane == 0) {
          s_first[s] = -1;
          mbar_arrive(&full[s]);
        }
        end_slot = s;
        break;
      }
      const int nr = (int)(rows - r0 < RYG ? rows - r0 : RYG);
      if (lane == 0) {
        if (dyn) s_first[s] = r0;
        // row coordinates for the consumers, published by the arrive below
        for (int yy = 0; yy < nr; ++yy) {
          const int r = (int)(r0 + yy);
          s_row[s * RYG + yy] = make_int2(r % ny, r / ny);
        }
        mbar_arrive_expect_tx(&full[s], (uint32_t)nr * (19u * slot_bytes + (uint32_t)pitch));
      }
      __syncwarp();
      // copy c: row yy = c / 10, part g = c % 10 (9 direction groups, then the class bytes)
      for (int c = lane; c < nr * 10; c += 32) {
        const int yy = c / 10, g = c - yy * 10;
        const long long r = r0 + yy;
        if (g < kGroups) {
          const int2 yz = s_row[s * RYG + yy];
          const long long sr =
              clampi(yz.x - group_cy(g), 0, ny - 1) + (long long)ny * clampi(yz.y - group_cz(g), 0, nz - 1);
          const int first = group_first(g);
          bulk_load(spop + ((size_t)(s * RYG + yy) * 19 + first) * pitch, fs + (sr * 19 + first) * pitch,
                    (uint32_t)group_count(g) * slot_bytes, &full[s]);
        } else {
          bulk_load(scls + (size_t)(s * RYG + yy) * pitch, a.cls + r * pitch, (uint32_t)pitch, &full[s]);
        }
      }
      issued = j + 1;
      if (++s == S_) { s = 0; ph ^= 1u; }
    }
    if (failed && lane == 0) atomicOr(&a.st->error, STEP_ERR_PIPELINE_TIMEOUT);
    // No copy may still be in flight when the CTA exits: wait (bounded, always with the
    // full limit) for the last phase issued into every slot; completed phases return at
    // once.  A slot that took the dynamic deal's end mark after its last fill had that
    // fill consumed already (the producer waited for it), so it is skipped: its mbarrier
    // has completed one more phase than the copies.
    if (lane == 0) {
      for (int k = 0; k < S_ && k < issued; ++k) {
        if (k == end_slot) continue;
        const int last = k + ((issued - 1 - k) / S_) * S_;
        mbar_wait(&full[k], (uint32_t)((last / S_) & 1), kWaitLimit);
      }
    }
  } else if (warp < n_cons) {
    // ---------------- consumer warps ----------------
    const int pslot = (a.step_index + 1) & 1;  // pending rescale of the previous step
    const double corr = a.st->apply[pslot] ? a.st->corr[pslot] : 1.0;
    const float corrf = (float)corr;
    const float2 dec = make_float2(corrf * S::kRawScale, corrf - 1.0f);  // raw-moment decode
    const int ry = warp / wpr;
    const int nchunks = (nx + shift + span * CPT - 1) / (span * CPT);
    int my_nan = 0;
    int s = 0;
    uint32_t ph = 0;
    int seg = warp % wpr;  // the row-end segments rotate over the warps of a row
    long long row0 = item_row0 + ry;  // this warp's row of the item's first group
    UmmaGroup ug{};
    if constexpr (MLP == MLP_TCGEN05) {
      const int g = warp >> 2;
      const uint32_t ab = smem_addr(s_ua + g * (kStepUmmaA1 + kStepUmmaA2)), a2b = ab + (uint32_t)kStepUmmaA1;
      const uint32_t bb = smem_addr(s_ub);
      ug.a1 = s_ua + g * (kStepUmmaA1 + kStepUmmaA2);
      ug.a2 = ug.a1 + kStepUmmaA1;
      ug.dA1 = umma_smem_desc(ab, 128, 256);
      ug.dA2lo = umma_smem_desc(a2b, 128, 512);
      ug.dA2hi = umma_smem_desc(a2b + 256, 128, 512);
      ug.dB1 = umma_smem_desc(bb + kUmmaB1, 128, 256);
      ug.dB2lo = umma_smem_desc(bb + kUmmaB2, 128, 512);
      ug.dB2hi = umma_smem_desc(bb + kUmmaB2 + 256, 128, 512);
      ug.dB3lo = umma_smem_desc(bb + kUmmaB3, 128, 512);
      ug.dB3hi = umma_smem_desc(bb + kUmmaB3 + 256, 128, 512);
      ug.mbar = smem_addr(&s_umbar[g]);
      ug.tmem = *s_utmem + (uint32_t)(g * 64);
      ug.lane_addr = ug.tmem + ((uint32_t)((warp & 3) * 32) << 16);
      ug.row = (warp & 3) * 32 + lane;
      ug.bar_id = 1 + g;
      ug.limit = kWaitLimit;
      ug.issuer = (warp & 3) == 0 && lane == 0;
    }
    for (int j = 0; dyn || j < count; ++j, row0 += item_step) {
      {
        const bool ok = mbar_wait(&full[s], ph, a.wait_limit);
        if constexpr (MLP == MLP_TCGEN05) {
          // the four warps of the group leave together (a failed ring wait or closure)
          if (group_any(ug.bar_id, !__any_sync(0xffffffffu, ok) || ug.failed)) {
            failed = true;
            break;
          }
        } else if (!__any_sync(0xffffffffu, ok)) {
          failed = true;
          break;
        }
      }
      if (dyn) {  // the item the producer took for this slot
        const long long first = s_first[s];
        if (first < 0) break;
        row0 = first + ry;
      }
      for (int gq = 0; gq < G; ++gq) {  // the item's row groups
        const long long row = row0 + (long long)gq * RY;
        const bool row_ok = row < rows;
        int iy = 0, iz = 0;
        if (row_ok) {
          const int2 yz = s_row[s * RYG + gq * RY + ry];
          iy = yz.x;
          iz = yz.y;
        }
        const T* sp = spop + (size_t)(s * RYG + gq * RY + ry) * 19 * pitch;
        const uint8_t* sc = scls + (size_t)(s * RYG + gq * RY + ry) * pitch;
        const bool wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));

        if constexpr (CPT == 2) {
          // two adjacent cells per lane: 64 cells per segment, no row shift (nx even)
          auto inlet = [&](int y) { return make_float2((float)s_uxi[y], (float)s_uyi[y]); };
          for (int c = 0; c < nchunks; ++c) {
            const int cell_lo = c * span * 2 + seg * 64;  // first cell of lane 0
            const int x0 = cell_lo + 2 * lane;
            const bool active = row_ok && x0 < nx;
            const int lx = active ? x0 : 0;  // lanes outside the row read cells 0 and 1
            const uint32_t cls2 = *reinterpret_cast<const uint16_t*>(sc + lx);
            float2 v[19];
            // ---- pull-stream (lbmCpuReference.ts:189-231) from the staged rows: a pair
            // load where the two sources are adjacent and aligned (c_x = 0) ----
#pragma unroll
            for (int d = 0; d < 19; ++d) {
              const T* q = sp + slot_of(d) * pitch + lx;
              if (cx_of(d) == 0) v[d] = load_pair<S>(q);
              else v[d] = make_float2(S::raw(q[-cx_of(d)]), S::raw(q[1 - cx_of(d)]));
            }
            if (gq == G - 1 && c == nchunks - 1) {  // every value of this slot is in registers: release it
              __syncwarp();
              if (lane == 0) mbar_arrive(&empty[s]);
            }
            PairGeom g;
            g.row = row; g.nx = nx; g.ny = ny; g.nz = nz; g.pitch = pitch;
            g.iy = iy; g.iz = iz; g.x0 = x0; g.cell_lo = cell_lo; g.active = active;
            g.has_lo = row_ok && cell_lo == 0;
            g.has_hi = row_ok && cell_lo <= nx - 2 && nx - 2 < cell_lo + 64;
            g.wall_row = wall_row; g.ground_no_slip = a.ground_no_slip; g.write_macro = a.write_macro;
            g.c0 = (uint8_t)(cls2 & 0xffu);
            g.c1 = (uint8_t)(cls2 >> 8);
            pair_segment<S, decltype(inlet), !kHelperEnds>(v, fd, g, (float)a.tau0, (float)a.k_smag, dec, inlet, a,
                                                           s_xo + warp * 24, s_dcw,
                            s_dslot, lane, my_sum, my_nan);
          }
        } else
        for (int c = 0; c < nchunks; ++c) {
          const int cell_lo = c * span + seg * 32 - shift;  // cell of lane 0
          const int ix = cell_lo + lane;
          const bool active = row_ok && ix >= 0 && ix < nx;
          const int lx = (ix >= 0 && ix < nx) ? ix : 1;  // lanes outside the row read cell 1
          const uint8_t cl = sc[lx];
          const int flag = cl & CLS_FLAG_MASK;
          const bool near = (cl & CLS_NEAR) != 0;
          Real v[19];
          // ---- pull-stream (lbmCpuReference.ts:189-231) from the staged rows ----
#pragma unroll
          for (int d = 0; d < 19; ++d) {
            const T raw = sp[slot_of(d) * pitch + lx - cx_of(d)];
            if constexpr (MODE == MODE_FAST) v[d] = S::raw(raw);  // decoded in the moments
            else if constexpr (MODE == MODE_MIRROR) v[d] = (double)(float)(S::f_of(raw, d) * corr);
            else v[d] = S::f_of(raw, d) * corr;
          }
          if (gq == G - 1 && c == nchunks - 1) {  // every value of this slot is in registers: release it
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
          }

          if constexpr (MODE == MODE_FAST) {
            SegGeom g;
            g.row = row; g.nx = nx; g.ny = ny; g.nz = nz; g.pitch = pitch;
            g.iy = iy; g.iz = iz; g.cell_lo = cell_lo; g.ix = ix; g.flag = flag;
            g.row_ok = row_ok; g.active = active; g.near = near; g.wall_row = wall_row;
            g.ground_no_slip = a.ground_no_slip; g.write_macro = a.write_macro; g.cl = cl;
            auto inlet = [&](int y) { return make_float2((float)s_uxi[y], (float)s_uyi[y]); };
            if constexpr (MLP != MLP_NONE) {
              const MlpRefs mr{s_mfrag, s_mbias, s_mstage + warp * 128, a.mlp_nu0, 0.0f, lane, &ug};
              fast_segment<S, decltype(inlet), MLP>(v, fd, g, (float)a.tau0, (float)a.k_smag, dec, inlet, a,
                                                    s_xo + warp * 24, s_dcw, s_dslot, lane, my_sum, my_nan, &mr);
            } else {
              fast_segment<S>(v, fd, g, (float)a.tau0, (float)a.k_smag, dec, inlet, a, s_xo + warp * 24, s_dcw,
                              s_dslot,
                              lane, my_sum, my_nan);
            }
          } else {
            CellCtx cc;
            cc.row = row; cc.ix = ix; cc.iy = iy; cc.iz = iz; cc.cell_lo = cell_lo; cc.flag = flag;
            cc.active = active; cc.near = near;
            my_sum += general_cells<S, MODE, P>(a, v, cc, s_uxi, s_uyi, &my_nan);
          }
        }
        if (++seg == wpr) seg = 0;
      }
      if (++s == S_) { s = 0; ph ^= 1u; }
    }
    if (__any_sync(0xffffffffu, my_nan) && lane == 0) nan_flag = 1;
    if (failed && lane == 0) atomicOr(&a.st->error, STEP_ERR_PIPELINE_TIMEOUT);
    if constexpr (MLP == MLP_TCGEN05) {
      if (ug.failed && lane == 0) atomicOr(&a.st->error, STEP_ERR_PIPELINE_TIMEOUT);
      // no tensor-core operation may still be running when the TMEM is freed: the
      // issuing thread waits (full bound) for its last commit
      if (ug.issuer && ug.issued > 0) umma_mbar_wait(ug.mbar, (uint32_t)((ug.issued - 1) & 1), kWaitLimit);
    }
  }

#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_sum += __shfl_down_sync(0xffffffffu, my_sum, o);
  if (lane == 0) red[warp] = my_sum;
  if constexpr (MLP == MLP_TCGEN05) tc_fence_before();
  __syncthreads();
  if constexpr (MLP == MLP_TCGEN05) {
    tc_fence_after();
    if (warp == 0) tmem_dealloc(*s_utmem, kStepUmmaTmemCols);
  }
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
    a.st->next_item[slot ^ 1] = 0u;
  }
}

// ---------------------------------------------------------------------------
// Momentum exchange, forceIntegrator.ts:159-216, FP64 accumulation.
// One warp per boundary cell, lane l = link d = l + 1 (all 18 links' loads in flight
// together), grid-stride over the cells; per-cell sums by a fixed shuffle tree, then
// a deterministic tree across cells (warps -> CTA -> last CTA in block order).
// ---------------------------------------------------------------------------
template <class S, int MODE>
__global__ void __launch_bounds__(256) forces_kernel(const ForceArgs a) {
  using T = typename S::T;
  __shared__ double red[8][8];
  __shared__ bool is_last;
  // launched as a programmatic dependent of the step kernel in a frame: wait for the step
  // to complete before reading its populations (a no-op after an ordinary launch), and let
  // the slice kernel that follows start its launch
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const T* __restrict__ f = static_cast<const T*>(a.f);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int apply = a.prev_slot >= 0 ? a.st->apply[a.prev_slot] : 0;
  const double corr = apply ? a.st->corr[a.prev_slot] : 1.0;
  auto pop = [&](int d, long long row, int x) -> double {
    const double v = S::f_of(f[a.L.at_row(d, row, x)], d);
    if constexpr (MODE == MODE_MIRROR) return (double)(float)(v * corr);
    else return v * corr;
  };
  // this lane's link: direction d, its lattice vector and opposite
  const int d = lane + 1;
  int cx = 0, cy = 0, cz = 0, od = 0;
  double w2 = 0.0;
#pragma unroll
  for (int e = 1; e < 19; ++e)
    if (e == d) {
      cx = cx_of(e); cy = cy_of(e); cz = cz_of(e); od = opp_of(e); w2 = 2.0 * w32_of(e);
    }
  const int nx = a.L.nx, ny = a.L.ny, nz = a.L.nz;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long b = (long long)blockIdx.x * (blockDim.x >> 5) + warp; b < a.B; b += warps) {
    const int ci = a.bcells[b];  // cell indices are int32 in the voxel grid
    const int row = ci / nx;      // iy + ny * iz
    const int ix = ci - row * nx;
    const int iz = row / ny;
    const int iy = row - iz * ny;
    double cfx = 0.0, cfy = 0.0, cfz = 0.0, cut = 0.0;
    if (lane < 18) {
      const double qv = (double)a.q[b * 18 + lane];
      if (qv > 0.0) {
        const double fo = pop(d, row, ix);
        const int ax = clampi(ix - cx, 0, nx - 1);  // cell + c_opp(d)
        const int ay = clampi(iy - cy, 0, ny - 1);
        const int az = clampi(iz - cz, 0, nz - 1);
        const long long frow = ay + (long long)ny * az;
        double fi = fo;
        if ((a.cls[a.L.cls_at_row(frow, ax)] & CLS_FLAG_MASK) != 1) {
          if (qv < 0.5) {
            const double fon = pop(d, frow, ax);
            fi = 2.0 * qv * fo + (1.0 - 2.0 * qv) * fon;
          } else {
            const double fic = pop(od, row, ix);
            const double inv2q = 1.0 / (2.0 * qv);
            fi = inv2q * fo + (1.0 - inv2q) * fic;
          }
        }
        const double mom = fo + fi - w2;
        cfx = (double)cx * mom;
        cfy = (double)cy * mom;
        cfz = (double)cz * mom;
        cut = d <= 6 ? 1.0 : 0.0;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cfx += __shfl_down_sync(0xffffffffu, cfx, o);
      cfy += __shfl_down_sync(0xffffffffu, cfy, o);
      cfz += __shfl_down_sync(0xffffffffu, cfz, o);
      cut += __shfl_down_sync(0xffffffffu, cut, o);
    }
    if (lane == 0) {
      const double rx = (ix + 0.5) - 0.5 * nx;
      const double ry = (iy + 0.5) - 0.5 * ny;
      const double rz = (iz + 0.5) - 0.5 * nz;
      acc[0] += cfx; acc[1] += cfy; acc[2] += cfz;
      acc[3] += ry * cfz - rz * cfy;
      acc[4] += rz * cfx - rx * cfz;
      acc[5] += rx * cfy - ry * cfx;
      acc[6] += cut;
    }
  }
#pragma unroll
  for (int k = 0; k < 7; ++k)
    if (lane == 0) red[warp][k] = acc[k];
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
    // every thread adds a fixed stride of the CTAs' partials (its loads in flight
    // together), then shuffle trees and the warps in order: a fixed order, so the total
    // does not depend on which CTA finished last
    __threadfence();
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (unsigned int blk = threadIdx.x; blk < gridDim.x; blk += blockDim.x) {
#pragma unroll
      for (int k = 0; k < 7; ++k) s[k] += __ldcg(&a.partials[(long long)blk * 8 + k]);
    }
#pragma unroll
    for (int k = 0; k < 7; ++k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_down_sync(0xffffffffu, s[k], o);
      if (lane == 0) red[warp][k] = s[k];
    }
    __syncthreads();
    if (threadIdx.x < 7) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
      a.out[threadIdx.x] = t;
    }
    if (threadIdx.x == 0) {
      a.out[7] = (double)gridDim.x;
      if (a.err_out) *a.err_out = a.st->error;
      *a.ticket = 0u;
    }
  }
}

}  // namespace aerosim
