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

struct StepArgs {
  const void* fsrc;
  void* fdst;
  const uint8_t* cls;
  const int32_t* bmap;
  const float* q;
  float* mux;
  float* muy;
  float* muz;
  float* mrho;
  const double* abl;      // [ny] Math.min(1.15, 0.35 + 0.8 * yFrac^0.3)
  const double* sin_tab;  // [120 * ny] sin(step * 0.15 + (iy / ny) * PI * 2)
  StepState* st;
  long long stride;       // elements between direction planes (>= N)
  long long fluid_count;  // non-solid cells
  int nx, ny, nz;
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
  long long stride;
  long long B;
  int nx, ny, nz;
  int prev_slot;          // state slot of the step that produced f (-1: none)
};

template <class T>
struct MacroOf { using type = float; };
template <>
struct MacroOf<double> { using type = double; };

// Fixed-point weight of a density in the rescale sum.  A float density in
// [0.25, 2) is an exact multiple of 2^-25; double densities use 2^-36.
__device__ __forceinline__ long long rho_fixed(float r) { return llrint((double)r * 33554432.0); }
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

// FP32 equilibrium deviation feq_d - w_d for the fast path.
__device__ __forceinline__ float heq32(int d, float rho, float ux, float uy, float uz) {
  const float cu = 3.0f * ((float)cx_of(d) * ux + (float)cy_of(d) * uy + (float)cz_of(d) * uz);
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
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    fl[d] = MIRROR ? (double)(float)v[d] : v[d];
    r += v[d];
    ux += (double)cx_of(d) * v[d];
    uy += (double)cy_of(d) * v[d];
    uz += (double)cz_of(d) * v[d];
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
    pxx += cx * cx * fn;
    pyy += cy * cy * fn;
    pzz += cz * cz * fn;
    pxy += cx * cy * fn;
    pxz += cx * cz * fn;
    pyz += cy * cz * fn;
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

// FP32 path.  Works on deviations h_d = f_d - w_d: the moments are
//   rho - 1 = sum h,  j = sum c h,  Pi^neq = sum cc h - (rho - 1)/3 I - rho u u,
// which equals the reference's sum cc (f - feq) but keeps the small quantities
// free of the cancellation against w_d.
__device__ __forceinline__ void collide_f32(float (&h)[19], float& r, float& ux, float& uy,
                                            float& uz, float tau0, float k_smag) {
  float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
  float sxx = 0.f, syy = 0.f, szz = 0.f, sxy = 0.f, sxz = 0.f, syz = 0.f;
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    const float cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
    dr += h[d];
    if (cx_of(d)) jx += cx * h[d];
    if (cy_of(d)) jy += cy * h[d];
    if (cz_of(d)) jz += cz * h[d];
    if (cx_of(d)) sxx += h[d];
    if (cy_of(d)) syy += h[d];
    if (cz_of(d)) szz += h[d];
    if (cx_of(d) * cy_of(d)) sxy += cx * cy * h[d];
    if (cx_of(d) * cz_of(d)) sxz += cx * cz * h[d];
    if (cy_of(d) * cz_of(d)) syz += cy * cz * h[d];
  }
  r = fmaxf(0.5f, fminf(1.8f, 1.0f + dr));
  if (dr != dr) r = dr;  // keep NaN visible like Math.min/Math.max
  const float ir = 1.0f / r;
  ux = jx * ir; uy = jy * ir; uz = jz * ir;
  const float m2 = ux * ux + uy * uy + uz * uz;
  if (m2 > 0.0484f) {
    const float s = 0.22f * rsqrtf(m2);
    ux *= s; uy *= s; uz *= s;
  }
  const float drc = r - 1.0f;
  const float third = 1.0f / 3.0f;
  const float pxx = sxx - drc * third - r * ux * ux;
  const float pyy = syy - drc * third - r * uy * uy;
  const float pzz = szz - drc * third - r * uz * uz;
  const float pxy = sxy - r * ux * uy;
  const float pxz = sxz - r * ux * uz;
  const float pyz = syz - r * uy * uz;
  const float pn = sqrtf(pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * (pxy * pxy + pxz * pxz + pyz * pyz));
  const float tau = 0.5f * (tau0 + sqrtf(tau0 * tau0 + (k_smag * pn) / r));
  const float om = 1.0f / fmaxf(0.5015f, fminf(1.95f, tau));
  const float uSq = ux * ux + uy * uy + uz * uz;
  const float tr3 = (pxx + pyy + pzz) * third;
  const float g = (1.0f - om) * 4.5f;
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    const float cx = cx_of(d), cy = cy_of(d), cz = cz_of(d);
    const float cu = 3.0f * (cx * ux + cy * uy + cz * uz);
    const float heq = wf_of(d) * (drc + r * (cu + 0.5f * cu * cu - 1.5f * uSq));
    const float qpi = cx * cx * pxx + cy * cy * pyy + cz * cz * pzz +
                      2.0f * (cx * cy * pxy + cx * cz * pxz + cy * cz * pyz) - tr3;
    h[d] = heq + g * wf_of(d) * qpi;
  }
}

// ---------------------------------------------------------------------------
// The fused step kernel.  blockDim = (TX, RY): TX threads along x, RY rows per CTA.
// ---------------------------------------------------------------------------
template <int RY>
struct RowExchange {
  double rho1[RY];       // density at ix = 1 (after collision)
  double fprev[RY][19];  // populations at ix = nx-2 before wall conditions
  double mprev[RY][4];   // rho, ux, uy, uz at ix = nx-2 before wall conditions
};

template <class S, int MODE, int RY>
__global__ void __launch_bounds__(256) step_kernel(const StepArgs a) {
  using T = typename S::T;
  using Real = typename std::conditional<MODE == MODE_FAST, float, double>::type;
  using Mac = typename MacroOf<T>::type;
  constexpr bool DBL = MODE != MODE_FAST;

  __shared__ RowExchange<RY> ex;
  __shared__ long long red[32];
  __shared__ bool is_last;

  const T* __restrict__ fs = static_cast<const T*>(a.fsrc);
  T* __restrict__ fd = static_cast<T*>(a.fdst);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long rows = (long long)ny * nz;
  const long long row = (long long)blockIdx.x * RY + ty;
  const bool row_ok = row < rows;
  const int iy = row_ok ? (int)(row % ny) : 0;
  const int iz = row_ok ? (int)(row / ny) : 0;
  const long long stride = a.stride;

  // Pending rescale of the previous step (slot (step-1)&1; cleared at reset).
  const int pslot = (a.step_index + 1) & 1;
  const int apply = a.st->apply[pslot];
  const double corr = apply ? a.st->corr[pslot] : 1.0;
  const float corrf = (float)corr;

  // Clamped source row offsets for the 9 (cy, cz) combinations.
  auto srow = [&](int cy, int cz) -> long long {
    return (long long)nx * (clampi(iy - cy, 0, ny - 1) + (long long)ny * clampi(iz - cz, 0, nz - 1));
  };
  const long long rbase = (long long)nx * (iy + (long long)ny * iz);
  long long rb[19];
#pragma unroll
  for (int d = 0; d < 19; ++d) rb[d] = srow(cy_of(d), cz_of(d));
  const bool wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));

  long long my_sum = 0;
  int my_nan = 0;
  const int nchunks = (nx + blockDim.x - 1) / blockDim.x;
  for (int ch = 0; ch < nchunks; ++ch) {
    const int ix = ch * blockDim.x + tx;
    const bool active = row_ok && ix < nx;
    const long long idx = rbase + ix;
    const uint8_t c = active ? a.cls[idx] : CELL_SOLID;
    const int flag = c & CLS_FLAG_MASK;
    const bool solid = flag == CELL_SOLID;
    const bool xface = (ix == 0 || ix == nx - 1);
    Real v[19];
    Mac mr = (Mac)1, mx = (Mac)0, my = (Mac)0, mz = (Mac)0;

    if (active && !solid && !xface) {
      // ---- pull-stream (lbmCpuReference.ts:189-231) ----
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        const T raw = fs[d * stride + rb[d] + ix - cx_of(d)];
        if constexpr (MODE == MODE_FAST) {
          float h = S::h_of(raw, d);
          if (apply) h = h * corrf + wf_of(d) * (corrf - 1.0f);
          v[d] = h;
        } else if constexpr (MODE == MODE_MIRROR) {
          v[d] = (double)(float)(S::f_of(raw, d) * corr);
        } else {
          v[d] = S::f_of(raw, d) * corr;
        }
      }
      if (c & CLS_NEAR) {
        // Bouzidi interpolated bounce-back for solid pull sources (:196-221).
        const int bi = (flag == CELL_BOUNDARY) ? a.bmap[idx] : -1;
#pragma unroll
        for (int d = 1; d < 19; ++d) {
          const long long src = rb[d] + ix - cx_of(d);
          if ((a.cls[src] & CLS_FLAG_MASK) == CELL_SOLID) {
            const int wd = opp_of(d);
            const double qv = bi >= 0 ? (double)a.q[(long long)bi * 18 + (wd - 1)] : 0.5;
            const double qe = qv > 0.0 ? qv : 0.5;
            auto popf = [&](int dd, long long i) -> double {
              const double f = S::f_of(fs[dd * stride + i], dd);
              if constexpr (MODE == MODE_MIRROR) return (double)(float)(f * corr);
              else return f * corr;
            };
            const double fo = popf(wd, idx);
            const int fxi = clampi(ix + cx_of(d), 0, nx - 1);
            const int fyi = clampi(iy + cy_of(d), 0, ny - 1);
            const int fzi = clampi(iz + cz_of(d), 0, nz - 1);
            const long long ff = fxi + (long long)nx * (fyi + (long long)ny * fzi);
            double val;
            if ((a.cls[ff] & CLS_FLAG_MASK) != CELL_SOLID) {
              if (qe < 0.5) {
                const double fon = popf(wd, ff);
                val = 2.0 * qe * fo + (1.0 - 2.0 * qe) * fon;
              } else {
                const double fic = popf(d, idx);
                const double inv2q = 1.0 / (2.0 * qe);
                val = inv2q * fo + (1.0 - inv2q) * fic;
              }
            } else {
              val = fo;
            }
            if constexpr (MODE == MODE_FAST) v[d] = (float)(val - (double)wf_of(d));
            else v[d] = val;
          }
        }
      }
      // ---- collision (:233-304) ----
      Real r, ux, uy, uz;
      if constexpr (MODE == MODE_FAST) collide_f32(v, r, ux, uy, uz, (float)a.tau0, (float)a.k_smag);
      else collide_f64<MODE == MODE_MIRROR>(v, r, ux, uy, uz, a.tau0, a.k_smag);
      mr = (Mac)r; mx = (Mac)ux; my = (Mac)uy; mz = (Mac)uz;

      if (ix == 1) ex.rho1[ty] = (double)mr;
      if (ix == nx - 2) {
#pragma unroll
        for (int d = 0; d < 19; ++d) {
          // value as the outlet will read it back from fDst
          if constexpr (MODE == MODE_FAST) ex.fprev[ty][d] = (double)v[d];
          else ex.fprev[ty][d] = S::f_of(S::raw_of_f(v[d], d), d);
        }
        ex.mprev[ty][0] = mr; ex.mprev[ty][1] = mx; ex.mprev[ty][2] = my; ex.mprev[ty][3] = mz;
      }
      // ---- wall conditions (:375-429), own-cell moments only ----
      if (wall_row && flag == CELL_FLUID) {
        if (iy == 0) {
          if (a.ground_no_slip) { mx = (Mac)0; mz = (Mac)0; }
          my = (Mac)0;
        }
        if (iy == ny - 1) my = (Mac)0;
        if (nz > 4 && (iz == 0 || iz == nz - 1)) mz = (Mac)0;
#pragma unroll
        for (int d = 0; d < 19; ++d) {
          if constexpr (MODE == MODE_FAST) v[d] = heq32(d, (float)mr, (float)mx, (float)my, (float)mz);
          else v[d] = feq64(d, (double)mr, (double)mx, (double)my, (double)mz);
        }
      }
    } else if (active && solid) {
      // Solid cells: macro (0, 0, 0, 1); populations are never written (:173-179).
      if (ix == 1) ex.rho1[ty] = 1.0;
      if (ix == nx - 2) {
#pragma unroll
        for (int d = 0; d < 19; ++d) ex.fprev[ty][d] = S::f_of(fd[d * stride + idx], d) - (DBL ? 0.0 : (double)wf_of(d));
        ex.mprev[ty][0] = 1.0; ex.mprev[ty][1] = 0.0; ex.mprev[ty][2] = 0.0; ex.mprev[ty][3] = 0.0;
      }
    }
    __syncthreads();
    if (active && !solid && xface) {
      if (ix == 0) {
        // Velocity inlet with density relaxation (:328-352).
        double uxi = a.u_inlet;
        if (a.ground_no_slip) uxi = a.u_inlet * a.abl[iy];
        double uyi = 0.0;
        if (a.step_index < 120) uyi = 0.015 * a.u_inlet * a.sin_tab[(long long)a.step_index * ny + iy];
        if constexpr (MODE == MODE_FAST) {
          const float ri = 0.85f * (float)ex.rho1[ty] + 0.15f;
#pragma unroll
          for (int d = 0; d < 19; ++d) v[d] = heq32(d, ri, (float)uxi, (float)uyi, 0.f);
          mr = (Mac)ri;
        } else {
          const double ri = 0.85 * ex.rho1[ty] + 0.15 * 1.0;
#pragma unroll
          for (int d = 0; d < 19; ++d) v[d] = feq64(d, ri, uxi, uyi, 0.0);
          mr = (Mac)ri;
        }
        mx = (Mac)uxi; my = (Mac)uyi; mz = (Mac)0;
      } else {
        // Convective outlet (:354-371).
        const double rp = ex.mprev[ty][0];
        const double uxo = ex.mprev[ty][1], uyo = ex.mprev[ty][2], uzo = ex.mprev[ty][3];
        if constexpr (MODE == MODE_FAST) {
          const float ro = (float)rp * 0.85f + 0.15f;
#pragma unroll
          for (int d = 0; d < 19; ++d)
            v[d] = 0.75f * (float)ex.fprev[ty][d] + 0.25f * heq32(d, ro, (float)uxo, (float)uyo, (float)uzo);
          mr = (Mac)ro;
        } else {
          const double ro = rp * 0.85 + 1.0 * 0.15;
#pragma unroll
          for (int d = 0; d < 19; ++d)
            v[d] = 0.75 * ex.fprev[ty][d] + 0.25 * feq64(d, ro, uxo, uyo, uzo);
          mr = (Mac)ro;
        }
        mx = (Mac)uxo; my = (Mac)uyo; mz = (Mac)uzo;
      }
    }
    if (active && !solid) {
#pragma unroll
      for (int d = 0; d < 19; ++d) {
        if constexpr (MODE == MODE_FAST) fd[d * stride + idx] = S::raw_of_h(v[d], d);
        else fd[d * stride + idx] = S::raw_of_f(v[d], d);
      }
      if (mr == mr) my_sum += rho_fixed(mr);
      else my_nan = 1;
    }
    if (active && a.write_macro) {
      a.mux[idx] = (float)mx; a.muy[idx] = (float)my; a.muz[idx] = (float)mz; a.mrho[idx] = (float)mr;
    }
    __syncthreads();  // the exchange slots are reused by the next chunk
  }

  // ---- mean-density rescale (:431-455): CTA sum, last CTA finalises ----
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_sum += __shfl_down_sync(0xffffffffu, my_sum, o);
  my_nan = __any_sync(0xffffffffu, my_nan);
  if (lane == 0) red[warp] = my_sum;
  if (lane == 0 && my_nan) a.st->nan_seen = 1;
  __syncthreads();
  const int slot = a.step_index & 1;
  if (warp == 0) {
    long long s = lane < nwarps ? red[lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) {
      atomicAdd(&a.st->rho_sum[slot], (unsigned long long)s);
      __threadfence();
      const unsigned int t = atomicAdd(&a.st->ticket[slot], 1u);
      is_last = (t == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (is_last && threadIdx.x == 0 && threadIdx.y == 0) {
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
    const double v = S::f_of(f[d * a.stride + i], d);
    if constexpr (MODE == MODE_MIRROR) return (double)(float)(v * corr);
    else return v * corr;
  };
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (b < a.B) {
    const long long ci = a.bcells[b];
    const int ix = (int)(ci % a.nx);
    const long long rem = (ci - ix) / a.nx;
    const int iy = (int)(rem % a.ny);
    const int iz = (int)((rem - iy) / a.ny);
    double cfx = 0.0, cfy = 0.0, cfz = 0.0;
    double cut = 0.0;
#pragma unroll
    for (int d = 1; d < 19; ++d) {
      const double qv = (double)a.q[b * 18 + (d - 1)];
      if (qv > 0.0) {
        const int od = opp_of(d);
        const double fo = pop(d, ci);
        const int ax = clampi(ix + cx_of(od), 0, a.nx - 1);
        const int ay = clampi(iy + cy_of(od), 0, a.ny - 1);
        const int az = clampi(iz + cz_of(od), 0, a.nz - 1);
        const long long ff = ax + (long long)a.nx * (ay + (long long)a.ny * az);
        double fi = fo;
        if ((a.cls[ff] & CLS_FLAG_MASK) != 1) {
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
    const double rx = (ix + 0.5) - 0.5 * a.nx;
    const double ry = (iy + 0.5) - 0.5 * a.ny;
    const double rz = (iz + 0.5) - 0.5 * a.nz;
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
