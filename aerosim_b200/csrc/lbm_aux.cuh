// Solver support kernels: equilibrium initialisation, cell classes, population and
// macro readback with the pending mean-density rescale, mass statistics.
#pragma once
#include "common.cuh"
#include "lbm_kernels.cuh"

namespace aerosim {

// Cell classes from the reference flags: CLS_NEAR marks non-solid cells for which
// some clamped pull source clamp(x - c_d), d >= 1, is SOLID (lbmCpuReference.ts:190-196).
__global__ void classify_kernel(const uint8_t* __restrict__ flags, uint8_t* __restrict__ cls,
                                const Layout L) {
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const long long N = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const uint8_t f = flags[i];
    uint8_t c = f & CLS_FLAG_MASK;
    if (f != CELL_SOLID) {
      const int ix = (int)(i % nx);
      const long long r = i / nx;
      const int iy = (int)(r % ny), iz = (int)(r / ny);
      bool near = false;
#pragma unroll
      for (int d = 1; d < 19; ++d) {
        const int sx = clampi(ix - cx_of(d), 0, nx - 1);
        const int sy = clampi(iy - cy_of(d), 0, ny - 1);
        const int sz = clampi(iz - cz_of(d), 0, nz - 1);
        if (flags[sx + (long long)nx * (sy + (long long)ny * sz)] == CELL_SOLID) near = true;
      }
      if (near) c |= CLS_NEAR;
    }
    cls[L.cls_at(i)] = c;
  }
}

// resetEquilibrium, lbmCpuReference.ts:114-143: feq(1, (u0, 0, 0)) with u0 the
// inlet speed (ABL profile when groundNoSlip, 0 at iy = 0) and 0 inside solids.
template <class S>
__global__ void init_kernel(void* f0, void* f1, const uint8_t* __restrict__ cls, float* mux,
                            float* muy, float* muz, float* mrho, const double* abl, const Layout L,
                            double u_inlet, int ground_no_slip) {
  using T = typename S::T;
  T* a = static_cast<T*>(f0);
  T* b = static_cast<T*>(f1);
  const int nx = L.nx, ny = L.ny;
  const long long N = (long long)nx * ny * L.nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const int iy = (int)((i / nx) % ny);
    double u0 = u_inlet;
    if (ground_no_slip) {
      u0 = u_inlet * abl[iy];
      if (iy == 0) u0 = 0;
    }
    if ((cls[L.cls_at(i)] & CLS_FLAG_MASK) == CELL_SOLID) u0 = 0.0;
    mux[i] = (float)u0; muy[i] = 0.0f; muz[i] = 0.0f; mrho[i] = 1.0f;
#pragma unroll
    for (int d = 0; d < 19; ++d) {
      const T e = S::raw_of_f(feq64(d, 1.0, u0, 0.0, 0.0), d);
      a[L.at(d, i)] = e;
      b[L.at(d, i)] = e;
    }
  }
}

// Populations of the latest step with the pending rescale applied to non-solid
// cells, exactly as the reference's Float32Array holds them after the rescale.
template <class S, int MODE, class Out>
__global__ void read_pops_kernel(const void* f, const uint8_t* __restrict__ cls,
                                 const StepState* st, int prev_slot, const Layout L, long long N,
                                 Out* __restrict__ out) {
  using T = typename S::T;
  const T* src = static_cast<const T*>(f);
  const int apply = prev_slot >= 0 ? st->apply[prev_slot] : 0;
  const double corr = apply ? st->corr[prev_slot] : 1.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const bool solid = (cls[L.cls_at(i)] & CLS_FLAG_MASK) == CELL_SOLID;
#pragma unroll
    for (int d = 0; d < 19; ++d) {
      double v = S::f_of(src[L.at(d, i)], d);
      if (!solid && apply) {
        v = v * corr;
        if constexpr (MODE == MODE_MIRROR) v = (double)(float)v;
      }
      out[d * N + i] = (Out)v;
    }
  }
}

template <class S, class In>
__global__ void write_pops_kernel(void* f, const Layout L, long long N, const In* __restrict__ in) {
  using T = typename S::T;
  T* dst = static_cast<T*>(f);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int d = 0; d < 19; ++d) dst[L.at(d, i)] = S::raw_of_f((double)in[d * N + i], d);
  }
}

// Applies a pending rescale in place (used before the voxel grid changes without a
// flow reset, so the correction is not later applied with the new flags).
template <class S, int MODE>
__global__ void materialize_rescale_kernel(void* f, const uint8_t* __restrict__ cls,
                                           const StepState* st, int prev_slot, const Layout L,
                                           long long N) {
  using T = typename S::T;
  T* dst = static_cast<T*>(f);
  const int apply = prev_slot >= 0 ? st->apply[prev_slot] : 0;
  if (!apply) return;
  const double corr = st->corr[prev_slot];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if ((cls[L.cls_at(i)] & CLS_FLAG_MASK) == CELL_SOLID) continue;
#pragma unroll
    for (int d = 0; d < 19; ++d) dst[L.at(d, i)] = S::raw_of_f(S::f_of(dst[L.at(d, i)], d) * corr, d);
  }
}

// Macro readback with the pending rescale on rho (rho[idx] *= corr, :448).
__global__ void read_macro_kernel(const float* __restrict__ mrho, const uint8_t* __restrict__ cls,
                                  const StepState* st, int prev_slot, const Layout L, long long N,
                                  float* __restrict__ rho_out) {
  const int apply = prev_slot >= 0 ? st->apply[prev_slot] : 0;
  const double corr = apply ? st->corr[prev_slot] : 1.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    float r = mrho[i];
    if (apply && (cls[L.cls_at(i)] & CLS_FLAG_MASK) != CELL_SOLID) r = (float)((double)r * corr);
    rho_out[i] = r;
  }
}

// computeFluidMassStats (lbmCpuReference.ts:461-495) on the rescaled densities: exact
// fixed-point density sum,
// fluid count, max speed (ordered as unsigned bit patterns of non-negative doubles)
// and a NaN flag.  out: [sum_fixed, count, max_speed_bits, nan]
__global__ void mass_stats_kernel(const float* __restrict__ mux, const float* __restrict__ muy,
                                  const float* __restrict__ muz, const float* __restrict__ rho,
                                  const uint8_t* __restrict__ cls, const StepState* st,
                                  int prev_slot, const Layout L, long long N, unsigned long long* out) {
  const int apply = prev_slot >= 0 ? st->apply[prev_slot] : 0;
  const double corr = apply ? st->corr[prev_slot] : 1.0;
  long long s = 0, cnt = 0;
  double mx = 0.0;
  int nan = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    if ((cls[L.cls_at(i)] & CLS_FLAG_MASK) == CELL_SOLID) continue;
    float r = rho[i];
    if (apply) r = (float)((double)r * corr);
    const float u = mux[i], v = muy[i], w = muz[i];
    if (r != r || u != u || v != v || w != w) {
      nan = 1;
      continue;
    }
    s += llrint((double)r * 33554432.0);
    ++cnt;
    const double du = u, dv = v, dw = w;
    const double sp = sqrt(du * du + dv * dv + dw * dw);
    if (sp > mx) mx = sp;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  nan = __any_sync(0xffffffffu, nan);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], (unsigned long long)s);
    atomicAdd(&out[1], (unsigned long long)cnt);
    atomicMax(&out[2], (unsigned long long)__double_as_longlong(mx));
    if (nan) atomicOr(&out[3], 1ull);
  }
}

// ---- slice image: sampleCFDColormap + extractSliceRGBA, lbmCpuReference.ts:23-46, 499-596.
// FP64 in the reference's operation order (this unit is built with -fmad=false), so the
// bytes equal the reference's for the same macro fields.
__device__ __forceinline__ void cfd_colormap(double tv, double (&rgb)[3]) {
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

// axis 0 = x, 1 = y, 2 = z; mode 0 = velocity, 1 = vorticity, 2 = pressure (Cp).  rho is
// read with the pending mean-density rescale applied, as the reference's array holds it.
__global__ void slice_kernel(const float* __restrict__ mux, const float* __restrict__ muy,
                             const float* __restrict__ muz, const float* __restrict__ mrho,
                             const uint8_t* __restrict__ cls, const StepState* st, int prev_slot, const Layout L,
                             int axis, int fixed, int mode, double uref, int width, int height,
                             uint8_t* __restrict__ rgba) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // programmatic dependent of the frame's kernels
  const int apply = prev_slot >= 0 ? st->apply[prev_slot] : 0;
  const double corr = apply ? st->corr[prev_slot] : 1.0;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const long long P = (long long)width * height;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const int u = (int)(p % width), v = (int)(p / width);
    int ix = u, iy = v, iz = fixed;
    if (axis == 1) { ix = u; iy = fixed; iz = v; }
    else if (axis == 0) { ix = fixed; iy = v; iz = u; }
    const long long idx = ix + (long long)nx * (iy + (long long)ny * iz);
    uint8_t* px = rgba + p * 4;
    if ((cls[L.cls_at(idx)] & CLS_FLAG_MASK) == CELL_SOLID) {
      px[0] = px[1] = px[2] = px[3] = 0;
      continue;
    }
    double sn = 0.5, alpha = 215.0;
    if (mode == 0) {
      const double a = mux[idx], b = muy[idx], c = muz[idx];
      const double sp = sqrt(a * a + b * b + c * c);
      sn = js_min(1.0, js_max(0.0, sp / (uref * 1.55)));
    } else if (mode == 1) {
      const int ixP = ix + 1 < nx ? ix + 1 : nx - 1, ixM = ix > 0 ? ix - 1 : 0;
      const int iyP = iy + 1 < ny ? iy + 1 : ny - 1, iyM = iy > 0 ? iy - 1 : 0;
      const int izP = iz + 1 < nz ? iz + 1 : nz - 1, izM = iz > 0 ? iz - 1 : 0;
      auto at = [&](int x, int y, int z) { return x + (long long)nx * (y + (long long)ny * z); };
      const double wx = 0.5 * ((double)muz[at(ix, iyP, iz)] - (double)muz[at(ix, iyM, iz)]) -
                        0.5 * ((double)muy[at(ix, iy, izP)] - (double)muy[at(ix, iy, izM)]);
      const double wy = 0.5 * ((double)mux[at(ix, iy, izP)] - (double)mux[at(ix, iy, izM)]) -
                        0.5 * ((double)muz[at(ixP, iy, iz)] - (double)muz[at(ixM, iy, iz)]);
      const double wz = 0.5 * ((double)muy[at(ixP, iy, iz)] - (double)muy[at(ixM, iy, iz)]) -
                        0.5 * ((double)mux[at(ix, iyP, iz)] - (double)mux[at(ix, iyM, iz)]);
      const double vm = sqrt(wx * wx + wy * wy + wz * wz);
      const double vn = js_min(1.0, vm / (uref * 0.42));
      sn = 0.35 + 0.65 * vn;
      alpha = floor(70.0 + 175.0 * vn + 0.5);
    } else {
      float r = mrho[idx];
      if (apply) r = (float)((double)r * corr);
      const double cp = (((double)r - 1.0) / 3.0) / (0.5 * uref * uref);
      sn = js_min(1.0, js_max(0.0, (cp + 1.1) / 2.1));
    }
    double rgb[3];
    cfd_colormap(sn, rgb);
    px[0] = (uint8_t)(int)floor(rgb[0] * 255.0 + 0.5);
    px[1] = (uint8_t)(int)floor(rgb[1] * 255.0 + 0.5);
    px[2] = (uint8_t)(int)floor(rgb[2] * 255.0 + 0.5);
    px[3] = (uint8_t)(int)alpha;
  }
}

// ---- Q-criterion and vorticity, src/render/vortexIso.ts:22-122: FP64 per cell in the
// reference's operation order (-fmad=false), float outputs, 0 at solid cells (flags may be
// null); the maxima (starting at 1e-6) as the bit patterns of non-negative doubles, so an
// unsigned max is exact and order-free.
__global__ void q_criterion_kernel(int nx, int ny, int nz, double dx, const float* __restrict__ ux,
                                   const float* __restrict__ uy, const float* __restrict__ uz,
                                   const uint8_t* __restrict__ flags, float* __restrict__ q,
                                   float* __restrict__ om, float* __restrict__ omv,
                                   unsigned long long* __restrict__ maxima) {
  const long long N = (long long)nx * ny * nz;
  const double inv2dx = 1.0 / (2.0 * dx);
  double mq = 0.0, mo = 0.0;
  auto at = [&](int x, int y, int z) { return x + (long long)nx * (y + (long long)ny * z); };
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % nx);
    const long long r = i / nx;
    const int iy = (int)(r % ny), iz = (int)(r / ny);
    if (flags && flags[i] == CELL_SOLID) {
      q[i] = 0.0f; om[i] = 0.0f; omv[3 * i] = 0.0f; omv[3 * i + 1] = 0.0f; omv[3 * i + 2] = 0.0f;
      continue;
    }
    const int xp = ix > 0 ? ix - 1 : 0, xn = ix + 1 < nx ? ix + 1 : nx - 1;
    const int yp = iy > 0 ? iy - 1 : 0, yn = iy + 1 < ny ? iy + 1 : ny - 1;
    const int zp = iz > 0 ? iz - 1 : 0, zn = iz + 1 < nz ? iz + 1 : nz - 1;
    const double sx = xn > xp ? 1.0 / ((xn - xp) * dx) : inv2dx;
    const double sy = yn > yp ? 1.0 / ((yn - yp) * dx) : inv2dx;
    const double sz = zn > zp ? 1.0 / ((zn - zp) * dx) : inv2dx;
    const double a = ((double)ux[at(xn, iy, iz)] - (double)ux[at(xp, iy, iz)]) * sx;
    const double b = ((double)ux[at(ix, yn, iz)] - (double)ux[at(ix, yp, iz)]) * sy;
    const double c = ((double)ux[at(ix, iy, zn)] - (double)ux[at(ix, iy, zp)]) * sz;
    const double d = ((double)uy[at(xn, iy, iz)] - (double)uy[at(xp, iy, iz)]) * sx;
    const double e = ((double)uy[at(ix, yn, iz)] - (double)uy[at(ix, yp, iz)]) * sy;
    const double f = ((double)uy[at(ix, iy, zn)] - (double)uy[at(ix, iy, zp)]) * sz;
    const double g = ((double)uz[at(xn, iy, iz)] - (double)uz[at(xp, iy, iz)]) * sx;
    const double h = ((double)uz[at(ix, yn, iz)] - (double)uz[at(ix, yp, iz)]) * sy;
    const double k = ((double)uz[at(ix, iy, zn)] - (double)uz[at(ix, iy, zp)]) * sz;
    const double S12 = 0.5 * (b + d), S13 = 0.5 * (c + g), S23 = 0.5 * (f + h);
    const double nS = a * a + e * e + k * k + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
    const double O12 = 0.5 * (b - d), O13 = 0.5 * (c - g), O23 = 0.5 * (f - h);
    const double nO = 2.0 * (O12 * O12 + O13 * O13 + O23 * O23);
    const double qv = 0.5 * (nO - nS);
    q[i] = (float)qv;
    if (qv > mq) mq = qv;
    const double ox = h - f, oy = c - g, oz = d - b;
    const double m = sqrt(ox * ox + oy * oy + oz * oz);
    omv[3 * i] = (float)ox; omv[3 * i + 1] = (float)oy; omv[3 * i + 2] = (float)oz;
    om[i] = (float)m;
    if (m > mo) mo = m;
  }
  atomicMax(&maxima[0], (unsigned long long)__double_as_longlong(mq));
  atomicMax(&maxima[1], (unsigned long long)__double_as_longlong(mo));
}

}  // namespace aerosim
