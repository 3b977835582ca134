// The regularized collision of collide_fast for two cells at once, on packed FP32
// pairs: Blackwell's f32x2 add / mul / fma (sm_100) evaluate both cells in one
// instruction, so a thread that owns two adjacent cells of an x-row issues about half
// the floating-point instructions per cell.  Clamps, comparisons and the approximate
// reciprocal and square roots stay per component.  Same operations and order as
// collide_fast (lbm_kernels.cuh), so each component rounds exactly as collide_fast would
// for that cell, up to the compiler's FMA contraction.
#pragma once
#include "common.cuh"

namespace aerosim {

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
__device__ __forceinline__ float2 f2neg(float2 a) { return make_float2(-a.x, -a.y); }

__device__ __forceinline__ float rcp_approx_(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqrt_approx_(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// c_d . u of a pair with the zero components left out (d is a constant after unrolling).
__device__ __forceinline__ float2 dotc2(int d, float2 x, float2 y, float2 z) {
  const int a = cx_of(d), b = cy_of(d), c = cz_of(d);
  float2 s = a ? (a > 0 ? x : f2neg(x)) : (b ? (b > 0 ? y : f2neg(y)) : (c ? (c > 0 ? z : f2neg(z)) : f2(0.0f)));
  if (a && b) s = b > 0 ? f2add(s, y) : f2sub(s, y);
  if ((a || b) && c) s = c > 0 ? f2add(s, z) : f2sub(s, z);
  return s;
}

// Equilibrium of a pair in the storage domain, OS (feq_d - w_d) + OW w_d, with
// feq_d - w_d = w_d ((rho - 1) - 1.5 rho u^2 + rho (cu + cu^2 / 2)), cu = 3 c_d . u.
template <class S>
__device__ __forceinline__ void heq_pair(float2 (&v)[19], float2 r, float2 ux, float2 uy, float2 uz) {
  constexpr float OS = S::kOutScale, OW = S::kOutW;
  const float2 u2 = f2fma(ux, ux, f2fma(uy, uy, f2mul(uz, uz)));
  const float2 A = f2fma(f2mul(f2(-1.5f), r), u2, f2sub(r, f2(1.0f)));
#pragma unroll
  for (int d = 0; d < 19; ++d) {
    const float2 cu = f2mul(f2(3.0f), dotc2(d, ux, uy, uz));
    const float2 h = f2fma(r, f2fma(f2mul(f2(0.5f), cu), cu, cu), A);
    v[d] = f2fma(f2(OS * wf_of(d)), h, f2(OW * wf_of(d)));
  }
}

// h: the raw stored values of the two cells (x: first cell, y: second), replaced by the
// post-collision values in the storage domain; r, u: the clamped, Mach-limited moments.
// dec = (storage scale x pending rescale, rescale - 1) as in collide_fast.
template <class S>
__device__ __forceinline__ void collide_fast2(float2 (&h)[19], float2& r, float2& ux, float2& uy, float2& uz,
                                              float tau0, float k_smag, float2 dec) {
  static_assert(S::kRawMoments, "the FP32 collision runs on stored deviations");
  constexpr float OS = S::kOutScale, OW = S::kOutW;
  constexpr float w0 = 1.0f / 3.0f, w1 = 1.0f / 18.0f, w2 = 1.0f / 36.0f;
  float2 s[9], t[9];
#pragma unroll
  for (int p = 0; p < 9; ++p) {
    s[p] = f2add(h[2 * p + 1], h[2 * p + 2]);
    t[p] = f2sub(h[2 * p + 1], h[2 * p + 2]);
  }
  float2 dr = f2add(h[0], f2add(f2add(f2add(s[0], s[1]), f2add(s[2], s[3])),
                                f2add(f2add(f2add(s[4], s[5]), f2add(s[6], s[7])), s[8])));
  float2 jx = f2add(f2add(f2add(t[0], t[3]), f2add(t[4], t[5])), t[6]);
  float2 jy = f2add(f2sub(f2add(t[1], t[3]), t[4]), f2add(t[7], t[8]));
  float2 jz = f2add(f2sub(f2add(t[2], t[5]), t[6]), f2sub(t[7], t[8]));
  float2 sxx = f2add(f2add(f2add(s[0], s[3]), f2add(s[4], s[5])), s[6]);
  float2 syy = f2add(f2add(f2add(s[1], s[3]), f2add(s[4], s[7])), s[8]);
  float2 szz = f2add(f2add(f2add(s[2], s[5]), f2add(s[6], s[7])), s[8]);
  float2 sxy = f2sub(s[3], s[4]), sxz = f2sub(s[5], s[6]), syz = f2sub(s[7], s[8]);
  {
    const float2 dx = f2(dec.x), cw3 = f2(dec.y * (1.0f / 3.0f));
    dr = f2fma(dr, dx, f2(dec.y));
    jx = f2mul(jx, dx); jy = f2mul(jy, dx); jz = f2mul(jz, dx);
    sxx = f2fma(sxx, dx, cw3); syy = f2fma(syy, dx, cw3); szz = f2fma(szz, dx, cw3);
    sxy = f2mul(sxy, dx); sxz = f2mul(sxz, dx); syz = f2mul(syz, dx);
  }
  r.x = fmaxf(0.5f, fminf(1.8f, 1.0f + dr.x));
  r.y = fmaxf(0.5f, fminf(1.8f, 1.0f + dr.y));
  if (dr.x != dr.x) r.x = dr.x;  // keep NaN visible like Math.min / Math.max
  if (dr.y != dr.y) r.y = dr.y;
  const float2 ir = make_float2(rcp_approx_(r.x), rcp_approx_(r.y));
  ux = f2mul(jx, ir); uy = f2mul(jy, ir); uz = f2mul(jz, ir);
  {
    const float2 u2 = f2fma(ux, ux, f2fma(uy, uy, f2mul(uz, uz)));
    // Mach limiter |u| <= 0.22: a factor of exactly 1 leaves the other cell unchanged
    const float2 sc = make_float2(u2.x > 0.0484f ? 0.22f * rsqrtf(u2.x) : 1.0f,
                                  u2.y > 0.0484f ? 0.22f * rsqrtf(u2.y) : 1.0f);
    ux = f2mul(ux, sc); uy = f2mul(uy, sc); uz = f2mul(uz, sc);
  }
  const float2 drc = f2sub(r, f2(1.0f));
  const float2 d3 = f2mul(drc, f2(1.0f / 3.0f));
  const float2 jcx = f2mul(r, ux), jcy = f2mul(r, uy), jcz = f2mul(r, uz);
  const float2 dxx = f2sub(sxx, d3), dyy = f2sub(syy, d3), dzz = f2sub(szz, d3);
  const float2 pxx = f2fma(f2neg(jcx), ux, dxx), pyy = f2fma(f2neg(jcy), uy, dyy), pzz = f2fma(f2neg(jcz), uz, dzz);
  const float2 pxy = f2fma(f2neg(jcx), uy, sxy), pxz = f2fma(f2neg(jcx), uz, sxz), pyz = f2fma(f2neg(jcy), uz, syz);
  const float2 off = f2fma(pxy, pxy, f2fma(pxz, pxz, f2mul(pyz, pyz)));
  const float2 pq = f2fma(pxx, pxx, f2fma(pyy, pyy, f2fma(pzz, pzz, f2mul(f2(2.0f), off))));
  const float2 pn = make_float2(sqrt_approx_(pq.x), sqrt_approx_(pq.y));
  const float2 arg = f2fma(f2(tau0), f2(tau0), f2mul(f2mul(f2(k_smag), pn), ir));
  const float2 tau = f2mul(f2(0.5f), f2add(f2(tau0), make_float2(sqrt_approx_(arg.x), sqrt_approx_(arg.y))));
  const float2 om = make_float2(rcp_approx_(fmaxf(0.5015f, fminf(1.95f, tau.x))),
                                rcp_approx_(fmaxf(0.5015f, fminf(1.95f, tau.y))));
  const float2 nom = f2neg(om);
  const float2 xxx = f2fma(nom, pxx, dxx), xyy = f2fma(nom, pyy, dyy), xzz = f2fma(nom, pzz, dzz);
  const float2 xxy = f2fma(nom, pxy, sxy), xxz = f2fma(nom, pxz, sxz), xyz = f2fma(nom, pyz, syz);
  const float2 B = f2fma(f2(-1.5f), f2add(f2add(xxx, xyy), xzz), drc);
  const float2 b = OW == 0.0f ? f2mul(f2(OS), B) : f2fma(f2(OS), B, f2(OW));
  h[0] = f2mul(f2(w0), b);
  const float2 b1 = f2mul(f2(w1), b);
  constexpr float kf = OS * 4.5f * w1, of = OS * 3.0f * w1;
  {
    const float2 E = f2fma(f2(kf), xxx, b1), O = f2mul(f2(of), jcx);
    h[1] = f2add(E, O); h[2] = f2sub(E, O);
  }
  {
    const float2 E = f2fma(f2(kf), xyy, b1), O = f2mul(f2(of), jcy);
    h[3] = f2add(E, O); h[4] = f2sub(E, O);
  }
  {
    const float2 E = f2fma(f2(kf), xzz, b1), O = f2mul(f2(of), jcz);
    h[5] = f2add(E, O); h[6] = f2sub(E, O);
  }
  const float2 b2 = f2mul(f2(w2), b);
  constexpr float ke = OS * 4.5f * w2, ke2 = OS * 9.0f * w2, oe = OS * 3.0f * w2;
  const float2 qx = f2mul(f2(oe), jcx), qy = f2mul(f2(oe), jcy), qz = f2mul(f2(oe), jcz);
  {
    const float2 base = f2fma(f2(ke), f2add(xxx, xyy), b2);
    const float2 Ep = f2fma(f2(ke2), xxy, base), Em = f2fma(f2(-ke2), xxy, base);
    const float2 Op = f2add(qx, qy), Om = f2sub(qx, qy);
    h[7] = f2add(Ep, Op); h[8] = f2sub(Ep, Op); h[9] = f2add(Em, Om); h[10] = f2sub(Em, Om);
  }
  {
    const float2 base = f2fma(f2(ke), f2add(xxx, xzz), b2);
    const float2 Ep = f2fma(f2(ke2), xxz, base), Em = f2fma(f2(-ke2), xxz, base);
    const float2 Op = f2add(qx, qz), Om = f2sub(qx, qz);
    h[11] = f2add(Ep, Op); h[12] = f2sub(Ep, Op); h[13] = f2add(Em, Om); h[14] = f2sub(Em, Om);
  }
  {
    const float2 base = f2fma(f2(ke), f2add(xyy, xzz), b2);
    const float2 Ep = f2fma(f2(ke2), xyz, base), Em = f2fma(f2(-ke2), xyz, base);
    const float2 Op = f2add(qy, qz), Om = f2sub(qy, qz);
    h[15] = f2add(Ep, Op); h[16] = f2sub(Ep, Op); h[17] = f2add(Em, Om); h[18] = f2sub(Em, Om);
  }
}

}  // namespace aerosim
