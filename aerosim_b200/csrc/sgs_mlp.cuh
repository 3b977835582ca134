// Learned subgrid-scale closure: a per-cell MLP that predicts the eddy viscosity.
//
//   inputs  x[8]  = 100 * S_ab (6 strain-rate components xx yy zz xy xz yz, estimated
//                   from the non-equilibrium stress), 100 * (rho - 1), wall distance / 16
//   hidden  h1 = GELU(W1 x + b1)  (32),  h2 = GELU(W2 h1 + b2)  (32)
//   output  nu_t / nu_0 = softplus(W3 h2 + b3)
//
// GELU is the tanh form 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))) (Hendrycks &
// Gimpel, 2016).  Parameters (FP32 master copy, this order): W1[32][8], b1[32],
// W2[32][32], b2[32], W3[32], b3.  In the step kernel the weights are BF16 and the
// products accumulate in FP32 on the tensor cores.
#pragma once
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace aerosim {

constexpr int kMlpIn = 8, kMlpHidden = 32;
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpHidden * kMlpIn, kMlpW2 = kMlpB1 + kMlpHidden,
              kMlpB2 = kMlpW2 + kMlpHidden * kMlpHidden, kMlpW3 = kMlpB2 + kMlpHidden, kMlpB3 = kMlpW3 + kMlpHidden,
              kMlpParams = kMlpB3 + 1;
constexpr float kGeluK = 0.7978845608028654f;  // sqrt(2 / pi)

__host__ __device__ inline float gelu_f(float x) {
  return 0.5f * x * (1.0f + tanhf(kGeluK * (x + 0.044715f * x * x * x)));
}
__host__ __device__ inline float gelu_grad(float x) {
  const float t = tanhf(kGeluK * (x + 0.044715f * x * x * x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluK * (1.0f + 3.0f * 0.044715f * x * x);
}
__host__ __device__ inline float softplus_f(float o) { return o > 20.0f ? o : log1pf(expf(o)); }
__host__ __device__ inline float sigmoid_f(float o) { return 1.0f / (1.0f + expf(-o)); }

// Model inputs of a cell from its non-equilibrium stress: the strain-rate estimate
// S = -3 Pi^neq / (2 rho tau) with tau the Smagorinsky relaxation time the reference
// computes from |Pi^neq| (lbmCpuReference.ts:264-282), so the closure sees the same
// strain-rate field a box-filtered fine-grid run provides for training.
__host__ __device__ inline void mlp_features(float pxx, float pyy, float pzz, float pxy, float pxz, float pyz,
                                             float rho, float tau_s, float wall_dist, float (&x)[kMlpIn]) {
  const float k = -150.0f / (rho * tau_s);  // 100 * (-3 / (2 rho tau))
  x[0] = k * pxx; x[1] = k * pyy; x[2] = k * pzz;
  x[3] = k * pxy; x[4] = k * pxz; x[5] = k * pyz;
  x[6] = 100.0f * (rho - 1.0f);
  x[7] = wall_dist * (1.0f / 16.0f);
}

// ---- in-kernel inference on the tensor cores ---------------------------------------
// A warp evaluates the MLP for its 32 cells (lane = cell) as BF16 m16n8k16 tile
// contractions with FP32 accumulation: two 16-cell M tiles, hidden width 32 = four
// N tiles, the 8 inputs padded to K = 16.  The D fragments of a layer are, pair by
// pair, the A fragments of the next, so activations never leave the registers.
//
// Weight fragments are pre-packed per lane (mlp_pack_fragments): word w of lane l at
// frag[w * 32 + l] (a warp's load of one word touches 32 consecutive words):
//   w 0..3        layer 1, N tile t:       (W1[n][k], W1[n][k+1]),  n = 8t + l/4, k = 2(l%4)
//   w 4..19       layer 2, (kt, t, half):  (W2[n][k], W2[n][k+1]),  k = 16kt + 2(l%4) + 8 half
//   w 20..23      layer 3, (kt, half):     (W3[k], W3[k+1]) for l/4 == 0, else 0
// Biases: bias[0..31] = b1, bias[32..63] = b2, bias[64] = b3.
constexpr int kMlpFragWords = 24;
constexpr int kMlpBias = 65;

__host__ inline uint16_t bf16_bits_rn(float f) {  // round to nearest even
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

__host__ inline void mlp_pack_fragments(const float* P, uint32_t* frag /*[24 * 32]*/, float* bias /*[65]*/) {
  auto pair = [](float lo, float hi) { return (uint32_t)bf16_bits_rn(lo) | ((uint32_t)bf16_bits_rn(hi) << 16); };
  for (int l = 0; l < 32; ++l) {
    const int k0 = 2 * (l % 4), n0 = l / 4;
    for (int t = 0; t < 4; ++t) {
      const int n = 8 * t + n0;
      frag[t * 32 + l] = pair(P[kMlpW1 + n * kMlpIn + k0], P[kMlpW1 + n * kMlpIn + k0 + 1]);
    }
    for (int kt = 0; kt < 2; ++kt)
      for (int t = 0; t < 4; ++t)
        for (int h = 0; h < 2; ++h) {
          const int n = 8 * t + n0, k = 16 * kt + k0 + 8 * h;
          frag[(4 + (kt * 4 + t) * 2 + h) * 32 + l] =
              pair(P[kMlpW2 + n * kMlpHidden + k], P[kMlpW2 + n * kMlpHidden + k + 1]);
        }
    for (int kt = 0; kt < 2; ++kt)
      for (int h = 0; h < 2; ++h) {
        const int k = 16 * kt + k0 + 8 * h;
        frag[(20 + kt * 2 + h) * 32 + l] = n0 == 0 ? pair(P[kMlpW3 + k], P[kMlpW3 + k + 1]) : 0u;
      }
  }
  for (int j = 0; j < 32; ++j) {
    bias[j] = P[kMlpB1 + j];
    bias[32 + j] = P[kMlpB2 + j];
  }
  bias[64] = P[kMlpB3];
}

#ifdef __CUDACC__
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t bf16x2_of(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
// GELU of two pre-activations as one packed BF16 pair, the operand type of the next
// layer: the pair is rounded to BF16 first and the tanh form is evaluated in bf16x2
// arithmetic (x/2 (1 + tanh(x (k + k c x^2))), k = sqrt(2/pi) and k c = k * 0.044715 as
// BF16 constants 0x3f4c and 0x3d12), about a third of the instructions of two FP32 GELUs.
__device__ __forceinline__ uint32_t gelu_bf16x2(float a, float b) {
  const uint32_t x = bf16x2_of(a, b);
  uint32_t x2, u, t, r;
  asm("mul.rn.bf16x2 %0, %1, %1;" : "=r"(x2) : "r"(x));
  asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(u) : "r"(x2), "r"(0x3d123d12u), "r"(0x3f4c3f4cu));
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(u) : "r"(u), "r"(x));
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(u));
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(u) : "r"(x), "r"(0x3f003f00u));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(r) : "r"(u), "r"(t));
  return r;
}

// nu_t / nu_0 of this lane's cell.  All 32 lanes must call it together.  x: the lane's
// 8 inputs; frag / bias: the packed weights (shared memory); stage: 32 x 8 BF16 of
// shared memory owned by the warp.
__device__ __forceinline__ float mlp_nut_warp(const float (&x)[kMlpIn], const uint32_t* __restrict__ frag,
                                              const float* __restrict__ bias, uint32_t* __restrict__ stage,
                                              int lane) {
  // inputs to the A-fragment layout through shared memory (row = cell, 4 words each)
#pragma unroll
  for (int i = 0; i < 4; ++i) stage[lane * 4 + i] = bf16x2_of(x[2 * i], x[2 * i + 1]);
  __syncwarp();
  const int r = lane >> 2, q = lane & 3;
  uint32_t a1[2][2];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    a1[mt][0] = stage[(16 * mt + r) * 4 + q];
    a1[mt][1] = stage[(16 * mt + r + 8) * 4 + q];
  }
  __syncwarp();
  // layer 1: 8 (padded to 16) -> 32
  float h[2][4][4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const uint32_t b = frag[t * 32 + lane];
    const float c0 = bias[8 * t + 2 * q], c1 = bias[8 * t + 2 * q + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      h[mt][t][0] = c0; h[mt][t][1] = c1; h[mt][t][2] = c0; h[mt][t][3] = c1;
      mma_bf16_16816(h[mt][t], a1[mt][0], a1[mt][1], 0u, 0u, b, 0u);
    }
  }
  uint32_t a2[2][2][4];  // [mt][kt][reg]
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
      const float* lo = h[mt][2 * kt];
      const float* hi = h[mt][2 * kt + 1];
      a2[mt][kt][0] = gelu_bf16x2(lo[0], lo[1]);
      a2[mt][kt][1] = gelu_bf16x2(lo[2], lo[3]);
      a2[mt][kt][2] = gelu_bf16x2(hi[0], hi[1]);
      a2[mt][kt][3] = gelu_bf16x2(hi[2], hi[3]);
    }
  // layer 2: 32 -> 32
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const float c0 = bias[32 + 8 * t + 2 * q], c1 = bias[32 + 8 * t + 2 * q + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      h[mt][t][0] = c0; h[mt][t][1] = c1; h[mt][t][2] = c0; h[mt][t][3] = c1;
    }
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
      const uint32_t b0 = frag[(4 + (kt * 4 + t) * 2) * 32 + lane];
      const uint32_t b1 = frag[(5 + (kt * 4 + t) * 2) * 32 + lane];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
        mma_bf16_16816(h[mt][t], a2[mt][kt][0], a2[mt][kt][1], a2[mt][kt][2], a2[mt][kt][3], b0, b1);
    }
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
      const float* lo = h[mt][2 * kt];
      const float* hi = h[mt][2 * kt + 1];
      a2[mt][kt][0] = gelu_bf16x2(lo[0], lo[1]);
      a2[mt][kt][1] = gelu_bf16x2(lo[2], lo[3]);
      a2[mt][kt][2] = gelu_bf16x2(hi[0], hi[1]);
      a2[mt][kt][3] = gelu_bf16x2(hi[2], hi[3]);
    }
  // layer 3: 32 -> 1 (N padded to 8; column 0 is the output)
  float o[2][4];
  const float c3 = q == 0 ? bias[64] : 0.0f;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    o[mt][0] = c3; o[mt][1] = 0.0f; o[mt][2] = c3; o[mt][3] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 2; ++kt)
      mma_bf16_16816(o[mt], a2[mt][kt][0], a2[mt][kt][1], a2[mt][kt][2], a2[mt][kt][3],
                     frag[(20 + kt * 2) * 32 + lane], frag[(21 + kt * 2) * 32 + lane]);
  }
  // cell i's output sits in lane 4 (i % 8): o[i / 16][0] for i % 16 < 8, else o[i / 16][2]
  const int src = 4 * (lane & 7);
  const float v00 = __shfl_sync(0xffffffffu, o[0][0], src), v02 = __shfl_sync(0xffffffffu, o[0][2], src);
  const float v10 = __shfl_sync(0xffffffffu, o[1][0], src), v12 = __shfl_sync(0xffffffffu, o[1][2], src);
  const float out = lane < 16 ? (lane < 8 ? v00 : v02) : (lane < 24 ? v10 : v12);
  return softplus_f(out);
}
#endif

}  // namespace aerosim
