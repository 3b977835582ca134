// Learned SGS closure support: training of the eddy-viscosity MLP on the GPU (forward,
// backward, Adam), its FP32 evaluation, the wall-distance field of a voxel grid (jump
// flooding) and the training samples of a box-filtered fine-grid flow.  No counterpart
// in the reference, whose only closure is Smagorinsky (lbmCpuReference.ts:264-282).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/aerosim.h"
#include "common.cuh"
#include "engine_internal.h"
#include "sgs_mlp.cuh"
#include "sgs_umma.cuh"

namespace aerosim {
namespace {

constexpr int kTrainBlock = 128;

// Forward pass of one sample; keeps the pre-activations for the backward pass.
__device__ __forceinline__ float mlp_forward_keep(const float* P, const float (&x)[kMlpIn], float (&z1)[kMlpHidden],
                                                  float (&z2)[kMlpHidden], float& o) {
  float h1[kMlpHidden];
#pragma unroll
  for (int j = 0; j < kMlpHidden; ++j) {
    float s = P[kMlpB1 + j];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) s = fmaf(P[kMlpW1 + j * kMlpIn + i], x[i], s);
    z1[j] = s;
    h1[j] = gelu_f(s);
  }
  o = P[kMlpB3];
#pragma unroll 4
  for (int j = 0; j < kMlpHidden; ++j) {
    float s = P[kMlpB2 + j];
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) s = fmaf(P[kMlpW2 + j * kMlpHidden + i], h1[i], s);
    z2[j] = s;
    o = fmaf(P[kMlpW3 + j], gelu_f(s), o);
  }
  return softplus_f(o);
}

// Loss and gradient of the mean squared error (prediction - target)^2 over n samples
// (rows of X, or the rows listed in idx), accumulated into G and *loss.
__global__ void __launch_bounds__(kTrainBlock) mlp_grad_kernel(const float* __restrict__ Pg, const float* __restrict__ X,
                                                               const float* __restrict__ Y,
                                                               const long long* __restrict__ idx, long long n,
                                                               float inv_n, float* __restrict__ G,
                                                               double* __restrict__ loss) {
  __shared__ float P[kMlpParams];
  __shared__ float sG[kMlpParams];
  for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) {
    P[p] = Pg[p];
    sG[p] = 0.0f;
  }
  __syncthreads();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (t < n) {
    const long long r = idx ? idx[t] : t;
    float x[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) x[i] = X[r * kMlpIn + i];
    float z1[kMlpHidden], z2[kMlpHidden], o;
    const float pred = mlp_forward_keep(P, x, z1, z2, o);
    const float e = pred - Y[r];
    l = (double)e * e;
    const float d_o = 2.0f * e * sigmoid_f(o) * inv_n;
    atomicAdd(&sG[kMlpB3], d_o);
    float d1[kMlpHidden];
#pragma unroll
    for (int k = 0; k < kMlpHidden; ++k) d1[k] = 0.0f;
    for (int j = 0; j < kMlpHidden; ++j) {
      const float h2 = gelu_f(z2[j]);
      atomicAdd(&sG[kMlpW3 + j], d_o * h2);
      const float d2 = d_o * P[kMlpW3 + j] * gelu_grad(z2[j]);
      atomicAdd(&sG[kMlpB2 + j], d2);
#pragma unroll
      for (int k = 0; k < kMlpHidden; ++k) {
        atomicAdd(&sG[kMlpW2 + j * kMlpHidden + k], d2 * gelu_f(z1[k]));
        d1[k] = fmaf(d2, P[kMlpW2 + j * kMlpHidden + k], d1[k]);
      }
    }
    for (int k = 0; k < kMlpHidden; ++k) {
      const float dk = d1[k] * gelu_grad(z1[k]);
      atomicAdd(&sG[kMlpB1 + k], dk);
#pragma unroll
      for (int i = 0; i < kMlpIn; ++i) atomicAdd(&sG[kMlpW1 + k * kMlpIn + i], dk * x[i]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l * (double)inv_n);
  __syncthreads();
  for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) atomicAdd(&G[p], sG[p]);
}

__global__ void mlp_forward_kernel(const float* __restrict__ Pg, const float* __restrict__ X, long long n,
                                   float* __restrict__ out) {
  __shared__ float P[kMlpParams];
  for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) P[p] = Pg[p];
  __syncthreads();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float x[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) x[i] = X[t * kMlpIn + i];
  float z1[kMlpHidden], z2[kMlpHidden], o;
  out[t] = mlp_forward_keep(P, x, z1, z2, o);
}

// The step kernel's tensor-core evaluation (mlp_nut_warp) over rows of X: one warp per
// 32 rows, rows past n evaluated on zeros and discarded.
__global__ void mlp_forward_tc_kernel(const uint32_t* __restrict__ frag_g, const float* __restrict__ bias_g,
                                      const float* __restrict__ X, long long n, float* __restrict__ out) {
  __shared__ uint32_t frag[kMlpFragWords * 32];
  __shared__ float bias[kMlpBias];
  __shared__ uint32_t stage[4][32 * 4];
  for (int i = threadIdx.x; i < kMlpFragWords * 32; i += blockDim.x) frag[i] = frag_g[i];
  for (int i = threadIdx.x; i < kMlpBias; i += blockDim.x) bias[i] = bias_g[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long row = ((long long)blockIdx.x * 4 + warp) * 32 + lane;
  float x[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) x[i] = row < n ? X[row * kMlpIn + i] : 0.0f;
  const float y = mlp_nut_warp(x, frag, bias, stage[warp], lane);
  if (row < n) out[row] = y;
}

// The MLP over rows of X on the 5th-generation tensor cores: a CTA of 4 warps takes
// 128-row tiles (grid-stride); thread t owns row t of the tile and TMEM lane t.  The
// dynamic shared memory (kUmmaSmem) caps residency at 8 CTAs per SM, so the 8 x 64
// allocated TMEM columns always fit: D1 in columns 0..31, D2 in 32..63, and D3 back in
// 0..15 once D1 has been read.  Every mbarrier wait is bounded: on a timeout the
// CTA records the error, waits (bounded) for its last commit and frees its TMEM.
constexpr int kUmmaCols = 64;
constexpr int kUmmaSmem = 27 * 1024;
constexpr int kUmmaWaitLimit = 1 << 22;

__global__ void __launch_bounds__(kUmmaRows) mlp_forward_umma_kernel(const uint4* __restrict__ bimg,
                                                                     const float* __restrict__ bias_g,
                                                                     const float* __restrict__ X, long long n,
                                                                     float* __restrict__ out, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* sA1 = sm;                                          // 128 x 16 BF16
  uint8_t* sA2 = sm + 4096;                                   // 128 x 32 BF16
  uint8_t* sB = sm + 12288;                                   // weight image
  float* sbias = reinterpret_cast<float*>(sm + 16384);        // [65]
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + 16384 + 512);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 16384 + 520);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < kUmmaBBytes / 16; i += kUmmaRows) reinterpret_cast<uint4*>(sB)[i] = bimg[i];
  for (int i = tid; i < kMlpBias; i += kUmmaRows) sbias[i] = bias_g[i];
  *reinterpret_cast<uint4*>(sA1 + umma_off(tid, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);  // K padding
  const uint32_t mb = (uint32_t)__cvta_generic_to_shared(mbar);
  if (tid == 0) umma_mbar_init(mb);
  if (warp == 0) {
    tmem_alloc((uint32_t)__cvta_generic_to_shared(tslot), kUmmaCols);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t a1 = (uint32_t)__cvta_generic_to_shared(sA1), a2 = (uint32_t)__cvta_generic_to_shared(sA2),
                 b = (uint32_t)__cvta_generic_to_shared(sB);
  const uint64_t dA1 = umma_smem_desc(a1, 128, 256);
  const uint64_t dA2[2] = {umma_smem_desc(a2, 128, 512), umma_smem_desc(a2 + 256, 128, 512)};
  const uint64_t dB1 = umma_smem_desc(b + kUmmaB1, 128, 256);
  const uint64_t dB2[2] = {umma_smem_desc(b + kUmmaB2, 128, 512), umma_smem_desc(b + kUmmaB2 + 256, 128, 512)};
  const uint64_t dB3[2] = {umma_smem_desc(b + kUmmaB3, 128, 512), umma_smem_desc(b + kUmmaB3 + 256, 128, 512)};
  constexpr uint32_t id32 = umma_idesc_bf16(kUmmaRows, 32), id16 = umma_idesc_bf16(kUmmaRows, 16);
  const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  int issued = 0;  // commits issued (thread 0)
  bool failed = false;
  const long long tiles = (n + kUmmaRows - 1) / kUmmaRows;
  // one layer: thread 0 issues, everyone waits; false when the CTA timed out
  auto run = [&](auto issue) -> bool {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      issue();
      umma_commit(mb);
      ++issued;
    }
    const bool ok = umma_mbar_wait(mb, phase, kUmmaWaitLimit);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) return false;
    tc_fence_after();
    return true;
  };
  for (long long tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
    const long long row = tile * kUmmaRows + tid;
    float x[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) x[i] = row < n ? X[row * kMlpIn + i] : 0.0f;
    *reinterpret_cast<uint4*>(sA1 + umma_off(tid, 0, 16)) =
        make_uint4(bf16x2_of(x[0], x[1]), bf16x2_of(x[2], x[3]), bf16x2_of(x[4], x[5]), bf16x2_of(x[6], x[7]));
    if (!run([&] { umma_bf16(tbase, dA1, dB1, id32, 0u); })) { failed = true; break; }
    float d[32];
    tmem_ld32(lane_base, d);
    umma_store_hidden(sA2, tid, d, sbias);
    if (!run([&] {
          umma_bf16(tbase + 32, dA2[0], dB2[0], id32, 0u);
          umma_bf16(tbase + 32, dA2[1], dB2[1], id32, 1u);
        })) { failed = true; break; }
    tmem_ld32(lane_base + 32, d);
    umma_store_hidden(sA2, tid, d, sbias + 32);
    if (!run([&] {
          umma_bf16(tbase, dA2[0], dB3[0], id16, 0u);
          umma_bf16(tbase, dA2[1], dB3[1], id16, 1u);
        })) { failed = true; break; }
    const float o = tmem_ld1(lane_base) + sbias[64];
    if (row < n) out[row] = softplus_f(o);
    tc_fence_before();
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err, 1);
      umma_mbar_wait(mb, (uint32_t)((issued - 1) & 1), kUmmaWaitLimit);  // the last commit
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tbase, kUmmaCols);
}

// Adam (Kingma & Ba, 2015) on the FP32 parameters.
__global__ void adam_kernel(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ G, float lr, float b1t, float b2t) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const float g = G[p];
  const float mp = 0.9f * m[p] + 0.1f * g;
  const float vp = 0.999f * v[p] + 0.001f * g * g;
  m[p] = mp;
  v[p] = vp;
  const float mh = mp / (1.0f - b1t), vh = vp / (1.0f - b2t);
  P[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// Mini-batch rows: a splitmix64 hash of (seed, iteration, slot) modulo n.
__global__ void batch_index_kernel(long long* __restrict__ idx, int B, unsigned long long seed, int it, long long n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B) return;
  unsigned long long z = seed + 0x9e3779b97f4a7c15ull * ((unsigned long long)it * 1000003ull + (unsigned long long)i + 1ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  idx[i] = (long long)(z % (unsigned long long)n);
}

// ---- wall distance: jump flooding over the solid cells (Rong & Tan, 2006) ----------
// Each cell keeps the packed coordinates (10 bits each) of the nearest solid cell seen.
constexpr uint32_t kNoSeed = 0xffffffffu;
__device__ __forceinline__ uint32_t pack_xyz(int x, int y, int z) {
  return (uint32_t)x | ((uint32_t)y << 10) | ((uint32_t)z << 20);
}
__device__ __forceinline__ float seed_dist2(uint32_t s, int x, int y, int z) {
  const float dx = (float)((int)(s & 1023u) - x), dy = (float)((int)((s >> 10) & 1023u) - y),
              dz = (float)((int)((s >> 20) & 1023u) - z);
  return dx * dx + dy * dy + dz * dz;
}

__global__ void jfa_init_kernel(const uint8_t* __restrict__ flags, int nx, int ny, int nz, uint32_t* __restrict__ seed) {
  const long long N = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long r = i / nx;
    seed[i] = flags[i] == CELL_SOLID ? pack_xyz(x, (int)(r % ny), (int)(r / ny)) : kNoSeed;
  }
}

__global__ void jfa_pass_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int nx, int ny, int nz,
                                int k) {
  const long long N = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long r = i / nx;
    const int y = (int)(r % ny), z = (int)(r / ny);
    uint32_t best = in[i];
    float bd = best == kNoSeed ? 3.0e38f : seed_dist2(best, x, y, z);
    for (int dz = -k; dz <= k; dz += k)
      for (int dy = -k; dy <= k; dy += k)
        for (int dx = -k; dx <= k; dx += k) {
          const int xx = x + dx, yy = y + dy, zz = z + dz;
          if (xx < 0 || yy < 0 || zz < 0 || xx >= nx || yy >= ny || zz >= nz) continue;
          const uint32_t s = in[xx + (long long)nx * (yy + (long long)ny * zz)];
          if (s == kNoSeed) continue;
          const float d = seed_dist2(s, x, y, z);
          if (d < bd) {
            bd = d;
            best = s;
          }
        }
    out[i] = best;
  }
}

// Distances (cells) into a dense float array and, rounded and capped at 31, into
// bits 3..7 of the solver's class bytes.
__global__ void jfa_finish_kernel(const uint32_t* __restrict__ seed, int nx, int ny, int nz, float* __restrict__ dist,
                                  uint8_t* __restrict__ cls, int pitch) {
  const long long N = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long r = i / nx;
    const int y = (int)(r % ny), z = (int)(r / ny);
    const uint32_t s = seed[i];
    const float d = s == kNoSeed ? 1.0e4f : sqrtf(seed_dist2(s, x, y, z));
    if (dist) dist[i] = d;
    if (cls) {
      const int q = d >= 31.0f ? 31 : (int)lrintf(d);
      uint8_t& c = cls[r * pitch + x];
      c = (uint8_t)((c & 7) | (q << 3));
    }
  }
}

// ---- training samples from a fine-grid flow -------------------------------------
// Coarse cell (X, Y, Z) covers fine cells (2X..2X+1, 2Y.., 2Z..).  Pass 1: box-filtered
// velocity, density and velocity products; cells with a solid child are invalid.
__global__ void sgs_filter_kernel(const float* __restrict__ ux, const float* __restrict__ uy,
                                  const float* __restrict__ uz, const float* __restrict__ rho,
                                  const uint8_t* __restrict__ fflags, int fx, int fy, int fz, int cx, int cy, int cz,
                                  float* __restrict__ ubar /*[Nc][4]*/, float* __restrict__ uu /*[Nc][6]*/) {
  const long long Nc = (long long)cx * cy * cz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < Nc; c += (long long)gridDim.x * blockDim.x) {
    const int X = (int)(c % cx);
    const long long R = c / cx;
    const int Y = (int)(R % cy), Z = (int)(R / cy);
    float su[3] = {0, 0, 0}, sr = 0.0f, sq[6] = {0, 0, 0, 0, 0, 0};
    bool ok = true;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const long long f = (2 * X + dx) + (long long)fx * ((2 * Y + dy) + (long long)fy * (2 * Z + dz));
          if (fflags[f] == CELL_SOLID) ok = false;
          const float a = ux[f], b = uy[f], d = uz[f];
          su[0] += a; su[1] += b; su[2] += d; sr += rho[f];
          sq[0] += a * a; sq[1] += b * b; sq[2] += d * d; sq[3] += a * b; sq[4] += a * d; sq[5] += b * d;
        }
    const float* qq = sq;
    ubar[c * 4 + 0] = su[0] * 0.125f;
    ubar[c * 4 + 1] = su[1] * 0.125f;
    ubar[c * 4 + 2] = su[2] * 0.125f;
    ubar[c * 4 + 3] = ok ? sr * 0.125f : -1.0f;  // density; -1 marks an invalid cell
    for (int k = 0; k < 6; ++k) uu[c * 6 + k] = qq[k] * 0.125f;
  }
}

// Pass 2: filtered strain rate (central differences), subgrid stress
// tau = (u u)~ - u~ u~ and the two terms of the least-squares eddy viscosity
// nu_t = -tau_d : S / (2 S : S): numerator and denominator per cell (0 where invalid);
// features as in mlp_features with the filtered strain rate.
__global__ void sgs_sample_kernel(const float* __restrict__ ubar, const float* __restrict__ uu,
                                  const uint8_t* __restrict__ ccls, int cpitch, int cx, int cy, int cz,
                                  float* __restrict__ Xo, float2* __restrict__ nd, uint8_t* __restrict__ valid) {
  const long long Nc = (long long)cx * cy * cz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < Nc; c += (long long)gridDim.x * blockDim.x) {
    const int X = (int)(c % cx);
    const long long R = c / cx;
    const int Y = (int)(R % cy), Z = (int)(R / cy);
    bool ok = X > 0 && Y > 0 && Z > 0 && X < cx - 1 && Y < cy - 1 && Z < cz - 1 && ubar[c * 4 + 3] > 0.0f;
    float g[3][3];  // g[a][b] = d u_a / d x_b
    const long long st[3] = {1, cx, (long long)cx * cy};
    for (int bdir = 0; bdir < 3 && ok; ++bdir) {
      const long long p = c + st[bdir], m = c - st[bdir];
      if (ubar[p * 4 + 3] <= 0.0f || ubar[m * 4 + 3] <= 0.0f) ok = false;
      for (int a = 0; a < 3; ++a) g[a][bdir] = 0.5f * (ubar[p * 4 + a] - ubar[m * 4 + a]);
    }
    valid[c] = ok ? 1 : 0;
    if (!ok) {
      nd[c] = make_float2(0.0f, 0.0f);
      continue;
    }
    const float sxx = g[0][0], syy = g[1][1], szz = g[2][2];
    const float sxy = 0.5f * (g[0][1] + g[1][0]), sxz = 0.5f * (g[0][2] + g[2][0]), syz = 0.5f * (g[1][2] + g[2][1]);
    const float ux = ubar[c * 4], uy = ubar[c * 4 + 1], uz = ubar[c * 4 + 2], r = ubar[c * 4 + 3];
    float t[6] = {uu[c * 6] - ux * ux, uu[c * 6 + 1] - uy * uy, uu[c * 6 + 2] - uz * uz,
                  uu[c * 6 + 3] - ux * uy, uu[c * 6 + 4] - ux * uz, uu[c * 6 + 5] - uy * uz};
    const float tr = (t[0] + t[1] + t[2]) * (1.0f / 3.0f);
    t[0] -= tr; t[1] -= tr; t[2] -= tr;
    const float ss = sxx * sxx + syy * syy + szz * szz + 2.0f * (sxy * sxy + sxz * sxz + syz * syz);
    const float ts = t[0] * sxx + t[1] * syy + t[2] * szz + 2.0f * (t[3] * sxy + t[4] * sxz + t[5] * syz);
    nd[c] = make_float2(-ts, 2.0f * ss);
    const float wd = (float)(ccls[R * cpitch + X] >> 3);
    float* xo = Xo + c * kMlpIn;
    xo[0] = 100.0f * sxx; xo[1] = 100.0f * syy; xo[2] = 100.0f * szz;
    xo[3] = 100.0f * sxy; xo[4] = 100.0f * sxz; xo[5] = 100.0f * syz;
    xo[6] = 100.0f * (r - 1.0f);
    xo[7] = wd * (1.0f / 16.0f);
  }
}

// Pass 3: the target nu_t / nu_0 of a valid cell: numerators and denominators summed
// over the valid cells of its (2 avg + 1)^3 neighbourhood, then divided and clipped to
// [min_ratio, max_ratio] (least-squares averaging, which keeps the sign information that a
// per-cell clip at zero would discard; min_ratio < 0 keeps backscatter in the targets, so
// that a regression onto a non-negative output learns the conditional mean rather than
// the mean of the clipped values, which lies above it).
__global__ void sgs_target_kernel(const float2* __restrict__ nd, const uint8_t* __restrict__ valid, int cx, int cy,
                                  int cz, int avg, float nu0, float min_ratio, float max_ratio,
                                  float* __restrict__ Yo) {
  const long long Nc = (long long)cx * cy * cz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < Nc; c += (long long)gridDim.x * blockDim.x) {
    if (!valid[c]) {
      Yo[c] = 0.0f;
      continue;
    }
    const int X = (int)(c % cx);
    const long long R = c / cx;
    const int Y = (int)(R % cy), Z = (int)(R / cy);
    float n = 0.0f, d = 0.0f;
    for (int dz = -avg; dz <= avg; ++dz)
      for (int dy = -avg; dy <= avg; ++dy)
        for (int dx = -avg; dx <= avg; ++dx) {
          const int xx = X + dx, yy = Y + dy, zz = Z + dz;
          if (xx < 0 || yy < 0 || zz < 0 || xx >= cx || yy >= cy || zz >= cz) continue;
          const float2 v = nd[xx + (long long)cx * (yy + (long long)cy * zz)];
          n += v.x;
          d += v.y;
        }
    float nut = d > 0.0f ? n / d : 0.0f;
    nut = fminf(fmaxf(nut, min_ratio * nu0), max_ratio * nu0);
    Yo[c] = nut / nu0;
  }
}

int sgs_fail(int code, const std::string& msg) {
  set_global_error(msg);
  return code;
}

// Device time of the last forward kernel run by aerosim_mlp_forward_tc / _umma.
double g_mlp_last_ms = 0.0;

// CUDA events around one kernel launch on the default stream.
struct KernelTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  KernelTimer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
  }
  double stop() {
    float ms = 0.0f;
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~KernelTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

#define SCU(x)                                                                                       \
  do {                                                                                               \
    cudaError_t e_ = (x);                                                                            \
    if (e_ != cudaSuccess) return sgs_fail(AEROSIM_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

// RAII device buffer for the host-array entry points below.
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 1); }
  template <class T> T* as() { return static_cast<T*>(p); }
};

}  // namespace

// Jump-flood wall distance of a dense flag array (device), written as float distances
// (dist, may be null) and into bits 3..7 of the pitched class bytes (cls, may be null).
cudaError_t compute_wall_distance(const uint8_t* flags, int nx, int ny, int nz, float* dist, uint8_t* cls, int pitch,
                                  cudaStream_t s) {
  const long long N = (long long)nx * ny * nz;
  if (nx > 1024 || ny > 1024 || nz > 1024) return cudaErrorInvalidValue;
  uint32_t *a = nullptr, *b = nullptr;
  cudaError_t e = cudaMallocAsync(&a, N * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&b, N * sizeof(uint32_t), s);
  const int grid = (int)std::min<long long>((N + 255) / 256, 148 * 16);
  if (e == cudaSuccess) jfa_init_kernel<<<grid, 256, 0, s>>>(flags, nx, ny, nz, a);
  int k = 1;
  while (2 * k < std::max(nx, std::max(ny, nz))) k *= 2;
  for (; k >= 1 && e == cudaSuccess; k /= 2) {
    jfa_pass_kernel<<<grid, 256, 0, s>>>(a, b, nx, ny, nz, k);
    std::swap(a, b);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {  // one more unit pass removes most of the flood's errors (JFA+1)
    jfa_pass_kernel<<<grid, 256, 0, s>>>(a, b, nx, ny, nz, 1);
    std::swap(a, b);
    jfa_finish_kernel<<<grid, 256, 0, s>>>(a, nx, ny, nz, dist, cls, pitch);
    e = cudaGetLastError();
  }
  cudaFreeAsync(a, s);
  cudaFreeAsync(b, s);
  return e;
}

cudaError_t launch_sgs_samples(const float* ux, const float* uy, const float* uz, const float* rho,
                               const uint8_t* fflags, int fx, int fy, int fz, const uint8_t* ccls, int cpitch, int cx,
                               int cy, int cz, float nu0, float min_ratio, float max_ratio, int avg, float* X,
                               float* Y, uint8_t* valid, cudaStream_t s) {
  const long long Nc = (long long)cx * cy * cz;
  float *ubar = nullptr, *uu = nullptr;
  float2* nd = nullptr;
  cudaError_t e = cudaMallocAsync(&ubar, Nc * 4 * sizeof(float), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&uu, Nc * 6 * sizeof(float), s);
  if (e == cudaSuccess) e = cudaMallocAsync(&nd, Nc * sizeof(float2), s);
  const int grid = (int)std::min<long long>((Nc + 255) / 256, 148 * 16);
  if (e == cudaSuccess) {
    sgs_filter_kernel<<<grid, 256, 0, s>>>(ux, uy, uz, rho, fflags, fx, fy, fz, cx, cy, cz, ubar, uu);
    sgs_sample_kernel<<<grid, 256, 0, s>>>(ubar, uu, ccls, cpitch, cx, cy, cz, X, nd, valid);
    sgs_target_kernel<<<grid, 256, 0, s>>>(nd, valid, cx, cy, cz, avg, nu0, min_ratio, max_ratio, Y);
    e = cudaGetLastError();
  }
  cudaFreeAsync(ubar, s);
  cudaFreeAsync(uu, s);
  cudaFreeAsync(nd, s);
  return e;
}

}  // namespace aerosim

using namespace aerosim;

extern "C" {

int aerosim_mlp_param_count(void) { return kMlpParams; }

int aerosim_mlp_forward(const float* params, const float* X, int64_t n, float* out) {
  if (!params || !X || !out || n < 0) return sgs_fail(AEROSIM_ERR_ARG, "mlp_forward: bad argument");
  if (n == 0) return AEROSIM_OK;
  DevBuf P, Xd, O;
  SCU(P.alloc(kMlpParams * 4));
  SCU(Xd.alloc((size_t)n * kMlpIn * 4));
  SCU(O.alloc((size_t)n * 4));
  SCU(cudaMemcpy(P.p, params, kMlpParams * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(Xd.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice));
  mlp_forward_kernel<<<(unsigned)((n + 127) / 128), 128>>>(P.as<float>(), Xd.as<float>(), n, O.as<float>());
  SCU(cudaGetLastError());
  SCU(cudaMemcpy(out, O.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return AEROSIM_OK;
}

int aerosim_mlp_forward_tc(const float* params, const float* X, int64_t n, float* out) {
  if (!params || !X || !out || n < 0) return sgs_fail(AEROSIM_ERR_ARG, "mlp_forward_tc: bad argument");
  if (n == 0) return AEROSIM_OK;
  std::vector<uint32_t> frag(kMlpFragWords * 32);
  std::vector<float> bias(kMlpBias);
  mlp_pack_fragments(params, frag.data(), bias.data());
  DevBuf F, B, Xd, O;
  SCU(F.alloc(frag.size() * 4));
  SCU(B.alloc(bias.size() * 4));
  SCU(Xd.alloc((size_t)n * kMlpIn * 4));
  SCU(O.alloc((size_t)n * 4));
  SCU(cudaMemcpy(F.p, frag.data(), frag.size() * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(B.p, bias.data(), bias.size() * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(Xd.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice));
  {
    KernelTimer t;
    mlp_forward_tc_kernel<<<(unsigned)((n + 127) / 128), 128>>>(F.as<uint32_t>(), B.as<float>(), Xd.as<float>(), n,
                                                                O.as<float>());
    SCU(cudaGetLastError());
    g_mlp_last_ms = t.stop();
  }
  SCU(cudaMemcpy(out, O.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return AEROSIM_OK;
}

int aerosim_mlp_forward_umma(const float* params, const float* X, int64_t n, float* out) {
  if (!params || !X || !out || n < 0) return sgs_fail(AEROSIM_ERR_ARG, "mlp_forward_umma: bad argument");
  if (n == 0) return AEROSIM_OK;
  std::vector<uint16_t> img(kUmmaBBytes / 2);
  std::vector<uint32_t> frag(kMlpFragWords * 32);
  std::vector<float> bias(kMlpBias);
  mlp_pack_umma(params, img.data());
  mlp_pack_fragments(params, frag.data(), bias.data());
  int dev = 0, sms = 0;
  SCU(cudaGetDevice(&dev));
  SCU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DevBuf Bi, B, Xd, O, E;
  SCU(Bi.alloc(kUmmaBBytes));
  SCU(B.alloc(bias.size() * 4));
  SCU(Xd.alloc((size_t)n * kMlpIn * 4));
  SCU(O.alloc((size_t)n * 4));
  SCU(E.alloc(4));
  SCU(cudaMemcpy(Bi.p, img.data(), kUmmaBBytes, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(B.p, bias.data(), bias.size() * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(Xd.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemset(E.p, 0, 4));
  SCU(cudaFuncSetAttribute(mlp_forward_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kUmmaSmem));
  const long long tiles = (n + kUmmaRows - 1) / kUmmaRows;
  const unsigned grid = (unsigned)std::min<long long>(tiles, 8LL * sms);
  {
    KernelTimer t;
    mlp_forward_umma_kernel<<<grid, kUmmaRows, kUmmaSmem>>>(static_cast<const uint4*>(Bi.p), B.as<float>(),
                                                            Xd.as<float>(), n, O.as<float>(), E.as<int>());
    SCU(cudaGetLastError());
    g_mlp_last_ms = t.stop();
  }
  int e = 0;
  SCU(cudaMemcpy(&e, E.p, 4, cudaMemcpyDeviceToHost));
  if (e) return sgs_fail(AEROSIM_ERR_DEVICE, "mlp_forward_umma: tensor-core commit wait timed out");
  SCU(cudaMemcpy(out, O.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return AEROSIM_OK;
}

int aerosim_mlp_last_timing(double* ms) {
  if (!ms) return sgs_fail(AEROSIM_ERR_ARG, "mlp_last_timing: bad argument");
  *ms = g_mlp_last_ms;
  return AEROSIM_OK;
}

int aerosim_mlp_gradients(const float* params, const float* X, const float* Y, int64_t n, float* grad,
                          double* loss) {
  if (!params || !X || !Y || !grad || !loss || n < 1) return sgs_fail(AEROSIM_ERR_ARG, "mlp_gradients: bad argument");
  DevBuf P, Xd, Yd, G, L;
  SCU(P.alloc(kMlpParams * 4));
  SCU(Xd.alloc((size_t)n * kMlpIn * 4));
  SCU(Yd.alloc((size_t)n * 4));
  SCU(G.alloc(kMlpParams * 4));
  SCU(L.alloc(8));
  SCU(cudaMemcpy(P.p, params, kMlpParams * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(Xd.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(Yd.p, Y, (size_t)n * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemset(G.p, 0, kMlpParams * 4));
  SCU(cudaMemset(L.p, 0, 8));
  mlp_grad_kernel<<<(unsigned)((n + kTrainBlock - 1) / kTrainBlock), kTrainBlock>>>(
      P.as<float>(), Xd.as<float>(), Yd.as<float>(), nullptr, n, 1.0f / (float)n, G.as<float>(), L.as<double>());
  SCU(cudaGetLastError());
  SCU(cudaMemcpy(grad, G.p, kMlpParams * 4, cudaMemcpyDeviceToHost));
  SCU(cudaMemcpy(loss, L.p, 8, cudaMemcpyDeviceToHost));
  return AEROSIM_OK;
}

int aerosim_mlp_train(float* params, const float* X, const float* Y, int64_t n, int32_t iters, int32_t batch,
                      float lr, uint64_t seed, float* loss_curve) {
  if (!params || !X || !Y || n < 1 || iters < 0 || batch < 1 || !(lr > 0.0f))
    return sgs_fail(AEROSIM_ERR_ARG, "mlp_train: bad argument");
  DevBuf P, Xd, Yd, G, M, V, L, I;
  SCU(P.alloc(kMlpParams * 4));
  SCU(Xd.alloc((size_t)n * kMlpIn * 4));
  SCU(Yd.alloc((size_t)n * 4));
  SCU(G.alloc(kMlpParams * 4));
  SCU(M.alloc(kMlpParams * 4));
  SCU(V.alloc(kMlpParams * 4));
  SCU(L.alloc((size_t)std::max(iters, 1) * 8));
  SCU(I.alloc((size_t)batch * 8));
  SCU(cudaMemcpy(P.p, params, kMlpParams * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(Xd.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemcpy(Yd.p, Y, (size_t)n * 4, cudaMemcpyHostToDevice));
  SCU(cudaMemset(M.p, 0, kMlpParams * 4));
  SCU(cudaMemset(V.p, 0, kMlpParams * 4));
  SCU(cudaMemset(L.p, 0, (size_t)std::max(iters, 1) * 8));
  float b1t = 1.0f, b2t = 1.0f;
  for (int it = 0; it < iters; ++it) {
    b1t *= 0.9f;
    b2t *= 0.999f;
    batch_index_kernel<<<(batch + 255) / 256, 256>>>(I.as<long long>(), batch, seed, it, n);
    SCU(cudaMemsetAsync(G.p, 0, kMlpParams * 4));
    mlp_grad_kernel<<<(batch + kTrainBlock - 1) / kTrainBlock, kTrainBlock>>>(
        P.as<float>(), Xd.as<float>(), Yd.as<float>(), I.as<long long>(), batch, 1.0f / (float)batch, G.as<float>(),
        L.as<double>() + it);
    adam_kernel<<<(kMlpParams + 255) / 256, 256>>>(P.as<float>(), M.as<float>(), V.as<float>(), G.as<float>(), lr,
                                                   b1t, b2t);
  }
  SCU(cudaGetLastError());
  SCU(cudaDeviceSynchronize());
  SCU(cudaMemcpy(params, P.p, kMlpParams * 4, cudaMemcpyDeviceToHost));
  if (loss_curve && iters > 0) {
    std::vector<double> l(iters);
    SCU(cudaMemcpy(l.data(), L.p, (size_t)iters * 8, cudaMemcpyDeviceToHost));
    for (int i = 0; i < iters; ++i) loss_curve[i] = (float)l[i];
  }
  return AEROSIM_OK;
}

}  // extern "C"
