// FP64-arithmetic kernels: the bit-parity mirror of the reference's JavaScript
// solver (FP32 storage) and the FP64 oracle run (FP64 storage), plus the force
// reduction, initialisation and readback kernels of every precision.  Compiled
// with -fmad=false so every multiply and add rounds separately, as in JavaScript.
#include <type_traits>
#include "common.cuh"
#include "engine_internal.h"
#include "lbm_launch.cuh"
#include "lbm_aux.cuh"
#include "../../include/aerosim.h"

namespace aerosim {

cudaError_t launch_step_fast(int precision, const StepArgs& a, dim3 block, unsigned grid, size_t smem,
                             cudaStream_t s, int* occ, int* launches);

size_t precision_bytes(int precision) {
  switch (precision) {
    case AEROSIM_PREC_F32: case AEROSIM_PREC_F32_MIRROR: return 4;
    case AEROSIM_PREC_F16S: case AEROSIM_PREC_BF16S: case AEROSIM_PREC_F16C: return 2;
    case AEROSIM_PREC_F64: return 8;
    default: return 0;
  }
}

cudaError_t launch_step(int precision, const StepArgs& a, dim3 block, unsigned grid, size_t smem,
                        cudaStream_t s, int* occ, int* launches) {
  switch (precision) {
    case AEROSIM_PREC_F32_MIRROR: return step_dispatch<StoreF32, MODE_MIRROR>(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_F64: return step_dispatch<StoreF64, MODE_F64>(a, block, grid, smem, s, occ, launches);
    default: return launch_step_fast(precision, a, block, grid, smem, s, occ, launches);
  }
}

// A launch as a programmatic dependent of the kernel before it on the stream: its CTAs may
// be scheduled while that kernel finishes and wait (griddepcontrol.wait) for its completion.
template <class K, class... Args>
static cudaError_t launch_dependent(K kernel, unsigned grid, unsigned block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, args...);
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_forces(int precision, const ForceArgs& a, unsigned grid, cudaStream_t s) {
  switch (precision) {
    case AEROSIM_PREC_F32: return launch_dependent(forces_kernel<StoreF32S, MODE_FAST>, grid, 256, s, a);
    case AEROSIM_PREC_F32_MIRROR: return launch_dependent(forces_kernel<StoreF32, MODE_MIRROR>, grid, 256, s, a);
    case AEROSIM_PREC_F16S: case AEROSIM_PREC_F16C: return launch_dependent(forces_kernel<StoreF16S, MODE_FAST>, grid, 256, s, a);
    case AEROSIM_PREC_BF16S: return launch_dependent(forces_kernel<StoreBF16S, MODE_FAST>, grid, 256, s, a);
    case AEROSIM_PREC_F64: return launch_dependent(forces_kernel<StoreF64, MODE_F64>, grid, 256, s, a);
    default: return cudaErrorInvalidValue;
  }
}

static unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148LL * 64) g = 148LL * 64;
  return (unsigned)(g < 1 ? 1 : g);
}

cudaError_t launch_classify(const uint8_t* flags, uint8_t* cls, const Layout& L, cudaStream_t s) {
  classify_kernel<<<grid_for((long long)L.nx * L.ny * L.nz), 256, 0, s>>>(flags, cls, L);
  return cudaGetLastError();
}

cudaError_t launch_init(int precision, void* f0, void* f1, const uint8_t* cls, float* mux, float* muy,
                        float* muz, float* mrho, const double* abl, const Layout& L, double u_inlet, int gns,
                        cudaStream_t s) {
  const unsigned g = grid_for((long long)L.nx * L.ny * L.nz);
#define AEROSIM_INIT(S) init_kernel<S><<<g, 256, 0, s>>>(f0, f1, cls, mux, muy, muz, mrho, abl, L, u_inlet, gns)
  switch (precision) {
    case AEROSIM_PREC_F32: AEROSIM_INIT(StoreF32S); break;
    case AEROSIM_PREC_F32_MIRROR: AEROSIM_INIT(StoreF32); break;
    case AEROSIM_PREC_F16S: case AEROSIM_PREC_F16C: AEROSIM_INIT(StoreF16S); break;
    case AEROSIM_PREC_BF16S: AEROSIM_INIT(StoreBF16S); break;
    case AEROSIM_PREC_F64: AEROSIM_INIT(StoreF64); break;
    default: return cudaErrorInvalidValue;
  }
#undef AEROSIM_INIT
  return cudaGetLastError();
}

template <class S, int MODE>
static void read_pops_t(const void* f, const uint8_t* cls, const StepState* st, int ps, const Layout& L,
                        long long N, void* out, int dtype, cudaStream_t s) {
  if (dtype == AEROSIM_DTYPE_F32)
    read_pops_kernel<S, MODE, float><<<grid_for(N), 256, 0, s>>>(f, cls, st, ps, L, N, (float*)out);
  else
    read_pops_kernel<S, MODE, double><<<grid_for(N), 256, 0, s>>>(f, cls, st, ps, L, N, (double*)out);
}

cudaError_t launch_read_pops(int precision, const void* f, const uint8_t* cls, const StepState* st,
                             int ps, const Layout& L, long long N, void* out, int dtype, cudaStream_t s) {
  switch (precision) {
    case AEROSIM_PREC_F32: read_pops_t<StoreF32S, MODE_FAST>(f, cls, st, ps, L, N, out, dtype, s); break;
    case AEROSIM_PREC_F32_MIRROR: read_pops_t<StoreF32, MODE_MIRROR>(f, cls, st, ps, L, N, out, dtype, s); break;
    case AEROSIM_PREC_F16S: case AEROSIM_PREC_F16C: read_pops_t<StoreF16S, MODE_FAST>(f, cls, st, ps, L, N, out, dtype, s); break;
    case AEROSIM_PREC_BF16S: read_pops_t<StoreBF16S, MODE_FAST>(f, cls, st, ps, L, N, out, dtype, s); break;
    case AEROSIM_PREC_F64: read_pops_t<StoreF64, MODE_F64>(f, cls, st, ps, L, N, out, dtype, s); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class S>
static void write_pops_t(void* f, const Layout& L, long long N, const void* in, int dtype, cudaStream_t s) {
  if (dtype == AEROSIM_DTYPE_F32)
    write_pops_kernel<S, float><<<grid_for(N), 256, 0, s>>>(f, L, N, (const float*)in);
  else
    write_pops_kernel<S, double><<<grid_for(N), 256, 0, s>>>(f, L, N, (const double*)in);
}

cudaError_t launch_write_pops(int precision, void* f, const Layout& L, long long N, const void* in,
                              int dtype, cudaStream_t s) {
  switch (precision) {
    case AEROSIM_PREC_F32: write_pops_t<StoreF32S>(f, L, N, in, dtype, s); break;
    case AEROSIM_PREC_F32_MIRROR: write_pops_t<StoreF32>(f, L, N, in, dtype, s); break;
    case AEROSIM_PREC_F16S: case AEROSIM_PREC_F16C: write_pops_t<StoreF16S>(f, L, N, in, dtype, s); break;
    case AEROSIM_PREC_BF16S: write_pops_t<StoreBF16S>(f, L, N, in, dtype, s); break;
    case AEROSIM_PREC_F64: write_pops_t<StoreF64>(f, L, N, in, dtype, s); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_materialize(int precision, void* f, const uint8_t* cls, const StepState* st, int ps,
                               const Layout& L, long long N, cudaStream_t s) {
  const unsigned g = grid_for(N);
  switch (precision) {
    case AEROSIM_PREC_F32: materialize_rescale_kernel<StoreF32S, MODE_FAST><<<g, 256, 0, s>>>(f, cls, st, ps, L, N); break;
    case AEROSIM_PREC_F32_MIRROR: materialize_rescale_kernel<StoreF32, MODE_MIRROR><<<g, 256, 0, s>>>(f, cls, st, ps, L, N); break;
    case AEROSIM_PREC_F16S: case AEROSIM_PREC_F16C: materialize_rescale_kernel<StoreF16S, MODE_FAST><<<g, 256, 0, s>>>(f, cls, st, ps, L, N); break;
    case AEROSIM_PREC_BF16S: materialize_rescale_kernel<StoreBF16S, MODE_FAST><<<g, 256, 0, s>>>(f, cls, st, ps, L, N); break;
    case AEROSIM_PREC_F64: materialize_rescale_kernel<StoreF64, MODE_F64><<<g, 256, 0, s>>>(f, cls, st, ps, L, N); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_read_macro(const float* mrho, const uint8_t* cls, const StepState* st, int ps,
                              const Layout& L, long long N, float* rho_out, cudaStream_t s) {
  read_macro_kernel<<<grid_for(N), 256, 0, s>>>(mrho, cls, st, ps, L, N, rho_out);
  return cudaGetLastError();
}

cudaError_t launch_mass_stats(const float* mux, const float* muy, const float* muz, const float* rho,
                              const uint8_t* cls, const StepState* st, int ps, const Layout& L, long long N,
                              unsigned long long* out, cudaStream_t s) {
  mass_stats_kernel<<<grid_for(N), 256, 0, s>>>(mux, muy, muz, rho, cls, st, ps, L, N, out);
  return cudaGetLastError();
}

cudaError_t launch_slice(const float* mux, const float* muy, const float* muz, const float* mrho,
                         const uint8_t* cls, const StepState* st, int prev_slot, const Layout& L, int axis, int fixed,
                         int mode, double uref, int width, int height, uint8_t* rgba, cudaStream_t s) {
  const long long P = (long long)width * height;
  const int grid = (int)std::min<long long>((P + 255) / 256, 1184);
  return launch_dependent(slice_kernel, (unsigned)grid, 256, s, mux, muy, muz, mrho, cls, st, prev_slot, L, axis,
                          fixed, mode, uref, width, height, rgba);
}

cudaError_t launch_q_criterion(int nx, int ny, int nz, double dx, const float* ux, const float* uy, const float* uz,
                               const uint8_t* flags, float* q, float* om, float* omv, unsigned long long* maxima,
                               cudaStream_t s) {
  const long long N = (long long)nx * ny * nz;
  cudaError_t e = cudaMemsetAsync(maxima, 0, 2 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  const int grid = (int)std::min<long long>((N + 255) / 256, 148 * 8);
  q_criterion_kernel<<<grid, 256, 0, s>>>(nx, ny, nz, dx, ux, uy, uz, flags, q, om, omv, maxima);
  return cudaGetLastError();
}

}  // namespace aerosim
