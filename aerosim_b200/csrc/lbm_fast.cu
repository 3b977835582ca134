// FP32-arithmetic step kernels (FP32, FP16-shifted and BF16-shifted storage).
// Compiled with FMA contraction enabled: these paths are checked against the
// oracle within a tolerance, not bit for bit.
#include <type_traits>
#include "common.cuh"
#include "engine_internal.h"
#include "lbm_kernels.cuh"
#include "../../include/aerosim.h"

namespace aerosim {

template <class S>
static cudaError_t step_fast(const StepArgs& a, int tx, int ry, cudaStream_t s) {
  const long long rows = (long long)a.ny * a.nz;
  const unsigned grid = (unsigned)((rows + ry - 1) / ry);
  const dim3 block(tx, ry);
  switch (ry) {
    case 1: step_kernel<S, MODE_FAST, 1><<<grid, block, 0, s>>>(a); break;
    case 2: step_kernel<S, MODE_FAST, 2><<<grid, block, 0, s>>>(a); break;
    case 4: step_kernel<S, MODE_FAST, 4><<<grid, block, 0, s>>>(a); break;
    case 8: step_kernel<S, MODE_FAST, 8><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_step_fast(int precision, const StepArgs& a, int tx, int ry, cudaStream_t s) {
  switch (precision) {
    case AEROSIM_PREC_F32: return step_fast<StoreF32>(a, tx, ry, s);
    case AEROSIM_PREC_F16S: return step_fast<StoreF16S>(a, tx, ry, s);
    case AEROSIM_PREC_BF16S: return step_fast<StoreBF16S>(a, tx, ry, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace aerosim
