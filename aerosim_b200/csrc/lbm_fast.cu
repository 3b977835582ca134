// Storage-type dispatch of the FP32-arithmetic step kernels (lbm_fast_<storage>.cu).
#include "common.cuh"
#include "engine_internal.h"
#include "../../include/aerosim.h"

namespace aerosim {

cudaError_t launch_step_fast_f32(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ,
                                 int* launches);
cudaError_t launch_step_fast_f16s(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s,
                                  int* occ, int* launches);
cudaError_t launch_step_fast_bf16s(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s,
                                   int* occ, int* launches);

cudaError_t launch_step_fast(int precision, const StepArgs& a, dim3 block, unsigned grid, size_t smem,
                             cudaStream_t s, int* occ, int* launches) {
  switch (precision) {
    case AEROSIM_PREC_F32: return launch_step_fast_f32(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_F16S: return launch_step_fast_f16s(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_BF16S: return launch_step_fast_bf16s(a, block, grid, smem, s, occ, launches);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace aerosim
