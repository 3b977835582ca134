// Storage-type dispatch of the FP32-arithmetic step and batch kernels (lbm_fast_<storage>.cu).
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
cudaError_t launch_step_fast_f16c(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s,
                                  int* occ, int* launches);

cudaError_t launch_batch_fast_f32(const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s,
                                  int* occ);
cudaError_t launch_batch_fast_f16s(const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s,
                                   int* occ);
cudaError_t launch_batch_fast_bf16s(const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s,
                                    int* occ);
cudaError_t launch_batch_fast_f16c(const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s,
                                   int* occ);

cudaError_t launch_batch(int precision, const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s,
                         int* occ) {
  switch (precision) {
    case AEROSIM_PREC_F32: return launch_batch_fast_f32(b, pitch, grid, smem, s, occ);
    case AEROSIM_PREC_F16S: return launch_batch_fast_f16s(b, pitch, grid, smem, s, occ);
    case AEROSIM_PREC_BF16S: return launch_batch_fast_bf16s(b, pitch, grid, smem, s, occ);
    case AEROSIM_PREC_F16C: return launch_batch_fast_f16c(b, pitch, grid, smem, s, occ);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_step_fast(int precision, const StepArgs& a, dim3 block, unsigned grid, size_t smem,
                             cudaStream_t s, int* occ, int* launches) {
  switch (precision) {
    case AEROSIM_PREC_F32: return launch_step_fast_f32(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_F16S: return launch_step_fast_f16s(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_BF16S: return launch_step_fast_bf16s(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_F16C: return launch_step_fast_f16c(a, block, grid, smem, s, occ, launches);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace aerosim
