// FP32-arithmetic step kernels (FP32, FP16-shifted and BF16-shifted storage).
// Compiled with FMA contraction enabled: these paths are checked against the
// oracle within a tolerance, not bit for bit.
#include <type_traits>
#include "common.cuh"
#include "engine_internal.h"
#include "lbm_launch.cuh"
#include "../../include/aerosim.h"

namespace aerosim {

cudaError_t launch_step_fast(int precision, const StepArgs& a, dim3 block, unsigned grid, size_t smem,
                             cudaStream_t s, int* occ, int* launches) {
  switch (precision) {
    case AEROSIM_PREC_F32: return step_entry<StoreF32, MODE_FAST>(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_F16S: return step_entry<StoreF16S, MODE_FAST>(a, block, grid, smem, s, occ, launches);
    case AEROSIM_PREC_BF16S: return step_entry<StoreBF16S, MODE_FAST>(a, block, grid, smem, s, occ, launches);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace aerosim
