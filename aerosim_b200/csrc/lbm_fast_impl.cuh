// Body of the FP32-arithmetic step translation units: each unit instantiates the step
// kernel for one storage type (AEROSIM_FAST_STORE) over every compiled row pitch, and
// the batched step kernel.
// Compiled with FMA contraction enabled: these paths are checked against the oracle
// within a tolerance, not bit for bit.
#include <type_traits>
#include "common.cuh"
#include "lbm_launch.cuh"

namespace aerosim {

cudaError_t AEROSIM_FAST_FN(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ,
                            int* launches) {
  return step_dispatch<AEROSIM_FAST_STORE, MODE_FAST>(a, block, grid, smem, s, occ, launches);
}

cudaError_t AEROSIM_BATCH_FN(const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s, int* occ) {
  return batch_dispatch<AEROSIM_FAST_STORE>(b, pitch, grid, smem, s, occ);
}

}  // namespace aerosim
