// Launch helper shared by the kernel translation units: the step kernel uses
// dynamic shared memory above 48 KB, so its attribute is raised before the
// occupancy query that sizes the persistent grid.
#pragma once
#include "lbm_kernels.cuh"

namespace aerosim {

template <class S, int MODE>
cudaError_t step_entry(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ) {
  auto k = step_kernel<S, MODE>;
  if (occ) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, (int)(block.x * block.y), smem);
  }
  k<<<grid, block, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace aerosim
