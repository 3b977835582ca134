// Launch helper shared by the kernel translation units: the step kernel uses
// dynamic shared memory above 48 KB, so its attribute is raised before the
// occupancy query that sizes the persistent grid.
#pragma once
#include "lbm_kernels.cuh"

namespace aerosim {

// One time step: a single main_kernel launch.  Returns the number of launches in
// *launches.
template <class S, int MODE>
cudaError_t step_entry(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ,
                       int* launches) {
  auto k = main_kernel<S, MODE>;
  if (occ) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, (int)(block.x * block.y), smem);
  }
  k<<<grid, block, smem, s>>>(a);
  if (launches) *launches = 1;
  return cudaGetLastError();
}

}  // namespace aerosim
