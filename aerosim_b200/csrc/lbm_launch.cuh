// Launch helper shared by the kernel translation units: the step kernel uses
// dynamic shared memory above 48 KB, so its attribute is raised before the
// occupancy query that sizes the persistent grid.
#pragma once
#include "lbm_kernels.cuh"

namespace aerosim {

// One time step: a single main_kernel launch.  Returns the number of launches in
// *launches.
template <class S, int MODE, int P>
cudaError_t step_entry(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ,
                       int* launches) {
  auto k = main_kernel<S, MODE, P>;
  if (occ) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, (int)(block.x * block.y), smem);
  }
  k<<<grid, block, smem, s>>>(a);
  if (launches) *launches = 1;
  return cudaGetLastError();
}

// The FP32-arithmetic kernels are compiled for every row pitch up to 256 (multiples
// of 32) with the pitch as a constant; other pitches and the double modes take the
// run-time pitch.
template <class S, int MODE>
cudaError_t step_dispatch(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ,
                          int* launches) {
  if constexpr (MODE == MODE_FAST) {
    switch (a.L.pitch) {
      case 32: return step_entry<S, MODE, 32>(a, block, grid, smem, s, occ, launches);
      case 64: return step_entry<S, MODE, 64>(a, block, grid, smem, s, occ, launches);
      case 96: return step_entry<S, MODE, 96>(a, block, grid, smem, s, occ, launches);
      case 128: return step_entry<S, MODE, 128>(a, block, grid, smem, s, occ, launches);
      case 160: return step_entry<S, MODE, 160>(a, block, grid, smem, s, occ, launches);
      case 192: return step_entry<S, MODE, 192>(a, block, grid, smem, s, occ, launches);
      case 224: return step_entry<S, MODE, 224>(a, block, grid, smem, s, occ, launches);
      case 256: return step_entry<S, MODE, 256>(a, block, grid, smem, s, occ, launches);
      default: break;
    }
  }
  return step_entry<S, MODE, 0>(a, block, grid, smem, s, occ, launches);
}

}  // namespace aerosim
