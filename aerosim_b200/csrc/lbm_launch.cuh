// Launch helpers shared by the kernel translation units: the step kernels use
// dynamic shared memory above 48 KB, so their limit is raised before the occupancy
// query that sizes the persistent grid.
#pragma once
#include "lbm_kernels.cuh"
#include "lbm_batch.cuh"

namespace aerosim {

// Raises a kernel's dynamic shared-memory limit to the device's opt-in maximum.  The
// limit belongs to the kernel, not to a launch, so engines that share a kernel instance
// with different ring sizes must never lower it below what another engine launches with.
// (The maximum is the opt-in per-block size less the kernel's static shared memory.)
template <class K>
cudaError_t raise_smem_limit(K k) {
  int dev = 0, mx = 0;
  cudaFuncAttributes fa{};
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, mx - (int)fa.sharedSizeBytes);
  return e;
}

// One time step: a single main_kernel launch.  Returns the number of launches in
// *launches.
template <class S, int MODE, int P, int MLP = MLP_NONE, int CPT = 1>
cudaError_t step_entry(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ,
                       int* launches) {
  auto k = main_kernel<S, MODE, P, MLP, CPT>;
  if (occ) {
    cudaError_t e = raise_smem_limit(k);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, (int)(block.x * block.y), smem);
  }
  // programmatic dependent launch: the CTAs of a step may start (and run their
  // shared-memory prologue) while the previous step's last CTAs finish
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k, a);
  if (launches) *launches = 1;
  return e != cudaSuccess ? e : cudaGetLastError();
}

// The FP32-arithmetic kernels are compiled for every row pitch up to 256 (multiples
// of 32) with the pitch as a constant; other pitches and the double modes take the
// run-time pitch.  With the learned closure (a.mlp_frag set): pitches 128 and 256, or
// the run-time pitch, as warp-level mma.sync tiles; with a.mlp_umma set as well, the
// 128-cell tcgen05 tiles, for pitches 128 and 256 (rows of 97..256 cells: every item
// keeps all 8 consumer warps busy, two full groups of four).
template <class S, int MODE>
cudaError_t step_dispatch(const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s, int* occ,
                          int* launches) {
  if constexpr (MODE == MODE_FAST) {
    if (a.mlp_frag && a.mlp_umma) {
      switch (a.L.pitch) {
        case 128: return step_entry<S, MODE, 128, MLP_TCGEN05>(a, block, grid, smem, s, occ, launches);
        case 256: return step_entry<S, MODE, 256, MLP_TCGEN05>(a, block, grid, smem, s, occ, launches);
        default: return cudaErrorInvalidValue;
      }
    }
    if (a.mlp_frag) {
      switch (a.L.pitch) {
        case 128: return step_entry<S, MODE, 128, MLP_WARP>(a, block, grid, smem, s, occ, launches);
        case 256: return step_entry<S, MODE, 256, MLP_WARP>(a, block, grid, smem, s, occ, launches);
        default: return step_entry<S, MODE, 0, MLP_WARP>(a, block, grid, smem, s, occ, launches);
      }
    }
    if (a.cells_per_thread == 2) {  // two cells per thread (even nx)
      switch (a.L.pitch) {
        case 32: return step_entry<S, MODE, 32, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        case 64: return step_entry<S, MODE, 64, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        case 96: return step_entry<S, MODE, 96, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        case 128: return step_entry<S, MODE, 128, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        case 160: return step_entry<S, MODE, 160, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        case 192: return step_entry<S, MODE, 192, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        case 224: return step_entry<S, MODE, 224, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        case 256: return step_entry<S, MODE, 256, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
        default: return step_entry<S, MODE, 0, MLP_NONE, 2>(a, block, grid, smem, s, occ, launches);
      }
    }
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

// One step of a batch (batch_kernel) for a row pitch P (0: run time) and CPT cells per
// consumer thread.
template <class S, int P, int CPT>
cudaError_t batch_entry(const BatchArgs& b, unsigned grid, size_t smem, cudaStream_t s, int* occ) {
  auto k = batch_kernel<S, P, CPT>;
  if (occ) {
    cudaError_t e = raise_smem_limit(k);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, kStepThreads, smem);
  }
  k<<<grid, kStepThreads, smem, s>>>(b);
  return cudaGetLastError();
}

template <class S, int CPT>
cudaError_t batch_dispatch_cpt(const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s, int* occ) {
  switch (pitch) {
    case 64: return batch_entry<S, 64, CPT>(b, grid, smem, s, occ);
    case 128: return batch_entry<S, 128, CPT>(b, grid, smem, s, occ);
    case 192: return batch_entry<S, 192, CPT>(b, grid, smem, s, occ);
    case 256: return batch_entry<S, 256, CPT>(b, grid, smem, s, occ);
    default: return batch_entry<S, 0, CPT>(b, grid, smem, s, occ);
  }
}

// One step of a batch (batch_kernel).  pitch: the row pitch shared by every instance,
// or 0 when the instances differ (the kernel then reads each instance's pitch).
template <class S>
cudaError_t batch_dispatch(const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s, int* occ) {
  return b.cells_per_thread == 2 ? batch_dispatch_cpt<S, 2>(b, pitch, grid, smem, s, occ)
                                 : batch_dispatch_cpt<S, 1>(b, pitch, grid, smem, s, occ);
}

}  // namespace aerosim
