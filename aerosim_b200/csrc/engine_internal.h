// Internal interfaces between the C-ABI layer and the kernel translation units.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "common.cuh"

namespace aerosim {

struct StepArgs;
struct ForceArgs;
struct BatchArgs;

// A voxel grid resident on the device (VoxelGridResult, voxelizer.ts:19-59).
struct DevGrid {
  int nx = 0, ny = 0, nz = 0;
  long long N = 0;
  double h = 0, ox = 0, oy = 0, oz = 0;
  uint8_t* flags = nullptr;   // reference flags
  uint8_t* cls = nullptr;     // solver cell classes
  int32_t* bmap = nullptr;    // boundaryIndexMap
  int32_t* bcells = nullptr;  // boundaryCellIndices
  float* q = nullptr;         // boundaryQValues [B * 18]
  float* minq = nullptr;      // boundaryMinQ
  long long B = 0, solid = 0;
  int window[6] = {0, 0, 0, 0, 0, 0};
  double vox_ms = 0;
};

// voxelize.cu
int run_voxelizer(const float* pos, int64_t nverts, const int32_t* idx, int64_t nidx,
                  const double* world16, double tunnel_height, int nx, int ny, int nz,
                  cudaStream_t s, DevGrid* g, std::string* err);

// Message returned by aerosim_last_error(NULL) (calls that take no engine handle).
void set_global_error(const std::string& msg);

// Element size of the population storage of a precision mode.
size_t precision_bytes(int precision);

// lbm_fast.cu / lbm_exact.cu
// occ != nullptr: only query the resident CTAs per SM (and raise the shared-memory
// attribute) for this block and dynamic shared-memory size.
cudaError_t launch_step(int precision, const StepArgs& a, dim3 block, unsigned grid, size_t smem, cudaStream_t s,
                        int* occ, int* launches);
// One batched step (FP32-arithmetic precisions only); pitch: the instances' common row
// pitch or 0.  occ != nullptr: occupancy query as for launch_step.
cudaError_t launch_batch(int precision, const BatchArgs& b, int pitch, unsigned grid, size_t smem, cudaStream_t s,
                         int* occ);
cudaError_t launch_forces(int precision, const ForceArgs& a, unsigned grid, cudaStream_t s);
cudaError_t launch_classify(const uint8_t* flags, uint8_t* cls, const Layout& L, cudaStream_t s);
cudaError_t launch_init(int precision, void* f0, void* f1, const uint8_t* cls, float* mux, float* muy,
                        float* muz, float* mrho, const double* abl, const Layout& L, double u_inlet,
                        int ground_no_slip, cudaStream_t s);
cudaError_t launch_read_pops(int precision, const void* f, const uint8_t* cls, const StepState* st,
                             int prev_slot, const Layout& L, long long N, void* out, int dtype,
                             cudaStream_t s);
cudaError_t launch_write_pops(int precision, void* f, const Layout& L, long long N, const void* in,
                              int dtype, cudaStream_t s);
cudaError_t launch_materialize(int precision, void* f, const uint8_t* cls, const StepState* st,
                               int prev_slot, const Layout& L, long long N, cudaStream_t s);
cudaError_t launch_read_macro(const float* mrho, const uint8_t* cls, const StepState* st, int prev_slot,
                              const Layout& L, long long N, float* rho_out, cudaStream_t s);
cudaError_t launch_mass_stats(const float* mux, const float* muy, const float* muz, const float* rho,
                              const uint8_t* cls, const StepState* st, int prev_slot, const Layout& L,
                              long long N, unsigned long long* out, cudaStream_t s);

// Slice image of the macro fields (extractSliceRGBA): RGBA bytes [height][width].
cudaError_t launch_slice(const float* mux, const float* muy, const float* muz, const float* mrho,
                         const uint8_t* cls, const StepState* st, int prev_slot, const Layout& L, int axis, int fixed,
                         int mode, double uref, int width, int height, uint8_t* rgba, cudaStream_t s);

// computeQCriterion over dense float velocity fields (flags may be null); maxima[2]
// receive the bit patterns of max Q and max |omega| before the reference's 1e-6 floor.
cudaError_t launch_q_criterion(int nx, int ny, int nz, double dx, const float* ux, const float* uy, const float* uz,
                               const uint8_t* flags, float* q, float* om, float* omv, unsigned long long* maxima,
                               cudaStream_t s);

// sgs.cu: jump-flood wall distance of a dense flag array into float distances (dist,
// may be null) and bits 3..7 of the pitched class bytes (cls, may be null); training
// samples of the learned closure from a fine flow's macro fields and a 2x coarser grid.
cudaError_t compute_wall_distance(const uint8_t* flags, int nx, int ny, int nz, float* dist, uint8_t* cls, int pitch,
                                  cudaStream_t s);
cudaError_t launch_sgs_samples(const float* ux, const float* uy, const float* uz, const float* rho,
                               const uint8_t* fflags, int fx, int fy, int fz, const uint8_t* ccls, int cpitch, int cx,
                               int cy, int cz, float nu0, float min_ratio, float max_ratio, int avg, float* X,
                               float* Y, uint8_t* valid, cudaStream_t s);

}  // namespace aerosim
