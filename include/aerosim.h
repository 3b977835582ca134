/*
 * aerosim.h -- C ABI of the B200-native AeroSim solver hot path (libaerosim.so).
 *
 * The library replaces the WebGPU compute path of the reference application
 * (necrolingus/aerosim): the D3Q19 regularized-BGK + Smagorinsky stream/collide
 * step with Bouzidi curved walls, the domain boundary conditions and mass
 * rescale, the momentum-exchange force reduction, and the BVH triangle
 * voxelizer.  Every entry point returns an int status (AEROSIM_OK == 0,
 * negative on error); aerosim_last_error() returns a message for the handle.
 *
 * Ownership: the caller owns every host buffer passed in or out; the library
 * owns all device memory behind an aerosim_engine handle.  Calls on one handle
 * are not thread-safe (the reference serialises steps with an isBusy flag,
 * src/solver/lbmEngine.ts:420,478).  Each handle owns one CUDA stream; every
 * call returns after its device work is complete.
 *
 * Cell indexing everywhere: idx = ix + nx * (iy + ny * iz); populations are
 * structure-of-arrays, direction d of cell idx at f[d * nx*ny*nz + idx]
 * (src/solver/lbmCpuReference.ts:138, shaders/collideStream.wgsl:2).
 */
#ifndef AEROSIM_H_
#define AEROSIM_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AEROSIM_ABI_VERSION 1

enum aerosim_status {
  AEROSIM_OK = 0,
  AEROSIM_ERR_ARG = -1,       /* invalid argument or inconsistent voxel grid */
  AEROSIM_ERR_STATE = -2,     /* call out of order (e.g. step before a voxel grid) */
  AEROSIM_ERR_CUDA = -3,      /* CUDA runtime error */
  AEROSIM_ERR_DEVICE = -4,    /* a kernel reported an error status */
  AEROSIM_ERR_NOMEM = -5,     /* device allocation failed */
  AEROSIM_ERR_FORMAT = -6     /* malformed input file (STL) */
};

/* Cell flags, src/geometry/voxelizer.ts:12-14 */
enum aerosim_cell_flag { AEROSIM_CELL_FLUID = 0, AEROSIM_CELL_SOLID = 1, AEROSIM_CELL_BOUNDARY = 2 };

/* Population storage / arithmetic of the solver. */
enum aerosim_precision {
  AEROSIM_PREC_F32 = 0,        /* FP32 storage of (f - w), FP32 collision (the production path) */
  AEROSIM_PREC_F32_MIRROR = 1, /* FP32 storage of f, FP64 arithmetic rounded exactly like the
                                  reference's JavaScript CPU solver (bit-parity mode) */
  AEROSIM_PREC_F16S = 2,       /* FP16 storage of (f - w) scaled by 2^15, FP32 collision */
  AEROSIM_PREC_BF16S = 3,      /* BF16 storage of (f - w), FP32 collision */
  AEROSIM_PREC_F64 = 4,        /* FP64 storage and arithmetic (the GPU FP64 oracle run) */
  AEROSIM_PREC_F16C = 5        /* F16S values with mass-compensated rounding: the rounding errors of a
                                  cell's 18 moving populations go into its rest population */
};

/* Element type for population read/write. */
enum aerosim_dtype { AEROSIM_DTYPE_F32 = 0, AEROSIM_DTYPE_F64 = 1 };

typedef struct aerosim_engine aerosim_engine;

/* TunnelDimensions, src/core/types.ts:73 */
typedef struct {
  double length, width, height; /* metres */
} aerosim_tunnel;

/* Scalar part of VoxelGridResult, src/geometry/voxelizer.ts:19-59 */
typedef struct {
  int32_t nx, ny, nz;
  double dx, dy, dz;
  double origin_x, origin_y, origin_z;
  int64_t solid_cell_count, boundary_cell_count, fluid_cell_count;
  double voxelization_time_ms;
} aerosim_voxel_info;

/* Solver part of LBMSolverConfig, src/solver/lbmEngine.ts:17-32 */
typedef struct {
  double u_inlet_lattice;          /* uInletLattice */
  double nu_lattice;               /* nuLattice */
  double smagorinsky_cs;           /* smagorinskyCs */
  int32_t ground_no_slip;          /* groundNoSlip */
  int32_t precision;               /* enum aerosim_precision */
  double frontal_area_m2;          /* frontalAreaM2 (A_ref) */
  double characteristic_length_m;  /* characteristicLengthM (L_ref) */
  aerosim_tunnel tunnel;           /* tunnel */
} aerosim_config;

/* Raw momentum-exchange sums (lattice units) and the normalized coefficients of
 * integrateLatticeMomentumExchange / computeNormalizedForceCoefficients,
 * src/solver/forceIntegrator.ts:106-315.  Moments are about the domain centre. */
typedef struct {
  double fx, fy, fz;
  double mx, my, mz;
  double cd_raw, cd, cl, cm, xcp;
  int64_t cut_face_links;
  int64_t step;
} aerosim_forces;

/* computeFluidMassStats, src/solver/lbmCpuReference.ts:461-495, plus the
 * cumulative product and count of the mean-density rescales (:434-455). */
typedef struct {
  double total_mass, mean_rho, max_speed;
  int32_t has_nan;
  int32_t reserved;
  double cumulative_rescale;
  int64_t rescale_count;
} aerosim_mass;

/* ---- lifetime ------------------------------------------------------------ */

/* new LBMEngine(device), src/solver/lbmEngine.ts:92.  device = CUDA ordinal. */
int aerosim_create(int device, aerosim_engine** out);
int aerosim_destroy(aerosim_engine* h);
/* Message of the last failing call on h (or of the last failing aerosim_create when
 * h is NULL).  The pointer stays valid until the next call on h. */
const char* aerosim_last_error(const aerosim_engine* h);
int aerosim_abi_version(void);

/* ---- geometry -> lattice ------------------------------------------------ */

/* voxelizeMeshToLattice(geometry, worldMatrix, tunnel, grid), voxelizer.ts:86-281,
 * run on the GPU.  positions: float xyz per vertex (BufferGeometry 'position');
 * indices: optional triangle index list (NULL for a triangle soup); world16:
 * optional column-major 4x4 matrix (THREE.Matrix4.elements) or NULL.  The result
 * stays on the device and becomes the engine's voxel grid, as setVoxelGrid would
 * install it (lbmEngine.ts:142-287); reset_flow re-initialises the populations. */
int aerosim_voxelize(aerosim_engine* h, const float* positions, int64_t vertex_count,
                     const int32_t* indices, int64_t index_count, const double* world16,
                     aerosim_tunnel tunnel, int32_t nx, int32_t ny, int32_t nz,
                     int32_t reset_flow, aerosim_voxel_info* out);

/* Copies the engine's voxel grid to host arrays (any pointer may be NULL):
 * flags u8[N], boundary_index_map i32[N], boundary_cells i32[B], q f32[B*18]
 * (index bIdx*18 + d-1), min_q f32[B]. */
int aerosim_read_voxel_grid(aerosim_engine* h, uint8_t* flags, int32_t* boundary_index_map,
                            int32_t* boundary_cells, float* q, float* min_q);
int aerosim_get_voxel_info(aerosim_engine* h, aerosim_voxel_info* out);

/* setVoxelGrid(voxel, config, resetFlow), lbmEngine.ts:142-287, from host arrays
 * of a VoxelGridResult.  boundary_index_map may be NULL (rebuilt from the list). */
int aerosim_set_voxel_grid(aerosim_engine* h, int32_t nx, int32_t ny, int32_t nz, double dx,
                           const double origin[3], const uint8_t* flags,
                           const int32_t* boundary_index_map, const int32_t* boundary_cells,
                           const float* q, int64_t boundary_count, int32_t reset_flow);

/* ---- solver --------------------------------------------------------------- */

/* updateConfig(config), lbmEngine.ts:289-300.  A precision change re-allocates the
 * population buffers and re-initialises the flow. */
int aerosim_set_config(aerosim_engine* h, const aerosim_config* cfg);
int aerosim_get_config(aerosim_engine* h, aerosim_config* cfg);
/* resetFlow(), lbmEngine.ts:677-688 (resetEquilibrium, lbmCpuReference.ts:114-143). */
int aerosim_reset_flow(aerosim_engine* h);
/* The substep loop of stepAndExtractSlice, lbmEngine.ts:483-527 (step(n),
 * lbmCpuReference.ts:145-156): n x (stream/collide, boundaries, mass rescale). */
int aerosim_step(aerosim_engine* h, int32_t n);
/* getStepCount(), lbmEngine.ts:690. */
int aerosim_get_step_count(aerosim_engine* h, int64_t* out);
/* Force readout of stepAndExtractSlice, lbmEngine.ts:555-658: FP64 momentum exchange
 * on the device, coefficients with the configured A_ref, L_ref and tunnel. */
int aerosim_read_forces(aerosim_engine* h, aerosim_forces* out);
/* macroField readback (readMacroField = true), lbmEngine.ts:577-625. */
int aerosim_read_macro(aerosim_engine* h, float* ux, float* uy, float* uz, float* rho);
/* Populations of the latest step (fSrc after the swap) as f32 or f64, 19*N values. */
int aerosim_read_populations(aerosim_engine* h, void* f, int32_t dtype);
int aerosim_write_populations(aerosim_engine* h, const void* f, int32_t dtype);
/* computeFluidMassStats, lbmCpuReference.ts:461-495. */
int aerosim_mass_stats(aerosim_engine* h, aerosim_mass* out);
/* extractSliceRGBA(axis, sliceFraction, fieldMode) of the macro fields of the last step
 * (src/solver/lbmCpuReference.ts:499-596, the image stepAndExtractSlice returns,
 * src/solver/lbmEngine.ts:548-553): axis 0 = x (width nz, height ny), 1 = y (nx, nz),
 * 2 = z (nx, ny); mode 0 = velocity, 1 = vorticity, 2 = pressure coefficient.  rgba:
 * width * height * 4 bytes, row v at v * width * 4; NULL only reports the size. */
int aerosim_extract_slice(aerosim_engine* h, int32_t axis, double fraction, int32_t mode, uint8_t* rgba,
                          int32_t* width, int32_t* height);
/* stepAndExtractSlice(substeps), lbmEngine.ts:404-675, as one call: n substeps, the
 * force readout (as aerosim_read_forces) and, when rgba is not NULL, the slice image
 * (as aerosim_extract_slice), with one synchronization instead of three. */
int aerosim_step_and_extract_slice(aerosim_engine* h, int32_t n, int32_t axis, double fraction, int32_t mode,
                                   uint8_t* rgba, int32_t* width, int32_t* height, aerosim_forces* forces);

/* ---- timing support -------------------------------------------------------- */

/* Device time of the last aerosim_step call in milliseconds (CUDA events on the
 * engine's stream) and the number of kernels it launched. */
int aerosim_last_step_timing(aerosim_engine* h, double* ms, int64_t* kernel_launches);

/* Bytes of solver parameters that travel host -> device with every step launch (the
 * kernel's argument block: step index, inlet velocity, tau, buffers).  The reference
 * uploads its SolverParams uniform (48 B) before every substep, lbmEngine.ts:330-354,484. */
int aerosim_step_param_bytes(void);

/* ---- failure path of the step kernels ----------------------------------------- */

/* Every ring wait of the step kernel (a consumer warp waiting for a bulk copy, the
 * producer waiting for a free slot) gives up after `polls` polls, sets the engine's
 * device error flag and lets the CTA return (after waiting, with the full limit, for
 * its own copies still in flight); the step call then returns AEROSIM_ERR_DEVICE and
 * aerosim_reset_flow clears the flag.  polls < 0 restores the default (2^22); 0 gives up
 * without polling, which makes the failure path run on purpose (tests).  The
 * reference's counterpart is the isBusy / null result of stepAndExtractSlice,
 * lbmEngine.ts:420, 593-600: a step that cannot complete reports it instead of hanging. */
int aerosim_set_pipeline_wait_limit(aerosim_engine* h, int32_t polls);

/* ---- allocation-free force reduction ------------------------------------------ */

/* Momentum-exchange forces (the reduction of aerosim_read_forces) over device buffers
 * the caller owns, without allocating any device memory.  No counterpart in the
 * reference: it serves hosts that own all device memory through their own allocator
 * and may not call cudaMalloc, and frame loops that cannot afford its synchronisation.
 * f: device float[19 * N], dense f[d * N + idx]; flags: device u8[N] (0 fluid, 1 solid,
 * 2 boundary); boundary_cells: device i32[B], each in [0, N) (not checked on the
 * device: an index outside the lattice reads out of bounds); q: device f32[B * 18],
 * q[b * 18 + d - 1] for link d of boundary_cells[b]; out: device double[8] = fx, fy, fz,
 * mx, my, mz (lattice units, moments about the domain centre), cut face links, CTAs
 * used (ceil(B / 256)).  stream: a cudaStream_t (NULL: the legacy default stream);
 * the work is enqueued, not waited for.  Limit: B <= 1 048 576 (4096 CTAs); larger B
 * returns AEROSIM_ERR_ARG.  Scratch is a fixed per-device array shared by all calls:
 * calls whose kernels overlap on the GPU race.  The first call on a device resolves the
 * array's address and should come before any stream capture on that device; after a
 * cudaDeviceReset the first call in the new context resolves it again.  Errors are
 * reported through aerosim_last_error(NULL). */
int aerosim_momentum_exchange_noalloc(const float* f, const uint8_t* flags, const int32_t* boundary_cells,
                                      const float* q, int64_t boundary_count, int32_t nx, int32_t ny,
                                      int32_t nz, double* out, void* stream);

/* ---- diagnostics of the flow field ------------------------------------------ */

/* computeQCriterion (src/render/vortexIso.ts:22-122) of the macro velocity of the last
 * step: Q = (|Omega|^2 - |S|^2) / 2 per cell, the vorticity magnitude and vector
 * (3 floats per cell), 0 at solid cells; maxima as the reference forms them (floor 1e-6).
 * Any output pointer may be NULL. */
int aerosim_q_criterion(aerosim_engine* h, float* q, float* omega_mag, float* omega_vec, double* max_q,
                        double* max_omega);
/* The same for caller velocity fields (host arrays, dense idx = ix + nx (iy + ny iz));
 * flags (0 fluid, 1 solid, 2 boundary) may be NULL. */
int aerosim_q_criterion_fields(aerosim_engine* h, int32_t nx, int32_t ny, int32_t nz, double dx, const float* ux,
                               const float* uy, const float* uz, const uint8_t* flags, float* q, float* omega_mag,
                               float* omega_vec, double* max_q, double* max_omega);

/* ---- learned subgrid-scale closure ----------------------------------------- */

/* A per-cell MLP (8 inputs -> 32 -> 32 -> 1, GELU; inputs: the strain rate estimated
 * from the non-equilibrium stress (6), density, wall distance) predicts nu_t / nu_0 in
 * place of the Smagorinsky eddy viscosity.  No counterpart in the reference, whose
 * closure is Smagorinsky only (src/solver/lbmCpuReference.ts:264-282); Smagorinsky
 * stays the fallback.  Parameter layout (aerosim_mlp_param_count() floats): W1[32][8],
 * b1[32], W2[32][32], b2[32], W3[32], b3.  The functions below take host arrays. */
int aerosim_mlp_param_count(void);
/* FP32 forward pass over n rows of X[n][8] (CUDA cores). */
int aerosim_mlp_forward(const float* params, const float* X, int64_t n, float* out);
/* The step kernel's evaluation: BF16 weights on the tensor cores, FP32 accumulation. */
int aerosim_mlp_forward_tc(const float* params, const float* X, int64_t n, float* out);
/* The same network on the 5th-generation tensor cores (tcgen05): 128-row tiles, BF16
 * operands in shared memory, FP32 accumulators in tensor memory.  No reference
 * counterpart.  AEROSIM_ERR_DEVICE when a tensor-core completion wait timed out. */
int aerosim_mlp_forward_umma(const float* params, const float* X, int64_t n, float* out);
/* Device time (CUDA events) of the kernel of the last aerosim_mlp_forward_tc /
 * aerosim_mlp_forward_umma call in this process. */
int aerosim_mlp_last_timing(double* ms);
/* Mean squared error against Y[n] and its gradient with respect to the parameters. */
int aerosim_mlp_gradients(const float* params, const float* X, const float* Y, int64_t n, float* grad,
                          double* loss);
/* Adam on the GPU: iters mini-batches of `batch` rows drawn by a seeded hash; params
 * in/out; loss_curve[iters] (may be NULL) receives each mini-batch loss. */
int aerosim_mlp_train(float* params, const float* X, const float* Y, int64_t n, int32_t iters, int32_t batch,
                      float lr, uint64_t seed, float* loss_curve);
/* params: the closure's weights for this engine's steps, NULL for Smagorinsky.  The
 * F32, F16S and BF16S precisions use it (near-wall Bouzidi cells keep Smagorinsky). */
int aerosim_set_sgs_mlp(aerosim_engine* h, const float* params);
/* Tensor-core path of the closure inside the step kernel.  AEROSIM_SGS_PATH_WARP: each
 * warp evaluates its 32 cells as BF16 mma.sync m16n8k16 tiles in registers (the default);
 * AEROSIM_SGS_PATH_TCGEN05: four consumer warps form one 128-cell tile, one thread issues
 * each layer as tcgen05.mma (M 128) with BF16 operands in shared memory and FP32
 * accumulators in tensor memory -- lattices with a row pitch of 128 or 256 (nx 97..256);
 * other lattices keep the warp path.  *in_use (may be NULL) receives the path the next
 * step will run (AEROSIM_SGS_PATH_DEFAULT when no closure is set).  No reference
 * counterpart. */
enum aerosim_sgs_path { AEROSIM_SGS_PATH_DEFAULT = 0, AEROSIM_SGS_PATH_WARP = 1, AEROSIM_SGS_PATH_TCGEN05 = 2 };
int aerosim_set_sgs_mlp_path(aerosim_engine* h, int32_t path, int32_t* in_use);
/* Euclidean distance (cells) of every cell centre to the nearest solid cell centre
 * (jump flooding), float[nx*ny*nz]. */
int aerosim_read_wall_distance(aerosim_engine* h, float* out);
/* Training samples of the closure from the flow of `fine` (its macro fields of the last
 * step) box-filtered onto `coarse`, whose lattice is exactly half as fine: per coarse
 * cell X[8] (filtered strain rate, density, wall distance as the closure sees them),
 * Y = nu_t / nu_0 of the least-squares eddy viscosity of the subgrid stress over the
 * (2 average_radius + 1)^3 neighbourhood (0..4), clipped to [min_ratio, max_ratio]
 * (-max_ratio <= min_ratio <= 0; 0 drops backscatter, a negative bound keeps it), and valid
 * (0 at solid, boundary-adjacent and edge cells). */
int aerosim_sgs_samples(aerosim_engine* fine, aerosim_engine* coarse, float min_ratio, float max_ratio,
                        int32_t average_radius, float* X, float* Y, uint8_t* valid);

/* ---- batches: many tunnels in one launch --------------------------------- */

/* A batch steps many wind-tunnel instances (angle-of-attack or specimen sweeps, uneven
 * lattice sizes) together: every step is ONE persistent kernel launch over the rows of
 * all instances, and runs of steps are replayed from a captured CUDA graph.  No
 * counterpart in the reference, which runs one tunnel per browser page; the instances
 * are ordinary engines, so every per-engine call (forces, macro field, populations,
 * mass statistics) works on them between batch steps. */
typedef struct aerosim_batch aerosim_batch;

/* Launch configuration of a batch, chosen by aerosim_batch_autotune or set by hand. */
typedef struct {
  int32_t stages;        /* shared-memory ring slots per CTA (2..6) */
  int32_t ctas_per_sm;   /* resident CTAs per SM of the persistent grid (1..3) */
  int32_t graph_steps;   /* launches per captured CUDA graph (1: no graph) */
  int32_t item_cells;    /* cells per work item: x-rows per item = clamp(item_cells / row span,
                            1, 8); 0 = 256 */
  double ms_per_step;    /* autotune: measured time of one batched step */
} aerosim_batch_tuning;

/* engines: n (1..64) engines on one device, each with a voxel grid, all with the same
 * FP32-arithmetic precision (F32, F16S or BF16S).  Resets the flow of every instance;
 * the engines must outlive the batch and must not be stepped alone while it exists
 * (per-engine reads are fine).  Errors: aerosim_last_error(NULL). */
int aerosim_batch_create(aerosim_engine* const* engines, int32_t n, aerosim_batch** out);
int aerosim_batch_destroy(aerosim_batch* b);
/* n steps of every instance; each engine's step count and readouts advance with it. */
int aerosim_batch_step(aerosim_batch* b, int32_t n);
/* Times every launch configuration that fits (work-item size 256 / 512 / 1024 cells x
 * ring depth x resident CTAs per SM) over steps_per_trial steps each, keeps the fastest,
 * then resets every instance's flow. */
int aerosim_batch_autotune(aerosim_batch* b, int32_t steps_per_trial, aerosim_batch_tuning* out);
int aerosim_batch_set_tuning(aerosim_batch* b, const aerosim_batch_tuning* t);
int aerosim_batch_get_tuning(aerosim_batch* b, aerosim_batch_tuning* out);
/* The ring-wait limit of the batched step kernel, as aerosim_set_pipeline_wait_limit;
 * a failed step returns AEROSIM_ERR_DEVICE until the next autotune resets the batch. */
int aerosim_batch_set_pipeline_wait_limit(aerosim_batch* b, int32_t polls);
/* Device time (CUDA events) and kernel launches of the last aerosim_batch_step call. */
int aerosim_batch_last_timing(aerosim_batch* b, double* ms, int64_t* kernel_launches);
/* Cells of all instances (the MLUPS numerator of one batched step). */
int aerosim_batch_cells(aerosim_batch* b, int64_t* out);

/* ---- host-side geometry inputs ------------------------------------------- */

/* computeProjectedFrontalArea(geometry, worldMatrix, gridResolution),
 * src/geometry/frontalArea.ts:22-179 (A_ref). */
int aerosim_frontal_area(const float* positions, int64_t vertex_count, const int32_t* indices,
                         int64_t index_count, const double* world16, int32_t grid_resolution,
                         double* out);

/* The same raster as a CUDA kernel on `device` (one warp per triangle, coverage bits
 * OR'ed per pixel); returns the host raster's area bit for bit.  grid_resolution is
 * at most 16384.  Errors: aerosim_last_error(NULL). */
int aerosim_frontal_area_cuda(int32_t device, const float* positions, int64_t vertex_count,
                              const int32_t* indices, int64_t index_count, const double* world16,
                              int32_t grid_resolution, double* out);

/* Formats told apart by aerosim_parse_stl. */
enum aerosim_stl_format { AEROSIM_STL_BINARY = 0, AEROSIM_STL_ASCII = 1 };

/* parseSTL(buffer), src/geometry/stlLoader.ts:9-38 (parseBinarySTL :40-75,
 * parseAsciiSTL :77-95): the triangle soup's vertex positions, float32 xyz per vertex.
 * With positions == NULL only *vertex_count (and *format) are set; otherwise
 * capacity_vertices must hold *vertex_count.  The reference's exceptions ("Invalid or
 * corrupted STL file.", "ASCII STL file contains no valid triangles.") become
 * AEROSIM_ERR_FORMAT with that message in aerosim_last_error(NULL). */
int aerosim_parse_stl(const uint8_t* bytes, int64_t byte_count, float* positions,
                      int64_t capacity_vertices, int64_t* vertex_count, int32_t* format);

/* normalizeAndCenterGeometry(geometry), stlLoader.ts:101-127, in place: centre the
 * bounding box on the origin, then scale by 0.001 (largest side > 50) or to unit size
 * (largest side in (10, 50]); *auto_scaled_from_mm (optional) is 1 when it scaled. */
int aerosim_normalize_and_center(float* positions, int64_t vertex_count, int32_t* auto_scaled_from_mm);

/* ModelTransform, src/core/types.ts:99-103 (Euler XYZ angles in degrees). */
typedef struct {
  double position[3];
  double rotation_deg[3];
  double scale[3];
} aerosim_model_transform;

/* MeshStats, src/core/types.ts:105-115 (the name stays with the caller). */
typedef struct {
  int64_t triangle_count;
  int64_t vertex_count;
  int64_t open_edge_count;
  int32_t is_watertight;
  int32_t reserved;
  double bounding_box_size[3];  /* world-space size after the transform */
  double characteristic_length; /* L_ref = max(1e-4, size x) */
  double frontal_area;          /* A_ref, 512 x 512 raster */
  double volume;
} aerosim_mesh_stats;

/* The world matrix computeMeshStats builds from a ModelTransform
 * (Matrix4.compose of position, the XYZ-Euler quaternion and scale,
 * stlLoader.ts:142-153); column-major like world16 everywhere in this header. */
int aerosim_model_matrix(const aerosim_model_transform* transform, double* world16);

/* computeMeshStats(geometry, name, transform), stlLoader.ts:133-244: welded-edge
 * watertightness (vertices quantised to 1e-5, meshes of at most 100 000 triangles),
 * world bounding box, L_ref, |signed volume|, and A_ref from the CUDA raster on
 * `device` (device < 0: the host raster). */
int aerosim_compute_mesh_stats(const float* positions, int64_t vertex_count, const int32_t* indices,
                               int64_t index_count, const aerosim_model_transform* transform,
                               int32_t device, aerosim_mesh_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* AEROSIM_H_ */
