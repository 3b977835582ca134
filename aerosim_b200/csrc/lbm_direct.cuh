// Direct-pull step kernel: the FP32-arithmetic step with two cells per thread (pair_segment)
// whose consumer warps pull their populations straight from global memory instead of a
// shared-memory ring filled by bulk copies.
//
// The ring of main_kernel stages each destination row's 9 source-row pieces with 1-D bulk
// copies; with 16-bit storage those pieces are 512 B and 1.5 KB, and the ring's pull bounds
// the step (the FP16S ring skeleton, without collision and without stores, takes 67 us at
// 256x128x128).  Here every warp takes whole x-rows from the step's counter and loads, per
// 64-cell segment, the 19 source values of its two cells directly: one aligned 4- or 8-byte
// load per direction with c_x = 0, two element loads for c_x = +-1, coalesced over the warp.
// No producer warp and no ring: the latency is hidden by the warps in flight.  The near-wall
// cells stay with a helper warp per CTA (near_cell), the mean-density rescale with the last
// CTA, exactly as in main_kernel; the cell semantics are pair_segment's.
#pragma once
#include "lbm_kernels.cuh"

namespace aerosim {

constexpr int kDirectConsumerWarps = 7;
constexpr int kDirectThreads = (kDirectConsumerWarps + 1) * 32;  // + the near-wall helper warp

// Dynamic shared memory: inlet tables ux_in[ny], uy_in[ny]; per consumer warp a 24-float
// scratch row (the outlet's parked sources); the direction table of the lane-transposed
// row ends (c, w; slot).
__host__ __device__ inline size_t direct_smem_bytes(const Layout& L) {
  return 2 * (size_t)L.ny * sizeof(double) + kDirectConsumerWarps * 24 * sizeof(float) + 16 +
         19 * sizeof(float4) + 19 * sizeof(int);
}

template <class S, int P>
__global__ void __launch_bounds__(kDirectThreads, 2) direct_kernel(const __grid_constant__ StepArgs a) {
  using T = typename S::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long red[kDirectConsumerWarps + 1];
  __shared__ int nan_flag;
  __shared__ int is_last;

  const Layout& L = a.L;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int pitch = P ? P : L.pitch;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long rows = (long long)ny * nz;
  const bool reverse = (a.step_index & 1) != 0;  // odd steps walk the rows last to first (L2 reuse)
  const int cur_slot = a.step_index & 1;

  double* s_uxi = reinterpret_cast<double*>(smem_raw);
  double* s_uyi = s_uxi + ny;
  float* s_xo = reinterpret_cast<float*>(s_uyi + ny);  // [kDirectConsumerWarps][24]
  float4* s_dcw = reinterpret_cast<float4*>(
      (reinterpret_cast<uintptr_t>(s_xo + kDirectConsumerWarps * 24) + 15) & ~uintptr_t(15));  // [19]
  int* s_dslot = reinterpret_cast<int*>(s_dcw + 19);                                            // [19]

  if (threadIdx.x == 0) nan_flag = 0;
  if (threadIdx.x < 19) {  // direction table of the lane-transposed row ends
    const int d = threadIdx.x;
    float cx = 0.f, cy = 0.f, cz = 0.f;
    int sl = d;
#pragma unroll
    for (int e = 0; e < 19; ++e)
      if (e == d) {
        cx = (float)cx_of(e); cy = (float)cy_of(e); cz = (float)cz_of(e);
        sl = slot_of(e);
      }
    s_dcw[d] = make_float4(cx, cy, cz, d == 0 ? 1.0f / 3.0f : (d <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f));
    s_dslot[d] = sl;
  }
  for (int i = threadIdx.x; i < ny; i += blockDim.x) {  // inlet velocity per iy (:334-342)
    double uxi = a.u_inlet;
    if (a.ground_no_slip) uxi = a.u_inlet * a.abl[i];
    double uyi = 0.0;
    if (a.step_index < 120) uyi = 0.015 * a.u_inlet * a.sin_tab[(long long)a.step_index * ny + i];
    s_uxi[i] = uxi;
    s_uyi[i] = uyi;
  }
  __syncthreads();
  // programmatic dependent launch, as in main_kernel: the previous step must be complete
  // before this one reads or writes global memory
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  long long my_sum = 0;
  const T* __restrict__ fs = static_cast<const T*>(a.fsrc);
  T* __restrict__ fd = static_cast<T*>(a.fdst);
  const int pslot = (a.step_index + 1) & 1;  // pending rescale of the previous step
  const double corr = a.st->apply[pslot] ? a.st->corr[pslot] : 1.0;

  if (warp == kDirectConsumerWarps) {
    // ---------------- helper warp: this CTA's share of the near-wall cells ----------------
    int my_nan = 0;
    for (long long t = (long long)blockIdx.x * 32 + lane; t < a.n_near; t += (long long)gridDim.x * 32)
      my_sum += near_cell<S, MODE_FAST, P>(a, a.fsrc, a.fdst, a.write_macro, t, corr,
                                           [&](int y) { return make_double2(s_uxi[y], s_uyi[y]); }, &my_nan);
    if (__any_sync(0xffffffffu, my_nan) && lane == 0) nan_flag = 1;
  } else {
    // ---------------- consumer warps: whole x-rows from the step's counter ----------------
    const float corrf = (float)corr;
    const float2 dec = make_float2(corrf * S::kRawScale, corrf - 1.0f);  // raw-moment decode
    const int nseg = (nx + 63) / 64;
    const float tau0 = (float)a.tau0, k_smag = (float)a.k_smag;
    auto inlet = [&](int y) { return make_float2((float)s_uxi[y], (float)s_uyi[y]); };
    float* xo = s_xo + warp * 24;
    int my_nan = 0;
    for (;;) {
      long long k = 0;
      if (lane == 0) k = (long long)atomicAdd(&a.st->next_item[cur_slot], 1u);
      k = __shfl_sync(0xffffffffu, k, 0);
      if (k >= rows) break;
      const long long row = reverse ? rows - 1 - k : k;
      const int iy = (int)(row % ny), iz = (int)(row / ny);
      const bool wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));
      // element offset of each direction group's source row block (the clamped pull,
      // lbmCpuReference.ts:189-195): slot s of group g sits at rb[g] + s * pitch
      long long rb[kGroups];
#pragma unroll
      for (int g = 0; g < kGroups; ++g)
        rb[g] = ((long long)clampi(iy - group_cy(g), 0, ny - 1) +
                 (long long)ny * clampi(iz - group_cz(g), 0, nz - 1)) * 19 * pitch;
      const uint8_t* crow = a.cls + row * pitch;
      for (int c = 0; c < nseg; ++c) {
        const int cell_lo = c * 64;
        const int x0 = cell_lo + 2 * lane;
        const bool active = x0 < nx;
        const int lx = active ? x0 : 0;  // lanes outside the row read cells 0 and 1
        const uint32_t cls2 = *reinterpret_cast<const uint16_t*>(crow + lx);
        float2 v[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) {
          const int sl = slot_of(d);
          const T* q = fs + rb[sl < 15 ? sl / 3 : sl - 10] + (long long)sl * pitch + lx;
          if (cx_of(d) == 0) v[d] = load_pair<S>(q);
          else v[d] = make_float2(S::raw(q[-cx_of(d)]), S::raw(q[1 - cx_of(d)]));
        }
        PairGeom g;
        g.row = row; g.nx = nx; g.ny = ny; g.nz = nz; g.pitch = pitch;
        g.iy = iy; g.iz = iz; g.x0 = x0; g.cell_lo = cell_lo; g.active = active;
        g.has_lo = cell_lo == 0;
        g.has_hi = cell_lo <= nx - 2 && nx - 2 < cell_lo + 64;
        g.wall_row = wall_row; g.ground_no_slip = a.ground_no_slip; g.write_macro = a.write_macro;
        g.c0 = (uint8_t)(cls2 & 0xffu);
        g.c1 = (uint8_t)(cls2 >> 8);
        pair_segment<S>(v, fd, g, tau0, k_smag, dec, inlet, a, xo, s_dcw, s_dslot, lane, my_sum, my_nan);
      }
    }
    if (__any_sync(0xffffffffu, my_nan) && lane == 0) nan_flag = 1;
  }

#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_sum += __shfl_down_sync(0xffffffffu, my_sum, o);
  if (lane == 0) red[warp] = my_sum;
  __syncthreads();
  const int slot = a.step_index & 1;
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w <= kDirectConsumerWarps; ++w) s += red[w];
    if (nan_flag) a.st->nan_seen = 1;
    if (s) atomicAdd(&a.st->rho_sum[slot], (unsigned long long)s);
    __threadfence();
    const unsigned int tk = atomicAdd(&a.st->ticket[slot], 1u);
    is_last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  // ---- mean-density rescale (:431-455): the last CTA takes the decision ----
  if (is_last && threadIdx.x == 0) {
    __threadfence();
    const long long total = (long long)atomicAdd(&a.st->rho_sum[slot], 0ull);
    int ap = 0;
    double cr = 1.0;
    if (a.fluid_count > 0) {
      const double mean = rho_unfixed(total, 0.0f) / (double)a.fluid_count;
      cr = 1.0 / mean;
      ap = fabs(mean - 1.0) > 1e-4 ? 1 : 0;
    }
    a.st->corr[slot] = cr;
    a.st->apply[slot] = ap;
    if (ap) {
      a.st->cumulative_rescale *= cr;
      a.st->rescale_count += 1;
    }
    // accumulators of the next step start from zero
    a.st->rho_sum[slot ^ 1] = 0ull;
    a.st->ticket[slot ^ 1] = 0u;
    a.st->next_item[slot ^ 1] = 0u;
  }
}

// One step with the direct-pull kernel (occ != nullptr: resident CTAs per SM only).
template <class S, int P>
cudaError_t direct_entry(const StepArgs& a, unsigned grid, size_t smem, cudaStream_t s, int* occ) {
  auto k = direct_kernel<S, P>;
  if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, kDirectThreads, smem);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kDirectThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, a);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <class S>
cudaError_t direct_dispatch(const StepArgs& a, unsigned grid, size_t smem, cudaStream_t s, int* occ) {
  switch (a.L.pitch) {
    case 64: return direct_entry<S, 64>(a, grid, smem, s, occ);
    case 128: return direct_entry<S, 128>(a, grid, smem, s, occ);
    case 192: return direct_entry<S, 192>(a, grid, smem, s, occ);
    case 256: return direct_entry<S, 256>(a, grid, smem, s, occ);
    default: return direct_entry<S, 0>(a, grid, smem, s, occ);
  }
}

}  // namespace aerosim
