// Batched step kernel: many wind-tunnel instances of uneven lattice sizes advance one
// time step in ONE persistent launch.  The items (x-row groups) of all instances form
// one flat work list; a CTA walks it with the producer / consumer / near-wall warp
// roles of main_kernel, switching the instance's arguments per item and dealing the
// 32-cell segments of an item to the consumer warps cyclically.  Each instance
// keeps its own mean-density rescale: CTAs write per-instance partial density sums and
// the last CTA takes every instance's decision.  The step counter lives in device
// memory and the ping-pong buffers are selected by its parity, so a CUDA graph of
// launches can be replayed without changing a kernel argument.
#pragma once
#include "lbm_kernels.cuh"

namespace aerosim {

constexpr int kMaxBatch = 64;  // instances per batch
constexpr int kMaxRowsPerItem = kConsumerWarps;

struct BatchArgs {
  const StepArgs* inst;          // [n_inst] solver arguments of each instance (its buffers,
                                 //   step index and macro flag come from the fields below)
  void* const* bufs;             // [2 * n_inst] population buffers 0 and 1 of instance k
  const long long* item_begin;   // [n_inst + 1] first item of each instance in the flat list
  const long long* near_begin;   // [n_inst + 1] first near-wall cell of each instance
  unsigned long long* partials;  // [gridDim.x * n_inst] per-CTA fixed-point density sums
  unsigned int* ticket;          // [2] CTAs done, per step parity
  const int4* geo;               // [n_inst] rows per item, 32-cell segments per row, row shift
  int* step;                     // step counter shared by all instances
  int* error;                    // pipeline timeout flag of the batch
  long long n_items, n_near;
  long long slot_elems;          // ring slot stride (elements) and class-byte slot stride
  long long slot_cls;
  int n_inst, stages, write_macro;
  int cells_per_thread;          // 1, or 2 when every instance has an even nx
  int wait_limit;                // polls of a ring wait before the step gives up (as StepArgs)
};

__device__ __forceinline__ int find_instance(const long long* begin, int n, long long x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (begin[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Shared memory of the batched kernel: like main_kernel, with ring slots sized for
// the largest item of the batch and the instance index of every slot.
__host__ __device__ inline size_t batch_smem_bytes(long long slot_elems, long long slot_cls, int stages,
                                                    size_t elem) {
  return kSmemGuard + (size_t)stages * ((size_t)slot_elems * elem + (size_t)slot_cls) + kSmemGuard + 16 +
         16 * (size_t)stages + (size_t)stages * kMaxRowsPerItem * sizeof(int2) + (size_t)stages * sizeof(int) +
         kConsumerWarps * 24 * sizeof(float) + 16 + 19 * sizeof(float4) + 19 * sizeof(int);
}

// CPT: consumer cells per thread, 1 or 2 (pair_segment; every instance with an even nx).
template <class S, int P, int CPT = 1>
__global__ void __launch_bounds__(kStepThreads, step_min_blocks<S, MODE_FAST, MLP_NONE, CPT>())
    batch_kernel(const __grid_constant__ BatchArgs b) {
  using T = typename S::T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ unsigned long long s_sum[kMaxBatch];  // this CTA's density sum per instance
  __shared__ int is_last;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S_ = b.stages;
  const int step = *b.step;  // every CTA reads it before the last CTA advances it
  const int cur = step & 1;  // buffer parity of this step's source populations
  const int pslot = (step + 1) & 1;
  const int my_count =
      blockIdx.x < b.n_items ? (int)((b.n_items - 1 - blockIdx.x) / gridDim.x + 1) : 0;

  T* spop = reinterpret_cast<T*>(smem_raw + kSmemGuard);
  uint8_t* scls = smem_raw + kSmemGuard + (size_t)S_ * b.slot_elems * sizeof(T);
  uint64_t* full = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(scls + (size_t)S_ * b.slot_cls + kSmemGuard) + 7) & ~uintptr_t(7));
  uint64_t* empty = full + S_;
  int2* s_row = reinterpret_cast<int2*>(empty + S_);            // [S_][kMaxRowsPerItem]
  int* s_inst = reinterpret_cast<int*>(s_row + S_ * kMaxRowsPerItem);  // [S_]
  float* s_xo = reinterpret_cast<float*>(s_inst + S_);          // [kConsumerWarps][24]
  float4* s_dcw = reinterpret_cast<float4*>(
      (reinterpret_cast<uintptr_t>(s_xo + kConsumerWarps * 24) + 15) & ~uintptr_t(15));
  int* s_dslot = reinterpret_cast<int*>(s_dcw + 19);

  if (threadIdx.x == 0) {
    for (int s = 0; s < S_; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);  // every consumer warp arrives, with or without a row
    }
    mbar_fence_init();
  }
  for (int k = threadIdx.x; k < b.n_inst; k += blockDim.x) s_sum[k] = 0ull;
  if (threadIdx.x < 19) {  // direction table of the lane-transposed row ends
    const int d = threadIdx.x;
    const int px = (1 << 1) | (1 << 7) | (1 << 9) | (1 << 11) | (1 << 13);
    const int mx_ = (1 << 2) | (1 << 8) | (1 << 10) | (1 << 12) | (1 << 14);
    const int py = (1 << 3) | (1 << 7) | (1 << 10) | (1 << 15) | (1 << 17);
    const int my_ = (1 << 4) | (1 << 8) | (1 << 9) | (1 << 16) | (1 << 18);
    const int pz = (1 << 5) | (1 << 11) | (1 << 14) | (1 << 15) | (1 << 18);
    const int mz_ = (1 << 6) | (1 << 12) | (1 << 13) | (1 << 16) | (1 << 17);
    const float w = d == 0 ? 1.0f / 3.0f : (d <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f);
    s_dcw[d] = make_float4((float)(((px >> d) & 1) - ((mx_ >> d) & 1)), (float)(((py >> d) & 1) - ((my_ >> d) & 1)),
                           (float)(((pz >> d) & 1) - ((mz_ >> d) & 1)), w);
    int sl = d;
#pragma unroll
    for (int e = 0; e < 19; ++e)
      if (e == d) sl = slot_of(e);
    s_dslot[d] = sl;
  }
  __syncthreads();

  // inlet velocity of row y of an instance (:334-342) at this step
  auto inlet_of = [&](const StepArgs& ia, int y) -> double2 {
    double ux = ia.u_inlet;
    if (ia.ground_no_slip) ux = ia.u_inlet * ia.abl[y];
    double uy = 0.0;
    if (step < 120) uy = 0.015 * ia.u_inlet * ia.sin_tab[(long long)step * ia.L.ny + y];
    return make_double2(ux, uy);
  };
  bool failed = false;

  if (warp == kHelperWarp) {
    // ---------------- near-wall cells of all instances ----------------
    int my_nan = 0;
    for (long long t = (long long)blockIdx.x * 32 + lane; t < b.n_near; t += (long long)gridDim.x * 32) {
      const int k = find_instance(b.near_begin, b.n_inst, t);
      const StepArgs& ia = b.inst[k];
      const double corr = ia.st->apply[pslot] ? ia.st->corr[pslot] : 1.0;
      const long long add = near_cell<S, MODE_FAST, P>(ia, b.bufs[2 * k + cur], b.bufs[2 * k + (cur ^ 1)],
                                                       b.write_macro, t - b.near_begin[k], corr,
                                                       [&](int y) { return inlet_of(ia, y); }, &my_nan);
      atomicAdd(&s_sum[k], (unsigned long long)add);
      if (my_nan) {
        ia.st->nan_seen = 1;
        my_nan = 0;
      }
    }
  } else if (warp == kProducerWarp) {
    // ---------------- producer warp ----------------
    int issued = 0;
    int s = 0;
    uint32_t ph = 0;
    for (int j = 0; j < my_count; ++j) {
      if (j >= S_) {
        const bool ok = mbar_wait(&empty[s], ph ^ 1u, b.wait_limit);
        if (!__any_sync(0xffffffffu, ok)) {
          failed = true;
          break;
        }
      }
      const long long gi = blockIdx.x + (long long)j * gridDim.x;
      const int k = find_instance(b.item_begin, b.n_inst, gi);
      const StepArgs& ia = b.inst[k];
      const int ny = ia.L.ny, nz = ia.L.nz;
      const int pitch = P ? P : ia.L.pitch;
      const int RY = b.geo[k].x;
      const long long rows = (long long)ny * nz;
      const long long r0 = (gi - b.item_begin[k]) * RY;
      const int nr = (int)(rows - r0 < RY ? rows - r0 : RY);
      const uint32_t slot_bytes = (uint32_t)(pitch * sizeof(T));
      if (lane == 0) {
        for (int yy = 0; yy < nr; ++yy) {
          const int r = (int)(r0 + yy);
          s_row[s * kMaxRowsPerItem + yy] = make_int2(r % ny, r / ny);
        }
        s_inst[s] = k;
        mbar_arrive_expect_tx(&full[s], (uint32_t)nr * (19u * slot_bytes + (uint32_t)pitch));
      }
      __syncwarp();
      const T* fs = static_cast<const T*>(b.bufs[2 * k + cur]);
      T* sbase = spop + (size_t)s * b.slot_elems;
      uint8_t* cbase = scls + (size_t)s * b.slot_cls;
      for (int c = lane; c < nr * 10; c += 32) {
        const int yy = c / 10, g = c - yy * 10;
        const long long r = r0 + yy;
        if (g < kGroups) {
          const int2 yz = s_row[s * kMaxRowsPerItem + yy];
          const long long sr =
              clampi(yz.x - group_cy(g), 0, ny - 1) + (long long)ny * clampi(yz.y - group_cz(g), 0, nz - 1);
          const int first = group_first(g);
          bulk_load(sbase + ((size_t)yy * 19 + first) * pitch, fs + (sr * 19 + first) * pitch,
                    (uint32_t)group_count(g) * slot_bytes, &full[s]);
        } else {
          bulk_load(cbase + (size_t)yy * pitch, ia.cls + r * pitch, (uint32_t)pitch, &full[s]);
        }
      }
      issued = j + 1;
      if (++s == S_) { s = 0; ph ^= 1u; }
    }
    if (failed && lane == 0) atomicOr(b.error, STEP_ERR_PIPELINE_TIMEOUT);
    if (lane == 0) {
      for (int k = 0; k < S_ && k < issued; ++k) {
        const int last = k + ((issued - 1 - k) / S_) * S_;
        mbar_wait(&full[k], (uint32_t)((last / S_) & 1), kWaitLimit);
      }
    }
  } else {
    // ---------------- consumer warps ----------------
    // The 32-cell segments of an item (RY rows of `segs` segments) are dealt to the 8
    // warps cyclically, starting where the previous item stopped, so every warp has
    // work whatever the row length.  A warp releases the slot after its last load.
    int s = 0;
    uint32_t ph = 0;
    int offset = 0;  // warp that takes segment 0 of the current item
    for (int j = 0; j < my_count; ++j) {
      {
        const bool ok = mbar_wait(&full[s], ph, b.wait_limit);
        if (!__any_sync(0xffffffffu, ok)) {
          failed = true;
          break;
        }
      }
      const long long gi = blockIdx.x + (long long)j * gridDim.x;
      const int k = s_inst[s];
      const StepArgs& ia = b.inst[k];
      const int nx = ia.L.nx, ny = ia.L.ny, nz = ia.L.nz;
      const int pitch = P ? P : ia.L.pitch;
      const int4 geo = b.geo[k];
      const int RY = geo.x, segs = geo.y, shift = geo.z;  // rows per item, segments per row, shift
      const long long rows = (long long)ny * nz;
      const long long row0 = (gi - b.item_begin[k]) * RY;
      const int nr = (int)(rows - row0 < RY ? rows - row0 : RY);
      const int total = nr * segs;
      const int first = (warp - offset + kConsumerWarps) % kConsumerWarps;  // this warp's first segment
      offset = (offset + total) % kConsumerWarps;
      if (first >= total) {  // no segment of this item for this warp
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (++s == S_) { s = 0; ph ^= 1u; }
        continue;
      }
      const double corr = ia.st->apply[pslot] ? ia.st->corr[pslot] : 1.0;
      const float corrf = (float)corr;
      const float2 dec = make_float2(corrf * S::kRawScale, corrf - 1.0f);  // raw-moment decode
      const float tau0f = (float)ia.tau0, ksmagf = (float)ia.k_smag;
      T* fd = static_cast<T*>(b.bufs[2 * k + (cur ^ 1)]);
      long long item_sum = 0;
      int my_nan = 0;
      int ry = first / segs, sr = first - ry * segs;  // row and segment of segment `sg`
      auto inlet = [&](int y) {
        const double2 u = inlet_of(ia, y);
        return make_float2((float)u.x, (float)u.y);
      };
      for (int sg = first; sg < total; sg += kConsumerWarps) {
        if constexpr (CPT == 2) {
          // two adjacent cells per lane, 64-cell segments (every instance has an even nx)
          const int cell_lo = sr * 64;
          const int2 yz = s_row[s * kMaxRowsPerItem + ry];
          const int iy = yz.x, iz = yz.y;
          const T* sp = spop + (size_t)s * b.slot_elems + (size_t)ry * 19 * pitch;
          const uint8_t* sc = scls + (size_t)s * b.slot_cls + (size_t)ry * pitch;
          const int x0 = cell_lo + 2 * lane;
          const bool active = x0 < nx;
          const int lx = active ? x0 : 0;  // lanes outside the row read cells 0 and 1
          const uint32_t cls2 = *reinterpret_cast<const uint16_t*>(sc + lx);
          float2 v[19];
#pragma unroll
          for (int d = 0; d < 19; ++d) {
            const T* q = sp + slot_of(d) * pitch + lx;
            if (cx_of(d) == 0) v[d] = load_pair<S>(q);
            else v[d] = make_float2(S::raw(q[-cx_of(d)]), S::raw(q[1 - cx_of(d)]));
          }
          if (sg + kConsumerWarps >= total) {  // this warp's last segment of the slot
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
          }
          PairGeom g;
          g.row = row0 + ry; g.nx = nx; g.ny = ny; g.nz = nz; g.pitch = pitch;
          g.iy = iy; g.iz = iz; g.x0 = x0; g.cell_lo = cell_lo; g.active = active;
          g.has_lo = cell_lo == 0;
          g.has_hi = cell_lo <= nx - 2 && nx - 2 < cell_lo + 64;
          g.wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));
          g.ground_no_slip = ia.ground_no_slip; g.write_macro = b.write_macro;
          g.c0 = (uint8_t)(cls2 & 0xffu);
          g.c1 = (uint8_t)(cls2 >> 8);
          pair_segment<S>(v, fd, g, tau0f, ksmagf, dec, inlet, ia, s_xo + warp * 24, s_dcw, s_dslot, lane,
                          item_sum, my_nan);
          for (sr += kConsumerWarps; sr >= segs; sr -= segs) ++ry;
          continue;
        }
        const int cell_lo = sr * 32 - shift;
        const int2 yz = s_row[s * kMaxRowsPerItem + ry];
        const int iy = yz.x, iz = yz.y;
        const T* sp = spop + (size_t)s * b.slot_elems + (size_t)ry * 19 * pitch;
        const uint8_t* sc = scls + (size_t)s * b.slot_cls + (size_t)ry * pitch;
        const int ix = cell_lo + lane;
        const bool active = ix >= 0 && ix < nx;
        const int lx = active ? ix : 1;
        const uint8_t cl = sc[lx];
        float v[19];
#pragma unroll
        for (int d = 0; d < 19; ++d) v[d] = S::raw(sp[slot_of(d) * pitch + lx - cx_of(d)]);  // decoded in the moments
        if (sg + kConsumerWarps >= total) {  // this warp's last segment of the slot
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[s]);
        }
        SegGeom g;
        g.row = row0 + ry; g.nx = nx; g.ny = ny; g.nz = nz; g.pitch = pitch;
        g.iy = iy; g.iz = iz; g.cell_lo = cell_lo; g.ix = ix; g.flag = cl & CLS_FLAG_MASK;
        g.row_ok = true; g.active = active; g.near = (cl & CLS_NEAR) != 0;
        g.wall_row = (iy == 0 || iy == ny - 1 || (nz > 4 && (iz == 0 || iz == nz - 1)));
        g.ground_no_slip = ia.ground_no_slip; g.write_macro = b.write_macro; g.cl = cl;
        fast_segment<S>(v, fd, g, tau0f, ksmagf, dec, inlet, ia, s_xo + warp * 24, s_dcw, s_dslot, lane, item_sum,
                        my_nan);
        for (sr += kConsumerWarps; sr >= segs; sr -= segs) ++ry;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) item_sum += __shfl_down_sync(0xffffffffu, item_sum, o);
      if (lane == 0 && item_sum) atomicAdd(&s_sum[k], (unsigned long long)item_sum);
      if (__any_sync(0xffffffffu, my_nan) && lane == 0) ia.st->nan_seen = 1;
      if (++s == S_) { s = 0; ph ^= 1u; }
    }
    if (failed && lane == 0) atomicOr(b.error, STEP_ERR_PIPELINE_TIMEOUT);
  }

  __syncthreads();
  for (int k = threadIdx.x; k < b.n_inst; k += blockDim.x)
    b.partials[(long long)blockIdx.x * b.n_inst + k] = s_sum[k];
  __threadfence();
  __syncthreads();
  const int slot = step & 1;
  if (threadIdx.x == 0) {
    const unsigned int tk = atomicAdd(&b.ticket[slot], 1u);
    is_last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  // ---- the last CTA: mean-density rescale decision of every instance (:431-455) ----
  __threadfence();
  for (int k = warp; k < b.n_inst; k += blockDim.x >> 5) {
    unsigned long long tot = 0;
    for (int c = lane; c < (int)gridDim.x; c += 32)
      tot += __ldcg(&b.partials[(long long)c * b.n_inst + k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_down_sync(0xffffffffu, tot, o);
    if (lane == 0) {
      const StepArgs& ia = b.inst[k];
      StepState* st = ia.st;
      int ap = 0;
      double cr = 1.0;
      if (ia.fluid_count > 0) {
        const double mean = rho_unfixed((long long)tot, 0.0f) / (double)ia.fluid_count;
        cr = 1.0 / mean;
        ap = fabs(mean - 1.0) > 1e-4 ? 1 : 0;
      }
      st->corr[slot] = cr;
      st->apply[slot] = ap;
      if (ap) {
        st->cumulative_rescale *= cr;
        st->rescale_count += 1;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    b.ticket[slot ^ 1] = 0u;
    *b.step = step + 1;
  }
}

}  // namespace aerosim
