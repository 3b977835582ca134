// C-ABI layer of libaerosim.so: the LBMEngine / voxelizeMeshToLattice surface of the
// reference (src/solver/lbmEngine.ts, src/geometry/voxelizer.ts) over the sm_100a
// kernels.  Host code only; every device buffer is owned by the engine handle.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/aerosim.h"
#include "common.cuh"
#include "engine_internal.h"
#include "lbm_kernels.cuh"
#include "lbm_batch.cuh"
#include "sgs_mlp.cuh"

using namespace aerosim;

struct aerosim_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  aerosim_config cfg{};
  bool have_grid = false;
  DevGrid g;
  double dx = 0, origin[3] = {0, 0, 0};
  long long fluid_count = 0;
  void* f[2] = {nullptr, nullptr};
  int cur = 0;                 // f[cur] holds the latest populations (fSrc)
  int f_prec = -1;
  long long f_cells = 0;
  Layout L{};
  // persistent step-kernel launch shape
  dim3 block{256, 1, 1};
  unsigned grid = 1;
  size_t smem = 0;
  int stages = 3;
  int item_groups = 1;  // row groups per work item of the step kernel
  int cells_per_thread = 1;  // consumer cells per thread of the step kernel (1 or 2)
  int dynamic_items = 1;     // work items from a device counter (1) or dealt round-robin (0)
  int occupancy = 0;
  int num_sms = 148;
  float *mux = nullptr, *muy = nullptr, *muz = nullptr, *mrho = nullptr;
  int32_t* near_cells = nullptr;  // near-wall cells and their link table
  NearLink* links = nullptr;
  NearLinkF* links_f = nullptr;  // compact table of the FP32-arithmetic kernels
  long long n_near = 0;
  double* abl = nullptr;
  double* sin_tab = nullptr;
  int tab_ny = 0;
  StepState* st = nullptr;
  double* force_partials = nullptr;
  unsigned int* force_ticket = nullptr;
  double* force_out = nullptr;
  long long force_blocks_cap = 0;
  unsigned long long* stats_buf = nullptr;
  void* staging = nullptr;
  size_t staging_bytes = 0;
  // pinned and mapped into the device's address space, written by the kernels directly
  double* frame_host = nullptr;  // force sums [8] and the device error flag of a frame
  double* frame_dev = nullptr;   // its device address
  uint8_t* slice_host = nullptr;  // pinned, not mapped: the slice image on its way to the caller
  size_t slice_host_bytes = 0;
  size_t slice_bytes = 0;         // size of the last enqueued slice image
  long long step_index = 0;
  double last_ms = 0;
  long long last_launches = 0;
  // learned SGS closure (null: Smagorinsky)
  uint32_t* mlp_frag = nullptr;
  float* mlp_bias = nullptr;
  uint4* mlp_umma = nullptr;  // weight image of the tcgen05 path
  int mlp_path = AEROSIM_SGS_PATH_DEFAULT;
  bool wall_ready = false;  // wall distances in the class bytes
  int wait_limit = kWaitLimit;  // polls of a step kernel's ring wait before it gives up
};

namespace {

std::string g_create_error;
std::mutex g_error_mu;

int fail(aerosim_engine* h, int code, const std::string& msg) {
  if (h) {
    h->err = msg;
  } else {
    std::lock_guard<std::mutex> lock(g_error_mu);
    g_create_error = msg;
  }
  return code;
}

#define CU(h, x)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess)                                                                \
      return fail(h, e_ == cudaErrorMemoryAllocation ? AEROSIM_ERR_NOMEM : AEROSIM_ERR_CUDA, \
                  std::string(#x) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

void free_grid(DevGrid& g) {
  cudaFree(g.flags); cudaFree(g.cls); cudaFree(g.bmap); cudaFree(g.bcells);
  cudaFree(g.q); cudaFree(g.minq);
  g = DevGrid();
}

void free_pops(aerosim_engine* h) {
  cudaFree(h->f[0]); cudaFree(h->f[1]);
  h->f[0] = h->f[1] = nullptr;
  cudaFree(h->mux); cudaFree(h->muy); cudaFree(h->muz); cudaFree(h->mrho);
  h->mux = h->muy = h->muz = h->mrho = nullptr;
  h->f_prec = -1;
  h->f_cells = 0;
}

int prev_slot(const aerosim_engine* h) { return (int)((h->step_index + 1) & 1); }

int reset_state(aerosim_engine* h) {
  StepState s{};
  s.corr[0] = s.corr[1] = 1.0;
  s.cumulative_rescale = 1.0;
  CU(h, cudaMemcpyAsync(h->st, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  return AEROSIM_OK;
}

// resetEquilibrium + fresh rescale state, lbmCpuReference.ts:114-143.
int do_reset(aerosim_engine* h) {
  const DevGrid& g = h->g;
  CU(h, launch_init(h->cfg.precision, h->f[0], h->f[1], g.cls, h->mux, h->muy, h->muz, h->mrho, h->abl,
                    h->L, h->cfg.u_inlet_lattice, h->cfg.ground_no_slip, h->stream));
  h->cur = 0;
  h->step_index = 0;
  int rc = reset_state(h);
  if (rc) return rc;
  CU(h, cudaStreamSynchronize(h->stream));
  return AEROSIM_OK;
}

// The tcgen05 weight image when the closure runs as 128-cell tcgen05 tiles: that path was
// chosen and the lattice's row pitch is 128 or 256 (every work item then keeps the 8
// consumer warps busy as two groups of four); otherwise null (warp-level mma.sync).
const uint4* closure_umma(const aerosim_engine* h) {
  if (!h->mlp_frag || !h->mlp_umma || !h->have_grid) return nullptr;
  const bool fits = h->L.pitch == 128 || h->L.pitch == 256;
  return (h->mlp_path == AEROSIM_SGS_PATH_TCGEN05 && fits) ? h->mlp_umma : nullptr;
}

// Chooses the persistent step-kernel launch: CTAs of 8 consumer warps + 1 producer
// warp, as many resident per SM as registers and shared memory allow, and the
// deepest shared-memory ring (up to 4 slots) that keeps that residency.
int configure_step(aerosim_engine* h) {
  const Layout& L = h->L;
  const size_t eb = precision_bytes(h->cfg.precision);
  const dim3 block(kStepThreads, 1, 1);
  StepArgs dummy{};
  dummy.L = L;  // the kernel instance depends on the row pitch and the closure
  dummy.mlp_frag = h->mlp_frag;
  dummy.mlp_umma = closure_umma(h);
  const int mlp = h->mlp_frag ? (dummy.mlp_umma ? 2 : 1) : 0;
  const bool half = h->cfg.precision == AEROSIM_PREC_F16S || h->cfg.precision == AEROSIM_PREC_BF16S ||
                    h->cfg.precision == AEROSIM_PREC_F16C;
  const bool fast = half || h->cfg.precision == AEROSIM_PREC_F32;
  // two cells per consumer thread (packed FP32 pairs) without the closure on rows of an
  // even cell count; AEROSIM_CELLS_PER_THREAD (1 or 2) overrides the choice for any
  // fast-mode lattice that allows it
  const bool pairs_fit = !mlp && L.nx % 2 == 0 && L.nx >= 4;
  // measured at 256x128x128 with the dynamic deal: FP32 103.5 vs 108.4 us per step, FP16S
  // 76.0 vs 80.6, BF16S 75.6 vs 80.4 (two cells per thread vs one)
  int cpt = (fast && pairs_fit) ? 2 : 1;
  if (const char* cenv = getenv("AEROSIM_CELLS_PER_THREAD")) {
    const int want = atoi(cenv);
    if (want == 1) cpt = 1;
    if (want == 2 && fast && pairs_fit) cpt = 2;
  }
  dummy.cells_per_thread = cpt;
  const bool grouped = !mlp && half;
  int groups = grouped ? item_groups_for(L.nx, cpt) : 1;
  if (const char* genv = getenv("AEROSIM_ITEM_GROUPS")) {  // override of the row groups per item (1..4)
    const int want = atoi(genv);
    if (grouped && want >= 1 && want <= 4) groups = want;
  }
  const char* env = getenv("AEROSIM_STAGES");
  const int forced = env ? atoi(env) : 0;
  int best_s = 0, best_occ = 0;
  for (int S = 2; S <= 8; ++S) {
    if (forced && S != forced) continue;
    const size_t smem = step_smem_bytes(L, S, eb, mlp, groups, cpt);
    if (smem > 227 * 1024) break;
    int occ = 0;
    cudaError_t e = launch_step(h->cfg.precision, dummy, block, 0, smem, h->stream, &occ, nullptr);
    if (e != cudaSuccess || occ < 1) break;
    // keep deepening the ring while the residency does not drop
    if (best_s == 0 || (occ >= best_occ && S <= 4)) {
      best_s = S;
      best_occ = occ;
    }
  }
  if (best_s == 0) return fail(h, AEROSIM_ERR_ARG, "step kernel: no launch configuration fits shared memory");
  h->block = block;
  h->stages = best_s;
  h->smem = step_smem_bytes(L, best_s, eb, mlp, groups, cpt);
  h->item_groups = groups;
  h->cells_per_thread = cpt;
  // work items from the step's counter (108.8 vs 115.8 us FP32 with one cell per thread):
  // AEROSIM_DYNAMIC_ITEMS (0 or 1) overrides the default deal
  if (const char* denv = getenv("AEROSIM_DYNAMIC_ITEMS")) h->dynamic_items = atoi(denv) ? 1 : 0;
  // the occupancy of the chosen configuration
  CU(h, launch_step(h->cfg.precision, dummy, block, 0, h->smem, h->stream, &best_occ, nullptr));
  h->occupancy = best_occ;
  const long long item_rows = (long long)rows_per_item(L.nx, cpt) * groups;
  const long long items = ((long long)L.ny * L.nz + item_rows - 1) / item_rows;
  long long grid = (long long)best_occ * h->num_sms;
  const char* genv = getenv("AEROSIM_CTAS_PER_SM");
  if (genv && atoi(genv) > 0 && atoi(genv) <= best_occ) grid = (long long)atoi(genv) * h->num_sms;
  if (grid > items) grid = items;
  h->grid = (unsigned)(grid < 1 ? 1 : grid);
  return AEROSIM_OK;
}

// Allocates population and macro buffers for the current grid and precision.
int ensure_pops(aerosim_engine* h, bool* reallocated) {
  *reallocated = false;
  const long long N = h->g.N;
  if (h->f[0] && h->f_prec == h->cfg.precision && h->f_cells == N) return configure_step(h);
  free_pops(h);
  const size_t eb = precision_bytes(h->cfg.precision);
  CU(h, cudaMalloc(&h->f[0], 19 * (size_t)h->L.plane * eb));
  CU(h, cudaMalloc(&h->f[1], 19 * (size_t)h->L.plane * eb));
  CU(h, cudaMalloc(&h->mux, N * sizeof(float)));
  CU(h, cudaMalloc(&h->muy, N * sizeof(float)));
  CU(h, cudaMalloc(&h->muz, N * sizeof(float)));
  CU(h, cudaMalloc(&h->mrho, N * sizeof(float)));
  h->f_prec = h->cfg.precision;
  h->f_cells = N;
  *reallocated = true;
  return configure_step(h);
}

int ensure_staging(aerosim_engine* h, size_t bytes) {
  if (h->staging_bytes >= bytes) return AEROSIM_OK;
  cudaFree(h->staging);
  h->staging = nullptr;
  h->staging_bytes = 0;
  CU(h, cudaMalloc(&h->staging, bytes));
  h->staging_bytes = bytes;
  return AEROSIM_OK;
}

// Tables of the inlet condition that the reference evaluates with Math.pow and
// Math.sin (lbmCpuReference.ts:121-125, 334-342), computed once on the host.
int upload_tables(aerosim_engine* h) {
  const int ny = h->g.ny;
  if (h->tab_ny == ny && h->abl) return AEROSIM_OK;
  cudaFree(h->abl); cudaFree(h->sin_tab);
  h->abl = nullptr; h->sin_tab = nullptr;
  std::vector<double> abl(ny), st((size_t)120 * ny);
  for (int iy = 0; iy < ny; ++iy) {
    const double yf = (iy + 0.5) / ny;
    abl[iy] = js_min(1.15, 0.35 + 0.8 * std::pow(yf, 0.3));
  }
  for (int s = 0; s < 120; ++s)
    for (int iy = 0; iy < ny; ++iy)
      st[(size_t)s * ny + iy] = std::sin(s * 0.15 + ((double)iy / ny) * M_PI * 2.0);
  CU(h, cudaMalloc(&h->abl, ny * sizeof(double)));
  CU(h, cudaMalloc(&h->sin_tab, st.size() * sizeof(double)));
  CU(h, cudaMemcpyAsync(h->abl, abl.data(), ny * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CU(h, cudaMemcpyAsync(h->sin_tab, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  h->tab_ny = ny;
  return AEROSIM_OK;
}

// Installs a freshly built device grid (voxelizer output or host upload).
int install_grid(aerosim_engine* h, DevGrid& ng, double dx, const double origin[3], int reset_flow) {
  // A pending rescale belongs to the old flags: apply it before they change.
  if (h->have_grid && h->f[0] && !reset_flow) {
    CU(h, launch_materialize(h->f_prec, h->f[h->cur], h->g.cls, h->st, prev_slot(h), h->L, h->g.N,
                             h->stream));
    int rc = reset_state(h);
    if (rc) return rc;
  }
  const Layout nl = make_layout(ng.nx, ng.ny, ng.nz);
  CU(h, cudaMalloc(&ng.cls, std::max<long long>((long long)ng.ny * ng.nz * nl.pitch, 1)));
  CU(h, cudaMemsetAsync(ng.cls, CELL_SOLID, (size_t)ng.ny * ng.nz * nl.pitch, h->stream));
  CU(h, launch_classify(ng.flags, ng.cls, nl, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  {
    // Near-wall cells (x faces excluded: the inlet and outlet overwrite them) and
    // their link table: for each direction, how the reference's pull obtains the
    // value (lbmCpuReference.ts:189-224), resolved once per voxel grid.
    const long long N = ng.N;
    std::vector<uint8_t> cls((size_t)ng.ny * ng.nz * nl.pitch);
    std::vector<int32_t> bmap(N);
    std::vector<float> q((size_t)std::max<long long>(ng.B, 1) * 18);
    // (the table is rebuilt with every voxel grid; the layout nl decides the offsets)
    CU(h, cudaMemcpy(cls.data(), ng.cls, cls.size(), cudaMemcpyDeviceToHost));
    CU(h, cudaMemcpy(bmap.data(), ng.bmap, N * 4, cudaMemcpyDeviceToHost));
    if (ng.B > 0) CU(h, cudaMemcpy(q.data(), ng.q, ng.B * 18 * 4, cudaMemcpyDeviceToHost));
    auto flag_at = [&](int x, int y, int z) {
      return cls[((size_t)y + (size_t)ng.ny * z) * nl.pitch + x] & CLS_FLAG_MASK;
    };
    auto clampi_h = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
    std::vector<int32_t> nearv;
    for (int iz = 0; iz < ng.nz; ++iz)
      for (int iy = 0; iy < ng.ny; ++iy) {
        const long long row = iy + (long long)ng.ny * iz;
        for (int ix = 1; ix < ng.nx - 1; ++ix)
          if (cls[row * nl.pitch + ix] & CLS_NEAR) nearv.push_back((int32_t)(row * ng.nx + ix));
      }
    const long long nn = (long long)nearv.size();
    if ((long long)19 * nl.plane >= (1LL << 32))
      return fail(h, AEROSIM_ERR_ARG, "lattice too large for 32-bit population offsets");
    auto off = [&](int d, long long c) -> uint32_t { return (uint32_t)nl.at(d, c); };
    std::vector<NearLink> links(19 * std::max<long long>(nn, 1));
    for (long long t = 0; t < nn; ++t) {
      const long long cell = nearv[t];
      const int ix = (int)(cell % ng.nx);
      const long long row = cell / ng.nx;
      const int iy = (int)(row % ng.ny), iz = (int)(row / ng.ny);
      const int flag = flag_at(ix, iy, iz);
      const int bi = flag == CELL_BOUNDARY ? bmap[cell] : -1;
      for (int d = 0; d < 19; ++d) {
        NearLink& L = links[(size_t)d * nn + t];
        const int sx = clampi_h(ix - cx_of(d), 0, ng.nx - 1), sy = clampi_h(iy - cy_of(d), 0, ng.ny - 1),
                  sz = clampi_h(iz - cz_of(d), 0, ng.nz - 1);
        const long long src = sx + (long long)ng.nx * (sy + (long long)ng.ny * sz);
        L.A = 1.0; L.B = 0.0;
        if (d > 0 && flag_at(sx, sy, sz) == CELL_SOLID) {
          // Bouzidi in the pull, lbmCpuReference.ts:196-221
          const int wd = opp_of(d);
          const double qv = bi >= 0 ? (double)q[(size_t)bi * 18 + (wd - 1)] : 0.5;
          const double qe = qv > 0.0 ? qv : 0.5;
          const int fx = clampi_h(ix + cx_of(d), 0, ng.nx - 1), fy = clampi_h(iy + cy_of(d), 0, ng.ny - 1),
                    fz = clampi_h(iz + cz_of(d), 0, ng.nz - 1);
          const long long ff = fx + (long long)ng.nx * (fy + (long long)ng.ny * fz);
          L.o1 = off(wd, cell); L.d1 = wd;
          L.o2 = L.o1; L.d2 = wd;
          if (flag_at(fx, fy, fz) != CELL_SOLID) {
            if (qe < 0.5) {
              L.A = 2.0 * qe; L.B = 1.0 - 2.0 * qe;
              L.o2 = off(wd, ff); L.d2 = wd;
            } else {
              const double inv2q = 1.0 / (2.0 * qe);
              L.A = inv2q; L.B = 1.0 - inv2q;
              L.o2 = off(d, cell); L.d2 = d;
            }
          }
        } else {
          L.o1 = off(d, src); L.d1 = d;
          L.o2 = L.o1; L.d2 = d;
        }
      }
    }
    std::vector<NearLinkF> links_f(links.size());
    for (size_t i = 0; i < links.size(); ++i)
      links_f[i] = NearLinkF{links[i].o1, links[i].o2, (float)links[i].A, (float)links[i].B};
    cudaFree(h->near_cells); cudaFree(h->links); cudaFree(h->links_f);
    h->near_cells = nullptr; h->links = nullptr; h->links_f = nullptr;
    h->n_near = nn;
    CU(h, cudaMalloc(&h->near_cells, std::max<long long>(nn, 1) * 4));
    CU(h, cudaMalloc(&h->links, links.size() * sizeof(NearLink)));
    CU(h, cudaMalloc(&h->links_f, links_f.size() * sizeof(NearLinkF)));
    if (nn) CU(h, cudaMemcpy(h->near_cells, nearv.data(), nn * 4, cudaMemcpyHostToDevice));
    CU(h, cudaMemcpy(h->links, links.data(), links.size() * sizeof(NearLink), cudaMemcpyHostToDevice));
    CU(h, cudaMemcpy(h->links_f, links_f.data(), links_f.size() * sizeof(NearLinkF), cudaMemcpyHostToDevice));
  }
  h->wall_ready = false;
  if (h->mlp_frag) {  // the learned closure reads wall distances from the class bytes
    CU(h, compute_wall_distance(ng.flags, ng.nx, ng.ny, ng.nz, nullptr, ng.cls, nl.pitch, h->stream));
    h->wall_ready = true;
  }
  if (h->f[0] && (nl.pitch != h->L.pitch || nl.plane != h->L.plane)) free_pops(h);
  free_grid(h->g);
  h->g = ng;
  h->L = nl;
  ng = DevGrid();
  h->have_grid = true;
  h->dx = dx;
  h->origin[0] = origin[0]; h->origin[1] = origin[1]; h->origin[2] = origin[2];
  h->fluid_count = h->g.N - h->g.solid;
  // force reduction: 8 boundary cells per CTA and round, at most 2 CTAs per SM
  const long long blocks = std::max<long long>(1, std::min<long long>((h->g.B + 7) / 8, 2LL * h->num_sms));
  if (blocks > h->force_blocks_cap) {
    cudaFree(h->force_partials);
    h->force_partials = nullptr;
    CU(h, cudaMalloc(&h->force_partials, blocks * 8 * sizeof(double)));
    h->force_blocks_cap = blocks;
  }
  int rc = upload_tables(h);
  if (rc) return rc;
  bool realloc = false;
  rc = ensure_pops(h, &realloc);
  if (rc) return rc;
  if (reset_flow || realloc) return do_reset(h);
  return AEROSIM_OK;
}

void default_config(aerosim_config* c) {
  // LBMEngine defaults, lbmEngine.ts:42-57
  c->u_inlet_lattice = 0.085;
  c->nu_lattice = 0.0005;
  c->smagorinsky_cs = 0.12;
  c->ground_no_slip = 0;
  c->precision = AEROSIM_PREC_F32;
  c->frontal_area_m2 = M_PI * 0.25;
  c->characteristic_length_m = 1.0;
  c->tunnel = aerosim_tunnel{6.0, 2.8, 2.4};
}

// computeNormalizedForceCoefficients, forceIntegrator.ts:240-315.
void coefficients(const aerosim_config& c, double dx, aerosim_forces* o) {
  const double cell_area = dx * dx;
  const double q_lat = js_max(1e-9, 0.5 * 1.0 * c.u_inlet_lattice * c.u_inlet_lattice);
  const double a_ref = js_max(1e-4, c.frontal_area_m2 / cell_area);
  const double l_ref = js_max(1.0, c.characteristic_length_m / dx);
  o->cd_raw = o->fx / (q_lat * a_ref);
  o->cl = o->fy / (q_lat * a_ref);
  o->cm = o->mz / (q_lat * a_ref * l_ref);
  const double tunnel_area = js_max(1e-4, c.tunnel.width * c.tunnel.height);
  const double blockage = js_min(0.40, c.frontal_area_m2 / tunnel_area);
  o->cd = o->cd_raw / (1.0 + 2.5 * js_max(0.0, o->cd_raw) * blockage);
  const double L = c.characteristic_length_m;
  o->xcp = std::fabs(o->fy) > 1e-5 ? js_max(-L * 0.5, js_min(L * 0.5, -(o->mz / o->fy) * dx)) : 0.0;
}

}  // namespace

namespace aerosim {
void set_global_error(const std::string& msg) { fail(nullptr, 0, msg); }
}  // namespace aerosim

extern "C" {

int aerosim_abi_version(void) { return AEROSIM_ABI_VERSION; }

const char* aerosim_last_error(const aerosim_engine* h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

int aerosim_create(int device, aerosim_engine** out) {
  if (!out) return fail(nullptr, AEROSIM_ERR_ARG, "aerosim_create: out is NULL");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(nullptr, AEROSIM_ERR_CUDA, std::string("aerosim_create: no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= n) return fail(nullptr, AEROSIM_ERR_ARG, "aerosim_create: bad device ordinal");
  aerosim_engine* h = new (std::nothrow) aerosim_engine();
  if (!h) return fail(nullptr, AEROSIM_ERR_NOMEM, "aerosim_create: out of host memory");
  h->device = device;
  default_config(&h->cfg);
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
  if (e == cudaSuccess) e = cudaMalloc(&h->st, sizeof(StepState));
  if (e == cudaSuccess) e = cudaMalloc(&h->force_ticket, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(&h->force_out, 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&h->stats_buf, 4 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(h->force_ticket, 0, sizeof(unsigned int));
  if (e != cudaSuccess) {
    std::string msg = std::string("aerosim_create: ") + cudaGetErrorString(e);
    aerosim_destroy(h);
    return fail(nullptr, AEROSIM_ERR_CUDA, msg);
  }
  if (reset_state(h) != AEROSIM_OK) {
    std::string msg = h->err;
    aerosim_destroy(h);
    return fail(nullptr, AEROSIM_ERR_CUDA, msg);
  }
  *out = h;
  return AEROSIM_OK;
}

int aerosim_destroy(aerosim_engine* h) {
  if (!h) return AEROSIM_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_grid(h->g);
  free_pops(h);
  cudaFree(h->abl); cudaFree(h->sin_tab); cudaFree(h->st);
  cudaFree(h->near_cells); cudaFree(h->links); cudaFree(h->links_f);
  cudaFree(h->force_partials); cudaFree(h->force_ticket); cudaFree(h->force_out);
  cudaFree(h->stats_buf); cudaFree(h->staging);
  if (h->frame_host) cudaFreeHost(h->frame_host);
  if (h->slice_host) cudaFreeHost(h->slice_host);
  cudaFree(h->mlp_frag); cudaFree(h->mlp_bias); cudaFree(h->mlp_umma);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return AEROSIM_OK;
}

int aerosim_voxelize(aerosim_engine* h, const float* positions, int64_t vertex_count,
                     const int32_t* indices, int64_t index_count, const double* world16,
                     aerosim_tunnel tunnel, int32_t nx, int32_t ny, int32_t nz, int32_t reset_flow,
                     aerosim_voxel_info* out) {
  if (!h) return AEROSIM_ERR_ARG;
  if (nx < 3 || ny < 1 || nz < 1) return fail(h, AEROSIM_ERR_ARG, "aerosim_voxelize: need nx >= 3, ny >= 1, nz >= 1");
  if ((long long)nx * ny * nz >= (1LL << 31)) return fail(h, AEROSIM_ERR_ARG, "aerosim_voxelize: lattice too large");
  if (vertex_count < 0 || (vertex_count > 0 && !positions)) return fail(h, AEROSIM_ERR_ARG, "aerosim_voxelize: bad positions");
  if (indices) {
    if (index_count < 0) return fail(h, AEROSIM_ERR_ARG, "aerosim_voxelize: bad index_count");
    for (int64_t i = 0; i < index_count; ++i)
      if (indices[i] < 0 || indices[i] >= vertex_count)
        return fail(h, AEROSIM_ERR_ARG, "aerosim_voxelize: index out of range");
  }
  if (!(tunnel.height > 0)) return fail(h, AEROSIM_ERR_ARG, "aerosim_voxelize: tunnel height must be > 0");
  CU(h, cudaSetDevice(h->device));
  DevGrid ng;
  std::string e;
  const int rc = run_voxelizer(positions, vertex_count, indices, index_count, world16, tunnel.height, nx, ny,
                               nz, h->stream, &ng, &e);
  if (rc) {
    free_grid(ng);
    return fail(h, rc == -4 ? AEROSIM_ERR_DEVICE : AEROSIM_ERR_CUDA, e);
  }
  const double origin[3] = {ng.ox, ng.oy, ng.oz};
  const double dx = ng.h;
  const int r2 = install_grid(h, ng, dx, origin, reset_flow);
  free_grid(ng);
  if (r2) return r2;
  h->cfg.tunnel = tunnel;
  return aerosim_get_voxel_info(h, out);
}

int aerosim_get_voxel_info(aerosim_engine* h, aerosim_voxel_info* out) {
  if (!h) return AEROSIM_ERR_ARG;
  if (!h->have_grid) return fail(h, AEROSIM_ERR_STATE, "no voxel grid");
  if (!out) return AEROSIM_OK;
  out->nx = h->g.nx; out->ny = h->g.ny; out->nz = h->g.nz;
  out->dx = out->dy = out->dz = h->dx;
  out->origin_x = h->origin[0]; out->origin_y = h->origin[1]; out->origin_z = h->origin[2];
  out->solid_cell_count = h->g.solid;
  out->boundary_cell_count = h->g.B;
  out->fluid_cell_count = h->g.N - h->g.solid - h->g.B;
  out->voxelization_time_ms = h->g.vox_ms;
  return AEROSIM_OK;
}

int aerosim_read_voxel_grid(aerosim_engine* h, uint8_t* flags, int32_t* bmap, int32_t* bcells, float* q,
                            float* minq) {
  if (!h) return AEROSIM_ERR_ARG;
  if (!h->have_grid) return fail(h, AEROSIM_ERR_STATE, "no voxel grid");
  CU(h, cudaSetDevice(h->device));
  const DevGrid& g = h->g;
  if (flags) CU(h, cudaMemcpyAsync(flags, g.flags, g.N, cudaMemcpyDeviceToHost, h->stream));
  if (bmap) CU(h, cudaMemcpyAsync(bmap, g.bmap, g.N * 4, cudaMemcpyDeviceToHost, h->stream));
  if (g.B > 0) {
    if (bcells) CU(h, cudaMemcpyAsync(bcells, g.bcells, g.B * 4, cudaMemcpyDeviceToHost, h->stream));
    if (q) CU(h, cudaMemcpyAsync(q, g.q, g.B * 18 * 4, cudaMemcpyDeviceToHost, h->stream));
    if (minq) CU(h, cudaMemcpyAsync(minq, g.minq, g.B * 4, cudaMemcpyDeviceToHost, h->stream));
  }
  CU(h, cudaStreamSynchronize(h->stream));
  return AEROSIM_OK;
}

int aerosim_set_voxel_grid(aerosim_engine* h, int32_t nx, int32_t ny, int32_t nz, double dx,
                           const double origin[3], const uint8_t* flags, const int32_t* bmap,
                           const int32_t* bcells, const float* q, int64_t B, int32_t reset_flow) {
  if (!h) return AEROSIM_ERR_ARG;
  if (nx < 3 || ny < 1 || nz < 1) return fail(h, AEROSIM_ERR_ARG, "set_voxel_grid: need nx >= 3, ny >= 1, nz >= 1");
  const long long N = (long long)nx * ny * nz;
  if (N >= (1LL << 31)) return fail(h, AEROSIM_ERR_ARG, "set_voxel_grid: lattice too large");
  if (!flags || B < 0 || (B > 0 && (!bcells || !q)))
    return fail(h, AEROSIM_ERR_ARG, "set_voxel_grid: missing flags / boundary arrays");
  long long solid = 0;
  for (long long i = 0; i < N; ++i) {
    if (flags[i] > 2) return fail(h, AEROSIM_ERR_ARG, "set_voxel_grid: flag value outside {0,1,2}");
    solid += flags[i] == 1;
  }
  std::vector<int32_t> map_built;
  if (!bmap) {
    map_built.assign(N, -1);
    for (int64_t b = 0; b < B; ++b) {
      if (bcells[b] < 0 || bcells[b] >= N) return fail(h, AEROSIM_ERR_ARG, "set_voxel_grid: boundary cell out of range");
      map_built[bcells[b]] = (int32_t)b;
    }
    bmap = map_built.data();
  } else {
    for (long long i = 0; i < N; ++i)
      if (bmap[i] < -1 || bmap[i] >= B) return fail(h, AEROSIM_ERR_ARG, "set_voxel_grid: boundary index map out of range");
  }
  for (int64_t b = 0; b < B; ++b)
    if (bcells[b] < 0 || bcells[b] >= N) return fail(h, AEROSIM_ERR_ARG, "set_voxel_grid: boundary cell out of range");
  CU(h, cudaSetDevice(h->device));
  DevGrid ng;
  ng.nx = nx; ng.ny = ny; ng.nz = nz; ng.N = N; ng.h = dx;
  ng.ox = origin ? origin[0] : -nx * dx * 0.5;
  ng.oy = origin ? origin[1] : -ny * dx * 0.5;
  ng.oz = origin ? origin[2] : -nz * dx * 0.5;
  ng.B = B; ng.solid = solid;
  auto bad = [&](cudaError_t e) {
    free_grid(ng);
    return fail(h, AEROSIM_ERR_CUDA, std::string("set_voxel_grid: ") + cudaGetErrorString(e));
  };
  cudaError_t e;
  if ((e = cudaMalloc(&ng.flags, N)) != cudaSuccess) return bad(e);
  if ((e = cudaMalloc(&ng.bmap, N * 4)) != cudaSuccess) return bad(e);
  if ((e = cudaMalloc(&ng.bcells, std::max<int64_t>(B, 1) * 4)) != cudaSuccess) return bad(e);
  if ((e = cudaMalloc(&ng.q, std::max<int64_t>(B, 1) * 18 * 4)) != cudaSuccess) return bad(e);
  if ((e = cudaMalloc(&ng.minq, std::max<int64_t>(B, 1) * 4)) != cudaSuccess) return bad(e);
  std::vector<float> mq(std::max<int64_t>(B, 1), 1.0f);
  for (int64_t b = 0; b < B; ++b)
    for (int k = 0; k < 18; ++k) {
      const float v = q[b * 18 + k];
      if (v > 0.0f && v < mq[b]) mq[b] = v;
    }
  if ((e = cudaMemcpy(ng.flags, flags, N, cudaMemcpyHostToDevice)) != cudaSuccess) return bad(e);
  if ((e = cudaMemcpy(ng.bmap, bmap, N * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return bad(e);
  if (B > 0) {
    if ((e = cudaMemcpy(ng.bcells, bcells, B * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return bad(e);
    if ((e = cudaMemcpy(ng.q, q, B * 18 * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return bad(e);
    if ((e = cudaMemcpy(ng.minq, mq.data(), B * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return bad(e);
  }
  const double org[3] = {ng.ox, ng.oy, ng.oz};
  const int rc = install_grid(h, ng, dx, org, reset_flow);
  free_grid(ng);
  return rc;
}

int aerosim_set_config(aerosim_engine* h, const aerosim_config* cfg) {
  if (!h || !cfg) return AEROSIM_ERR_ARG;
  if (precision_bytes(cfg->precision) == 0) return fail(h, AEROSIM_ERR_ARG, "set_config: unknown precision");
  CU(h, cudaSetDevice(h->device));
  const int old_prec = h->cfg.precision;
  h->cfg = *cfg;
  if (h->have_grid && cfg->precision != old_prec) {
    bool realloc = false;
    int rc = ensure_pops(h, &realloc);
    if (rc) return rc;
    return do_reset(h);
  }
  return AEROSIM_OK;
}

int aerosim_get_config(aerosim_engine* h, aerosim_config* cfg) {
  if (!h || !cfg) return AEROSIM_ERR_ARG;
  *cfg = h->cfg;
  return AEROSIM_OK;
}

int aerosim_reset_flow(aerosim_engine* h) {
  if (!h) return AEROSIM_ERR_ARG;
  if (!h->have_grid) return fail(h, AEROSIM_ERR_STATE, "reset_flow: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  return do_reset(h);
}

}  // extern "C"

namespace {

// Enqueues n steps on h's stream between the engine's timing events (the substep loop
// of stepAndExtractSlice, lbmEngine.ts:483-527); the caller synchronizes.
int enqueue_steps(aerosim_engine* h, int32_t n) {
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "step: no voxel grid");
  if (n < 0) return fail(h, AEROSIM_ERR_ARG, "step: negative step count");
  if (h->step_index + n > 0x7fffffffLL) return fail(h, AEROSIM_ERR_ARG, "step: step index overflow");
  CU(h, cudaSetDevice(h->device));
  const DevGrid& g = h->g;
  StepArgs a{};
  a.cls = g.cls; a.bmap = g.bmap; a.q = g.q;
  a.mux = h->mux; a.muy = h->muy; a.muz = h->muz; a.mrho = h->mrho;
  a.abl = h->abl; a.sin_tab = h->sin_tab; a.st = h->st;
  a.L = h->L; a.fluid_count = h->fluid_count;
  a.near_cells = h->near_cells; a.n_near = h->n_near;
  a.links = h->links;
  a.links_f = h->links_f;
  a.stages = h->stages;
  a.ground_no_slip = h->cfg.ground_no_slip;
  a.u_inlet = h->cfg.u_inlet_lattice;
  a.tau0 = 3.0 * h->cfg.nu_lattice + 0.5;
  const double cs2 = h->cfg.smagorinsky_cs * h->cfg.smagorinsky_cs;
  a.k_smag = 18.0 * M_SQRT2 * cs2;
  a.mlp_frag = h->mlp_frag;
  a.mlp_bias = h->mlp_bias;
  a.mlp_umma = closure_umma(h);
  a.mlp_nu0 = (float)((std::max(a.tau0, 0.5015) - 0.5) / 3.0);
  a.item_groups = h->item_groups;
  a.cells_per_thread = h->cells_per_thread;
  a.dynamic_items = h->dynamic_items;
  a.wait_limit = h->wait_limit;
  long long launches = 0;
  CU(h, cudaEventRecord(h->ev0, h->stream));
  for (int s = 0; s < n; ++s) {
    a.fsrc = h->f[h->cur];
    a.fdst = h->f[h->cur ^ 1];
    a.step_index = (int)h->step_index;
    a.write_macro = (s == n - 1) ? 1 : 0;
    int nl = 0;
    CU(h, launch_step(h->cfg.precision, a, h->block, h->grid, h->smem, h->stream, nullptr, &nl));
    launches += nl;
    h->cur ^= 1;
    h->step_index += 1;
  }
  CU(h, cudaEventRecord(h->ev1, h->stream));
  h->last_launches = launches;
  return AEROSIM_OK;
}

// Step timing after the stream has drained.
int finish_steps(aerosim_engine* h, int dev_err) {
  float ms = 0.f;
  CU(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->last_ms = ms;
  if (dev_err) return fail(h, AEROSIM_ERR_DEVICE, "step: the shared-memory pipeline timed out (device error flag set)");
  return AEROSIM_OK;
}

// Enqueues the momentum-exchange reduction of the current populations; its eight FP64
// sums land in `dst` (device-to-host, asynchronous when dst is pinned).
// With dst_dev (the device address of mapped pinned memory at dst) the kernel writes
// the sums, and err_dev the steps' error code, to the host directly.
int enqueue_forces(aerosim_engine* h, double* dst, double* dst_dev = nullptr, int* err_dev = nullptr) {
  ForceArgs a{};
  a.f = h->f[h->cur];
  a.cls = h->g.cls; a.bcells = h->g.bcells; a.q = h->g.q; a.st = h->st;
  a.partials = h->force_partials; a.ticket = h->force_ticket;
  a.out = dst_dev ? dst_dev : h->force_out;
  a.err_out = err_dev;
  a.L = h->L; a.B = h->g.B;
  a.prev_slot = prev_slot(h);
  const unsigned grid = (unsigned)std::min<long long>((h->g.B + 7) / 8, h->force_blocks_cap);
  CU(h, launch_forces(h->cfg.precision, a, grid, h->stream));
  if (!dst_dev) CU(h, cudaMemcpyAsync(dst, h->force_out, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return AEROSIM_OK;
}

// The engine's mapped pinned frame buffer (force sums and error code).
int ensure_frame_host(aerosim_engine* h) {
  if (h->frame_host) return AEROSIM_OK;
  CU(h, cudaHostAlloc((void**)&h->frame_host, 16 * sizeof(double), cudaHostAllocMapped));
  const cudaError_t e = cudaHostGetDevicePointer((void**)&h->frame_dev, h->frame_host, 0);
  if (e != cudaSuccess) {  // never keep a host buffer without its device address
    cudaFreeHost(h->frame_host);
    h->frame_host = nullptr;
    h->frame_dev = nullptr;
    return fail(h, AEROSIM_ERR_CUDA, std::string("cudaHostGetDevicePointer: ") + cudaGetErrorString(e));
  }
  return AEROSIM_OK;
}

void forces_from_sums(aerosim_engine* h, const double* r, aerosim_forces* out) {
  std::memset(out, 0, sizeof(*out));
  out->fx = r[0]; out->fy = r[1]; out->fz = r[2];
  out->mx = r[3]; out->my = r[4]; out->mz = r[5];
  out->cut_face_links = (int64_t)r[6];
  out->step = h->step_index;
  coefficients(h->cfg, h->dx, out);
}

}  // namespace

extern "C" {

int aerosim_step(aerosim_engine* h, int32_t n) {
  if (!h) return AEROSIM_ERR_ARG;
  int rc = enqueue_steps(h, n);
  if (rc) return rc;
  int dev_err = 0;
  CU(h, cudaMemcpyAsync(&dev_err, &h->st->error, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  return finish_steps(h, dev_err);
}

int aerosim_get_step_count(aerosim_engine* h, int64_t* out) {
  if (!h || !out) return AEROSIM_ERR_ARG;
  *out = h->step_index;
  return AEROSIM_OK;
}

int aerosim_read_forces(aerosim_engine* h, aerosim_forces* out) {
  if (!h || !out) return AEROSIM_ERR_ARG;
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "read_forces: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  double r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (h->g.B > 0) {
    int rc = ensure_frame_host(h);
    if (rc || (rc = enqueue_forces(h, h->frame_host, h->frame_dev))) return rc;
    CU(h, cudaStreamSynchronize(h->stream));
    std::memcpy(r, h->frame_host, sizeof(r));
  }
  forces_from_sums(h, r, out);
  return AEROSIM_OK;
}

int aerosim_read_macro(aerosim_engine* h, float* ux, float* uy, float* uz, float* rho) {
  if (!h) return AEROSIM_ERR_ARG;
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "read_macro: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  const long long N = h->g.N;
  if (ux) CU(h, cudaMemcpyAsync(ux, h->mux, N * 4, cudaMemcpyDeviceToHost, h->stream));
  if (uy) CU(h, cudaMemcpyAsync(uy, h->muy, N * 4, cudaMemcpyDeviceToHost, h->stream));
  if (uz) CU(h, cudaMemcpyAsync(uz, h->muz, N * 4, cudaMemcpyDeviceToHost, h->stream));
  if (rho) {
    int rc = ensure_staging(h, N * 4);
    if (rc) return rc;
    CU(h, launch_read_macro(h->mrho, h->g.cls, h->st, prev_slot(h), h->L, N, (float*)h->staging, h->stream));
    CU(h, cudaMemcpyAsync(rho, h->staging, N * 4, cudaMemcpyDeviceToHost, h->stream));
  }
  CU(h, cudaStreamSynchronize(h->stream));
  return AEROSIM_OK;
}

int aerosim_read_populations(aerosim_engine* h, void* f, int32_t dtype) {
  if (!h || !f) return AEROSIM_ERR_ARG;
  if (dtype != AEROSIM_DTYPE_F32 && dtype != AEROSIM_DTYPE_F64) return fail(h, AEROSIM_ERR_ARG, "read_populations: bad dtype");
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "read_populations: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  const long long N = h->g.N;
  const size_t bytes = (size_t)19 * N * (dtype == AEROSIM_DTYPE_F32 ? 4 : 8);
  int rc = ensure_staging(h, bytes);
  if (rc) return rc;
  CU(h, launch_read_pops(h->f_prec, h->f[h->cur], h->g.cls, h->st, prev_slot(h), h->L, N, h->staging,
                         dtype, h->stream));
  CU(h, cudaMemcpyAsync(f, h->staging, bytes, cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  return AEROSIM_OK;
}

int aerosim_write_populations(aerosim_engine* h, const void* f, int32_t dtype) {
  if (!h || !f) return AEROSIM_ERR_ARG;
  if (dtype != AEROSIM_DTYPE_F32 && dtype != AEROSIM_DTYPE_F64) return fail(h, AEROSIM_ERR_ARG, "write_populations: bad dtype");
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "write_populations: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  const long long N = h->g.N;
  const size_t bytes = (size_t)19 * N * (dtype == AEROSIM_DTYPE_F32 ? 4 : 8);
  int rc = ensure_staging(h, bytes);
  if (rc) return rc;
  CU(h, cudaMemcpyAsync(h->staging, f, bytes, cudaMemcpyHostToDevice, h->stream));
  CU(h, launch_write_pops(h->f_prec, h->f[h->cur], h->L, N, h->staging, dtype, h->stream));
  // the written values are final: no rescale is pending on them
  StepState s{};
  CU(h, cudaMemcpyAsync(&s, h->st, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  s.apply[0] = s.apply[1] = 0;
  CU(h, cudaMemcpyAsync(h->st, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  return AEROSIM_OK;
}

int aerosim_mass_stats(aerosim_engine* h, aerosim_mass* out) {
  if (!h || !out) return AEROSIM_ERR_ARG;
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "mass_stats: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  unsigned long long r[4];
  StepState s{};
  CU(h, cudaMemsetAsync(h->stats_buf, 0, sizeof(r), h->stream));
  CU(h, launch_mass_stats(h->mux, h->muy, h->muz, h->mrho, h->g.cls, h->st, prev_slot(h), h->L, h->g.N,
                          h->stats_buf, h->stream));
  CU(h, cudaMemcpyAsync(r, h->stats_buf, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaMemcpyAsync(&s, h->st, sizeof(s), cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  std::memset(out, 0, sizeof(*out));
  const double total = (double)(long long)r[0] * (1.0 / 33554432.0);
  const long long cnt = (long long)r[1];
  out->total_mass = total;
  out->mean_rho = cnt > 0 ? total / (double)cnt : 1.0;
  double ms;
  std::memcpy(&ms, &r[2], sizeof(ms));
  out->max_speed = ms;
  out->has_nan = (r[3] != 0 || s.nan_seen) ? 1 : 0;
  out->cumulative_rescale = s.cumulative_rescale;
  out->rescale_count = s.rescale_count;
  return AEROSIM_OK;
}

int aerosim_set_pipeline_wait_limit(aerosim_engine* h, int32_t polls) {
  if (!h) return AEROSIM_ERR_ARG;
  h->wait_limit = polls < 0 ? kWaitLimit : polls;
  return AEROSIM_OK;
}

int aerosim_step_param_bytes(void) { return (int)sizeof(StepArgs); }

int aerosim_last_step_timing(aerosim_engine* h, double* ms, int64_t* launches) {
  if (!h) return AEROSIM_ERR_ARG;
  if (ms) *ms = h->last_ms;
  if (launches) *launches = h->last_launches;
  return AEROSIM_OK;
}

// computeProjectedFrontalArea, frontalArea.ts:22-179: 4x4 supersampled coverage of
// the projected triangles on a res x res grid over the Y-Z bounding box.
int aerosim_frontal_area(const float* pos, int64_t nv, const int32_t* idx, int64_t ni, const double* m,
                         int32_t res, double* out) {
  if (!out || res <= 0 || nv < 0 || (nv > 0 && !pos)) return AEROSIM_ERR_ARG;
  *out = 0.0;
  if (nv < 3) return AEROSIM_OK;
  const int64_t T = idx ? ni / 3 : nv / 3;
  if (T == 0) return AEROSIM_OK;
  std::vector<double> py(nv), pz(nv);
  double y0 = INFINITY, y1 = -INFINITY, z0 = INFINITY, z1 = -INFINITY;
  for (int64_t i = 0; i < nv; ++i) {
    double x = pos[i * 3], y = pos[i * 3 + 1], z = pos[i * 3 + 2];
    if (m) {
      const double w = 1.0 / (m[3] * x + m[7] * y + m[11] * z + m[15]);
      const double ty = (m[1] * x + m[5] * y + m[9] * z + m[13]) * w;
      const double tz = (m[2] * x + m[6] * y + m[10] * z + m[14]) * w;
      y = ty; z = tz;
    }
    py[i] = y; pz[i] = z;
    y0 = y < y0 ? y : y0; y1 = y > y1 ? y : y1;
    z0 = z < z0 ? z : z0; z1 = z > z1 ? z : z1;
  }
  const double span_y = y1 - y0, span_z = z1 - z0;
  if (span_y <= 1e-9 || span_z <= 1e-9) return AEROSIM_OK;
  std::vector<uint16_t> cover((size_t)res * res, 0);
  const double sy = res / span_y, sz = res / span_z;
  static const double sub[4] = {0.125, 0.375, 0.625, 0.875};
  for (int64_t t = 0; t < T; ++t) {
    int64_t v[3];
    for (int k = 0; k < 3; ++k) v[k] = idx ? idx[t * 3 + k] : t * 3 + k;
    double Z[3], Y[3];
    for (int k = 0; k < 3; ++k) {
      if (v[k] < 0 || v[k] >= nv) return AEROSIM_ERR_ARG;
      Z[k] = (pz[v[k]] - z0) * sz;
      Y[k] = (py[v[k]] - y0) * sy;
    }
    const double area2 = (Z[1] - Z[0]) * (Y[2] - Y[0]) - (Y[1] - Y[0]) * (Z[2] - Z[0]);
    if (std::fabs(area2) < 1e-11) continue;
    if (area2 < 0) { std::swap(Z[1], Z[2]); std::swap(Y[1], Y[2]); }
    const int iz0 = (int)js_max(0, std::floor(js_min(js_min(Z[0], Z[1]), Z[2])));
    const int iz1 = (int)js_min(res - 1, std::floor(js_max(js_max(Z[0], Z[1]), Z[2])));
    const int iy0 = (int)js_max(0, std::floor(js_min(js_min(Y[0], Y[1]), Y[2])));
    const int iy1 = (int)js_min(res - 1, std::floor(js_max(js_max(Y[0], Y[1]), Y[2])));
    double ez[3], ey[3];
    for (int k = 0; k < 3; ++k) {
      ez[k] = Z[(k + 1) % 3] - Z[k];
      ey[k] = Y[(k + 1) % 3] - Y[k];
    }
    for (int iy = iy0; iy <= iy1; ++iy)
      for (int iz = iz0; iz <= iz1; ++iz) {
        uint16_t c = cover[(size_t)iy * res + iz];
        if (c == 0xffff) continue;
        for (int a = 0; a < 4; ++a)
          for (int b = 0; b < 4; ++b) {
            const uint16_t bit = (uint16_t)(1u << (a * 4 + b));
            if (c & bit) continue;
            const double Py = iy + sub[a], Pz = iz + sub[b];
            bool in = true;
            for (int k = 0; k < 3 && in; ++k) in = ez[k] * (Py - Y[k]) - ey[k] * (Pz - Z[k]) >= -1e-9;
            if (in) c |= bit;
          }
        cover[(size_t)iy * res + iz] = c;
      }
  }
  long long covered = 0;
  for (uint16_t c : cover) covered += __builtin_popcount(c);
  *out = ((double)covered / ((double)res * res * 16)) * (span_y * span_z);
  return AEROSIM_OK;
}

}  // extern "C"

namespace {

// Slice size and, with rgba, the enqueued slice kernel and its copy to rgba.
int enqueue_slice(aerosim_engine* h, int32_t axis, double fraction, int32_t mode, uint8_t* rgba, int32_t* width,
                  int32_t* height) {
  if (axis < 0 || axis > 2 || mode < 0 || mode > 2) return fail(h, AEROSIM_ERR_ARG, "extract_slice: bad axis or mode");
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "extract_slice: no voxel grid");
  const int nx = h->g.nx, ny = h->g.ny, nz = h->g.nz;
  int w = nx, hh = ny;
  if (axis == 1) { w = nx; hh = nz; }
  else if (axis == 0) { w = nz; hh = ny; }
  *width = w;
  *height = hh;
  if (!rgba) return AEROSIM_OK;
  // the fixed coordinate, Math.min(n - 1, Math.max(0, Math.floor(fraction * n)))
  const int n = axis == 0 ? nx : axis == 1 ? ny : nz;
  const int fixed = (int)js_min(n - 1, js_max(0, std::floor(fraction * n)));
  CU(h, cudaSetDevice(h->device));
  const size_t bytes = (size_t)w * hh * 4;
  int rc = ensure_staging(h, bytes);
  if (rc) return rc;
  if (bytes > h->slice_host_bytes) {
    if (h->slice_host) cudaFreeHost(h->slice_host);
    h->slice_host = nullptr;
    h->slice_host_bytes = 0;
    CU(h, cudaHostAlloc((void**)&h->slice_host, bytes, cudaHostAllocDefault));
    h->slice_host_bytes = bytes;
  }
  CU(h, launch_slice(h->mux, h->muy, h->muz, h->mrho, h->g.cls, h->st, prev_slot(h), h->L, axis, fixed, mode,
                     js_max(1e-4, h->cfg.u_inlet_lattice), w, hh, static_cast<uint8_t*>(h->staging), h->stream));
  // into pinned memory inside the stream (no host round trip of a pageable copy; the
  // kernel's own byte stores to mapped host memory measured slower); the caller copies
  // it into its buffer once the stream has drained
  CU(h, cudaMemcpyAsync(h->slice_host, h->staging, bytes, cudaMemcpyDeviceToHost, h->stream));
  h->slice_bytes = bytes;
  return AEROSIM_OK;
}

}  // namespace

extern "C" int aerosim_extract_slice(aerosim_engine* h, int32_t axis, double fraction, int32_t mode, uint8_t* rgba,
                                     int32_t* width, int32_t* height) {
  if (!h || !width || !height) return AEROSIM_ERR_ARG;
  int rc = enqueue_slice(h, axis, fraction, mode, rgba, width, height);
  if (rc || !rgba) return rc;
  CU(h, cudaStreamSynchronize(h->stream));
  std::memcpy(rgba, h->slice_host, h->slice_bytes);
  return AEROSIM_OK;
}

// stepAndExtractSlice(substeps), lbmEngine.ts:404-675, as one call: the substeps, the
// force reduction and (with rgba) the slice image are enqueued back to back and the
// stream is drained once; the force sums and the device error flag return through a
// pinned buffer of the engine.
extern "C" int aerosim_step_and_extract_slice(aerosim_engine* h, int32_t n, int32_t axis, double fraction,
                                              int32_t mode, uint8_t* rgba, int32_t* width, int32_t* height,
                                              aerosim_forces* forces) {
  if (!h || !forces || (rgba && (!width || !height))) return AEROSIM_ERR_ARG;
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "step_and_extract_slice: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  int rc = ensure_frame_host(h);
  if (rc) return rc;
  double* sums = h->frame_host;
  int* dev_err = reinterpret_cast<int*>(h->frame_host + 8);
  *dev_err = 0;
  for (int i = 0; i < 8; ++i) sums[i] = 0.0;
  if ((rc = enqueue_steps(h, n))) return rc;
  if (h->g.B > 0) {  // the force kernel's last CTA writes the sums and the error code
    if ((rc = enqueue_forces(h, sums, h->frame_dev, reinterpret_cast<int*>(h->frame_dev + 8)))) return rc;
  } else {
    CU(h, cudaMemcpyAsync(dev_err, &h->st->error, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  }
  if (rgba && (rc = enqueue_slice(h, axis, fraction, mode, rgba, width, height))) return rc;
  CU(h, cudaStreamSynchronize(h->stream));
  if (rgba) std::memcpy(rgba, h->slice_host, h->slice_bytes);
  if ((rc = finish_steps(h, *dev_err))) return rc;
  forces_from_sums(h, sums, forces);
  return AEROSIM_OK;
}

namespace {

// Q-criterion of device velocity fields into host outputs (staging: 5 floats per cell).
int q_criterion_to_host(aerosim_engine* h, int nx, int ny, int nz, double dx, const float* ux, const float* uy,
                        const float* uz, const uint8_t* flags, float* q, float* om, float* omv, double* max_q,
                        double* max_om) {
  const long long N = (long long)nx * ny * nz;
  int rc = ensure_staging(h, N * 5 * sizeof(float) + 16);
  if (rc) return rc;
  float* dq = static_cast<float*>(h->staging);
  float* dom = dq + N;
  float* domv = dom + N;
  unsigned long long* dmax = h->stats_buf;
  CU(h, launch_q_criterion(nx, ny, nz, dx, ux, uy, uz, flags, dq, dom, domv, dmax, h->stream));
  unsigned long long mx[2] = {0, 0};
  if (q) CU(h, cudaMemcpyAsync(q, dq, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (om) CU(h, cudaMemcpyAsync(om, dom, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (omv) CU(h, cudaMemcpyAsync(omv, domv, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaMemcpyAsync(mx, dmax, sizeof(mx), cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  double a, b;
  std::memcpy(&a, &mx[0], 8);
  std::memcpy(&b, &mx[1], 8);
  if (max_q) *max_q = std::max(1e-6, a);
  if (max_om) *max_om = std::max(1e-6, b);
  return AEROSIM_OK;
}

}  // namespace

extern "C" int aerosim_q_criterion(aerosim_engine* h, float* q, float* omega_mag, float* omega_vec, double* max_q,
                                   double* max_omega) {
  if (!h) return AEROSIM_ERR_ARG;
  if (!h->have_grid || !h->f[0]) return fail(h, AEROSIM_ERR_STATE, "q_criterion: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  return q_criterion_to_host(h, h->g.nx, h->g.ny, h->g.nz, h->dx, h->mux, h->muy, h->muz, h->g.flags, q, omega_mag,
                             omega_vec, max_q, max_omega);
}

extern "C" int aerosim_q_criterion_fields(aerosim_engine* h, int32_t nx, int32_t ny, int32_t nz, double dx,
                                          const float* ux, const float* uy, const float* uz, const uint8_t* flags,
                                          float* q, float* omega_mag, float* omega_vec, double* max_q,
                                          double* max_omega) {
  if (!h || !ux || !uy || !uz || nx < 1 || ny < 1 || nz < 1 || !(dx > 0.0))
    return fail(h, AEROSIM_ERR_ARG, "q_criterion_fields: bad argument");
  CU(h, cudaSetDevice(h->device));
  const long long N = (long long)nx * ny * nz;
  void* buf = nullptr;
  CU(h, cudaMalloc(&buf, N * (3 * sizeof(float) + 1)));
  float* d = static_cast<float*>(buf);
  uint8_t* df = reinterpret_cast<uint8_t*>(d + 3 * N);
  cudaError_t e = cudaMemcpyAsync(d, ux, N * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + N, uy, N * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + 2 * N, uz, N * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && flags) e = cudaMemcpyAsync(df, flags, N, cudaMemcpyHostToDevice, h->stream);
  int rc = e == cudaSuccess ? q_criterion_to_host(h, nx, ny, nz, dx, d, d + N, d + 2 * N, flags ? df : nullptr, q,
                                                  omega_mag, omega_vec, max_q, max_omega)
                            : fail(h, AEROSIM_ERR_CUDA, std::string("q_criterion_fields: ") + cudaGetErrorString(e));
  cudaStreamSynchronize(h->stream);
  cudaFree(buf);
  return rc;
}

// ---------------------------------------------------------------------------
// Learned SGS closure of an engine.
// ---------------------------------------------------------------------------
namespace {

int ensure_wall_distance(aerosim_engine* h) {
  if (h->wall_ready) return AEROSIM_OK;
  CU(h, compute_wall_distance(h->g.flags, h->g.nx, h->g.ny, h->g.nz, nullptr, h->g.cls, h->L.pitch, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  h->wall_ready = true;
  return AEROSIM_OK;
}

double effective_nu0(const aerosim_engine* h) {
  return (std::max(3.0 * h->cfg.nu_lattice + 0.5, 0.5015) - 0.5) / 3.0;
}

}  // namespace

extern "C" {

int aerosim_set_sgs_mlp(aerosim_engine* h, const float* params) {
  if (!h) return AEROSIM_ERR_ARG;
  CU(h, cudaSetDevice(h->device));
  if (!params) {
    cudaFree(h->mlp_frag); cudaFree(h->mlp_bias); cudaFree(h->mlp_umma);
    h->mlp_frag = nullptr;
    h->mlp_bias = nullptr;
    h->mlp_umma = nullptr;
  } else {
    for (int i = 0; i < kMlpParams; ++i)
      if (!std::isfinite(params[i])) return fail(h, AEROSIM_ERR_ARG, "set_sgs_mlp: non-finite parameter");
    std::vector<uint32_t> frag(kMlpFragWords * 32);
    std::vector<float> bias(kMlpBias);
    mlp_pack_fragments(params, frag.data(), bias.data());
    std::vector<uint16_t> img(kUmmaBBytes / 2);
    mlp_pack_umma(params, img.data());
    if (!h->mlp_frag) {
      CU(h, cudaMalloc(&h->mlp_frag, frag.size() * sizeof(uint32_t)));
      CU(h, cudaMalloc(&h->mlp_bias, bias.size() * sizeof(float)));
      CU(h, cudaMalloc(&h->mlp_umma, kUmmaBBytes));
    }
    CU(h, cudaMemcpy(h->mlp_frag, frag.data(), frag.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CU(h, cudaMemcpy(h->mlp_bias, bias.data(), bias.size() * sizeof(float), cudaMemcpyHostToDevice));
    CU(h, cudaMemcpy(h->mlp_umma, img.data(), kUmmaBBytes, cudaMemcpyHostToDevice));
    if (h->have_grid) {
      int rc = ensure_wall_distance(h);
      if (rc) return rc;
    }
  }
  if (h->have_grid && h->f[0]) return configure_step(h);
  return AEROSIM_OK;
}

int aerosim_set_sgs_mlp_path(aerosim_engine* h, int32_t path, int32_t* in_use) {
  if (!h) return AEROSIM_ERR_ARG;
  if (path != AEROSIM_SGS_PATH_DEFAULT && path != AEROSIM_SGS_PATH_WARP && path != AEROSIM_SGS_PATH_TCGEN05)
    return fail(h, AEROSIM_ERR_ARG, "set_sgs_mlp_path: unknown path");
  CU(h, cudaSetDevice(h->device));
  h->mlp_path = path;
  if (h->have_grid && h->f[0]) {
    const int rc = configure_step(h);
    if (rc) return rc;
  }
  if (in_use)
    *in_use = !h->mlp_frag ? AEROSIM_SGS_PATH_DEFAULT
                           : (closure_umma(h) ? AEROSIM_SGS_PATH_TCGEN05 : AEROSIM_SGS_PATH_WARP);
  return AEROSIM_OK;
}

int aerosim_read_wall_distance(aerosim_engine* h, float* out) {
  if (!h || !out) return AEROSIM_ERR_ARG;
  if (!h->have_grid) return fail(h, AEROSIM_ERR_STATE, "read_wall_distance: no voxel grid");
  CU(h, cudaSetDevice(h->device));
  const long long N = h->g.N;
  int rc = ensure_staging(h, N * sizeof(float));
  if (rc) return rc;
  CU(h, compute_wall_distance(h->g.flags, h->g.nx, h->g.ny, h->g.nz, static_cast<float*>(h->staging), h->g.cls,
                              h->L.pitch, h->stream));
  h->wall_ready = true;
  CU(h, cudaMemcpyAsync(out, h->staging, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  CU(h, cudaStreamSynchronize(h->stream));
  return AEROSIM_OK;
}

int aerosim_sgs_samples(aerosim_engine* fine, aerosim_engine* coarse, float min_ratio, float max_ratio,
                        int32_t average_radius, float* X, float* Y, uint8_t* valid) {
  if (!fine || !coarse || !X || !Y || !valid || !(max_ratio > 0.0f) || !(min_ratio <= 0.0f) ||
      !(min_ratio >= -max_ratio) || average_radius < 0 || average_radius > 4)
    return fail(nullptr, AEROSIM_ERR_ARG, "sgs_samples: bad argument");
  if (!fine->have_grid || !fine->f[0] || !coarse->have_grid)
    return fail(nullptr, AEROSIM_ERR_STATE, "sgs_samples: both engines need a voxel grid (and the fine one a flow)");
  if (fine->device != coarse->device) return fail(nullptr, AEROSIM_ERR_ARG, "sgs_samples: engines on different devices");
  const DevGrid &f = fine->g, &c = coarse->g;
  if (f.nx != 2 * c.nx || f.ny != 2 * c.ny || f.nz != 2 * c.nz)
    return fail(nullptr, AEROSIM_ERR_ARG, "sgs_samples: the fine lattice must be exactly twice the coarse one");
  CU(coarse, cudaSetDevice(coarse->device));
  CU(fine, cudaStreamSynchronize(fine->stream));
  int rc = ensure_wall_distance(coarse);
  if (rc) return rc;
  const long long Nc = c.N;
  float *dx = nullptr, *dy = nullptr;
  uint8_t* dv = nullptr;
  cudaError_t e = cudaMalloc(&dx, Nc * kMlpIn * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dy, Nc * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dv, Nc);
  if (e == cudaSuccess)
    e = launch_sgs_samples(fine->mux, fine->muy, fine->muz, fine->mrho, f.flags, f.nx, f.ny, f.nz, c.cls,
                           coarse->L.pitch, c.nx, c.ny, c.nz, (float)effective_nu0(coarse), min_ratio, max_ratio,
                           average_radius,
                           dx, dy, dv,
                           coarse->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(X, dx, Nc * kMlpIn * sizeof(float), cudaMemcpyDeviceToHost, coarse->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Y, dy, Nc * sizeof(float), cudaMemcpyDeviceToHost, coarse->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(valid, dv, Nc, cudaMemcpyDeviceToHost, coarse->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(coarse->stream);
  cudaFree(dx); cudaFree(dy); cudaFree(dv);
  if (e != cudaSuccess) return fail(nullptr, AEROSIM_ERR_CUDA, std::string("sgs_samples: ") + cudaGetErrorString(e));
  return AEROSIM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches: many engines stepped by one persistent launch per step.
// ---------------------------------------------------------------------------
struct aerosim_batch {
  int device = 0;
  int precision = 0;
  std::vector<aerosim_engine*> eng;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  StepArgs* d_inst = nullptr;
  void** d_bufs = nullptr;
  long long* d_item_begin = nullptr;
  long long* d_near_begin = nullptr;
  int4* d_geo = nullptr;
  unsigned long long* d_partials = nullptr;
  unsigned int* d_ticket = nullptr;  // [2]
  int* d_step = nullptr;
  int* d_error = nullptr;
  long long n_items = 0, n_near = 0, cells = 0;
  long long slot_elems = 0, slot_cls = 0;
  int item_cells = 0;  // cells per work item of the current item list
  int pitch = 0;  // row pitch shared by all instances (0: they differ)
  int num_sms = 148;
  aerosim_batch_tuning tune{};
  unsigned grid = 1;
  size_t smem = 0;
  cudaGraphExec_t graph = nullptr;
  int graph_len = 0;
  int step = 0;
  double last_ms = 0;
  long long last_launches = 0;
  int wait_limit = kWaitLimit;  // polls of a ring wait before the batched step gives up
  int cells_per_thread = 1;     // 2 when every instance has an even nx (pair_segment)
};

namespace {

int bfail(int code, const std::string& msg) { return fail(nullptr, code, msg); }

#define BCU(x)                                                                            \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) return bfail(AEROSIM_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

void batch_free(aerosim_batch* b) {
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->d_inst); cudaFree(b->d_bufs); cudaFree(b->d_item_begin); cudaFree(b->d_near_begin);
  cudaFree(b->d_geo);
  cudaFree(b->d_partials); cudaFree(b->d_ticket); cudaFree(b->d_step); cudaFree(b->d_error);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
}

// The solver arguments of every instance, from its engine's current configuration.
int batch_upload_table(aerosim_batch* b) {
  std::vector<StepArgs> t(b->eng.size());
  for (size_t k = 0; k < b->eng.size(); ++k) {
    const aerosim_engine* e = b->eng[k];
    StepArgs& a = t[k];
    a = StepArgs{};
    a.cls = e->g.cls; a.bmap = e->g.bmap; a.q = e->g.q;
    a.mux = e->mux; a.muy = e->muy; a.muz = e->muz; a.mrho = e->mrho;
    a.abl = e->abl; a.sin_tab = e->sin_tab; a.st = e->st;
    a.L = e->L; a.fluid_count = e->fluid_count;
    a.near_cells = e->near_cells; a.n_near = e->n_near; a.links = e->links; a.links_f = e->links_f;
    a.ground_no_slip = e->cfg.ground_no_slip;
    a.u_inlet = e->cfg.u_inlet_lattice;
    a.tau0 = 3.0 * e->cfg.nu_lattice + 0.5;
    a.k_smag = 18.0 * M_SQRT2 * e->cfg.smagorinsky_cs * e->cfg.smagorinsky_cs;
  }
  BCU(cudaMemcpyAsync(b->d_inst, t.data(), t.size() * sizeof(StepArgs), cudaMemcpyHostToDevice, b->stream));
  return AEROSIM_OK;
}

BatchArgs batch_args(const aerosim_batch* b, int write_macro) {
  BatchArgs a{};
  a.inst = b->d_inst; a.bufs = b->d_bufs; a.item_begin = b->d_item_begin; a.near_begin = b->d_near_begin;
  a.partials = b->d_partials; a.ticket = b->d_ticket; a.step = b->d_step; a.error = b->d_error;
  a.geo = b->d_geo;
  a.n_items = b->n_items; a.n_near = b->n_near; a.slot_elems = b->slot_elems; a.slot_cls = b->slot_cls;
  a.n_inst = (int)b->eng.size(); a.stages = b->tune.stages; a.write_macro = write_macro;
  a.wait_limit = b->wait_limit;
  a.cells_per_thread = b->cells_per_thread;
  return a;
}

// Launch shape of a tuning: the shared memory of its ring and the persistent grid, or
// an error when the configuration does not fit.
// Rows per work item of a lattice for a target of item_cells cells per item (0: 256).
int batch_rows_per_item(const Layout& L, int item_cells) {
  const int span = (L.nx + row_shift(L.nx) + 31) / 32 * 32;
  if (item_cells <= 0) return rows_per_item(L.nx);
  return std::max(1, std::min(kMaxRowsPerItem, item_cells / span));
}

// The flat item list for item_cells cells per item: first item of each instance, rows per
// item / segments per row / row shift of each instance, and the ring slot sizes.
int batch_build_items(aerosim_batch* b, int item_cells) {
  const int n = (int)b->eng.size();
  std::vector<long long> item_begin(n + 1, 0);
  std::vector<int4> geo(n);
  long long slot_elems = 0, slot_cls = 0;
  for (int k = 0; k < n; ++k) {
    const Layout& L = b->eng[k]->L;
    const int RY = batch_rows_per_item(L, item_cells);
    const long long rows = (long long)L.ny * L.nz;
    item_begin[k + 1] = item_begin[k] + (rows + RY - 1) / RY;
    geo[k] = b->cells_per_thread == 2 ? make_int4(RY, (L.nx + 63) / 64, 0, 0)  // 64-cell pair segments
                                      : make_int4(RY, (L.nx + row_shift(L.nx) + 31) / 32, row_shift(L.nx), 0);
    slot_elems = std::max<long long>(slot_elems, (long long)RY * 19 * L.pitch);
    slot_cls = std::max<long long>(slot_cls, (long long)RY * L.pitch);
  }
  BCU(cudaMemcpy(b->d_item_begin, item_begin.data(), item_begin.size() * sizeof(long long), cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(b->d_geo, geo.data(), geo.size() * sizeof(int4), cudaMemcpyHostToDevice));
  b->n_items = item_begin[n];
  b->slot_elems = slot_elems;
  b->slot_cls = slot_cls;
  b->item_cells = item_cells;
  return AEROSIM_OK;
}

int batch_configure(aerosim_batch* b, const aerosim_batch_tuning& t, unsigned* grid, size_t* smem) {
  if (t.stages < 2 || t.stages > 6 || t.ctas_per_sm < 1 || t.ctas_per_sm > 3 || t.graph_steps < 1 ||
      t.item_cells < 0 || t.item_cells > 2048)
    return bfail(AEROSIM_ERR_ARG,
                 "batch: tuning out of range (stages 2..6, ctas_per_sm 1..3, graph_steps >= 1, item_cells 0..2048)");
  if (t.item_cells != b->item_cells) {
    int rc = batch_build_items(b, t.item_cells);
    if (rc) return rc;
  }
  const size_t eb = precision_bytes(b->precision);
  const size_t sm = batch_smem_bytes(b->slot_elems, b->slot_cls, t.stages, eb);
  if (sm > 227 * 1024) return bfail(AEROSIM_ERR_ARG, "batch: the ring does not fit shared memory");
  BatchArgs a = batch_args(b, 0);
  a.stages = t.stages;
  int occ = 0;
  BCU(launch_batch(b->precision, a, b->pitch, 0, sm, b->stream, &occ));
  if (occ < t.ctas_per_sm) return bfail(AEROSIM_ERR_ARG, "batch: fewer resident CTAs per SM than requested");
  long long g = (long long)t.ctas_per_sm * b->num_sms;
  if (g > b->n_items) g = b->n_items;
  *grid = (unsigned)(g < 1 ? 1 : g);
  *smem = sm;
  return AEROSIM_OK;
}

int batch_apply_tuning(aerosim_batch* b, const aerosim_batch_tuning& t) {
  unsigned grid = 0;
  size_t smem = 0;
  const int prev_cells = b->item_cells;
  int rc = batch_configure(b, t, &grid, &smem);
  if (rc) {
    // keep the item list of the configuration in force
    if (b->item_cells != prev_cells) {
      std::string msg = aerosim_last_error(nullptr);
      if (batch_build_items(b, prev_cells) == AEROSIM_OK) bfail(rc, msg);
    }
    return rc;
  }
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->tune = t;
  b->grid = grid;
  b->smem = smem;
  return AEROSIM_OK;
}

// Fresh flow in every instance and the batch's step counter at zero.
int batch_reset(aerosim_batch* b) {
  for (aerosim_engine* e : b->eng) {
    BCU(cudaSetDevice(e->device));
    if (do_reset(e)) return bfail(AEROSIM_ERR_CUDA, "batch: reset of an instance failed: " + e->err);
  }
  BCU(cudaSetDevice(b->device));
  BCU(cudaMemsetAsync(b->d_step, 0, sizeof(int), b->stream));
  BCU(cudaMemsetAsync(b->d_ticket, 0, 2 * sizeof(unsigned int), b->stream));
  BCU(cudaMemsetAsync(b->d_error, 0, sizeof(int), b->stream));
  BCU(cudaStreamSynchronize(b->stream));
  b->step = 0;
  return AEROSIM_OK;
}

// Enqueues n batched steps: replays of the captured graph of tune.graph_steps launches,
// then single launches; the last step writes the macro fields.
int batch_enqueue(aerosim_batch* b, int n, long long* launches) {
  const int G = b->tune.graph_steps;
  int done = 0;
  if (G > 1 && n >= G) {
    if (!b->graph) {
      cudaGraph_t g = nullptr;
      BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t le = cudaSuccess;
      for (int i = 0; i < G && le == cudaSuccess; ++i) {
        const BatchArgs a = batch_args(b, i == G - 1 ? 1 : 0);
        le = launch_batch(b->precision, a, b->pitch, b->grid, b->smem, b->stream, nullptr);
      }
      const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
      if (le != cudaSuccess || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return bfail(AEROSIM_ERR_CUDA, std::string("batch: graph capture failed: ") +
                                           cudaGetErrorString(le != cudaSuccess ? le : ce));
      }
      const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        b->graph = nullptr;
        return bfail(AEROSIM_ERR_CUDA, std::string("batch: graph instantiation failed: ") + cudaGetErrorString(ie));
      }
      b->graph_len = G;
    }
    for (; done + G <= n; done += G) {
      BCU(cudaGraphLaunch(b->graph, b->stream));
      *launches += G;
    }
  }
  for (; done < n; ++done) {
    const BatchArgs a = batch_args(b, done == n - 1 ? 1 : 0);
    BCU(launch_batch(b->precision, a, b->pitch, b->grid, b->smem, b->stream, nullptr));
    *launches += 1;
  }
  return AEROSIM_OK;
}

}  // namespace

extern "C" {

int aerosim_batch_create(aerosim_engine* const* engines, int32_t n, aerosim_batch** out) {
  if (!out) return bfail(AEROSIM_ERR_ARG, "batch_create: out is NULL");
  *out = nullptr;
  if (!engines || n < 1 || n > kMaxBatch) return bfail(AEROSIM_ERR_ARG, "batch_create: 1..64 engines required");
  for (int k = 0; k < n; ++k) {
    const aerosim_engine* e = engines[k];
    if (!e) return bfail(AEROSIM_ERR_ARG, "batch_create: NULL engine");
    if (!e->have_grid || !e->f[0]) return bfail(AEROSIM_ERR_STATE, "batch_create: an engine has no voxel grid");
    if (e->device != engines[0]->device) return bfail(AEROSIM_ERR_ARG, "batch_create: engines on different devices");
    if (e->cfg.precision != engines[0]->cfg.precision)
      return bfail(AEROSIM_ERR_ARG, "batch_create: engines with different precisions");
    for (int j = 0; j < k; ++j)
      if (engines[j] == e) return bfail(AEROSIM_ERR_ARG, "batch_create: an engine appears twice");
  }
  const int prec = engines[0]->cfg.precision;
  if (prec != AEROSIM_PREC_F32 && prec != AEROSIM_PREC_F16S && prec != AEROSIM_PREC_BF16S && prec != AEROSIM_PREC_F16C)
    return bfail(AEROSIM_ERR_ARG, "batch_create: batches run the F32, F16S, BF16S and F16C precisions");
  aerosim_batch* b = new (std::nothrow) aerosim_batch();
  if (!b) return bfail(AEROSIM_ERR_NOMEM, "batch_create: out of host memory");
  b->device = engines[0]->device;
  b->precision = prec;
  b->eng.assign(engines, engines + n);
  b->num_sms = engines[0]->num_sms;
  // two cells per consumer thread when every instance's rows have an even cell count
  // (AEROSIM_CELLS_PER_THREAD=1 keeps one)
  b->cells_per_thread = 2;
  for (int k = 0; k < n; ++k)
    if (engines[k]->L.nx % 2 != 0 || engines[k]->L.nx < 4) b->cells_per_thread = 1;
  if (const char* cenv = getenv("AEROSIM_CELLS_PER_THREAD"))
    if (atoi(cenv) == 1) b->cells_per_thread = 1;
  auto bail = [&](int rc) {
    std::string msg = aerosim_last_error(nullptr);
    batch_free(b);
    delete b;
    return bfail(rc, msg);
  };
  cudaError_t e = cudaSetDevice(b->device);
  std::vector<long long> near_begin(n + 1, 0);
  std::vector<void*> bufs(2 * (size_t)n);
  int pitch = engines[0]->L.pitch;
  for (int k = 0; k < n; ++k) {
    const aerosim_engine* en = engines[k];
    const Layout& L = en->L;
    near_begin[k + 1] = near_begin[k] + en->n_near;
    bufs[2 * k] = en->f[0];
    bufs[2 * k + 1] = en->f[1];
    b->cells += en->g.N;
    if (L.pitch != pitch) pitch = 0;
  }
  b->pitch = (pitch == 64 || pitch == 128 || pitch == 192 || pitch == 256) ? pitch : 0;
  b->n_near = near_begin[n];
  const size_t part = (size_t)3 * b->num_sms * n;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_inst, n * sizeof(StepArgs));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_bufs, 2 * n * sizeof(void*));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_item_begin, (n + 1) * sizeof(long long));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_near_begin, (n + 1) * sizeof(long long));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_geo, n * sizeof(int4));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_partials, part * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_ticket, 2 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_step, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_error, sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_bufs, bufs.data(), bufs.size() * sizeof(void*), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_near_begin, near_begin.data(), near_begin.size() * sizeof(long long), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    bfail(AEROSIM_ERR_CUDA, std::string("batch_create: ") + cudaGetErrorString(e));
    return bail(AEROSIM_ERR_CUDA);
  }
  int rc = batch_build_items(b, 0);
  if (rc) return bail(rc);
  rc = batch_reset(b);
  if (!rc) rc = batch_upload_table(b);
  if (rc) return bail(rc);
  // default launch: the most resident CTAs per SM that a 3-slot ring allows (at least a
  // 2-slot ring), 20 launches per graph
  aerosim_batch_tuning t{3, 3, 20, 0, 0.0};
  rc = AEROSIM_ERR_ARG;
  for (int stages = 3; stages >= 2 && rc; --stages)
    for (int c = 3; c >= 1 && rc; --c) {
      t.stages = stages;
      t.ctas_per_sm = c;
      rc = batch_apply_tuning(b, t);
    }
  if (rc) return bail(rc);
  *out = b;
  return AEROSIM_OK;
}

int aerosim_batch_destroy(aerosim_batch* b) {
  if (!b) return AEROSIM_OK;
  batch_free(b);
  delete b;
  return AEROSIM_OK;
}

int aerosim_batch_step(aerosim_batch* b, int32_t n) {
  if (!b) return bfail(AEROSIM_ERR_ARG, "batch_step: NULL batch");
  if (n < 0) return bfail(AEROSIM_ERR_ARG, "batch_step: negative step count");
  if ((long long)b->step + n > 0x7fffffffLL) return bfail(AEROSIM_ERR_ARG, "batch_step: step index overflow");
  BCU(cudaSetDevice(b->device));
  for (aerosim_engine* e : b->eng) BCU(cudaStreamSynchronize(e->stream));
  int rc = batch_upload_table(b);
  if (rc) return rc;
  long long launches = 0;
  BCU(cudaEventRecord(b->ev0, b->stream));
  rc = batch_enqueue(b, n, &launches);
  if (rc) return rc;
  BCU(cudaEventRecord(b->ev1, b->stream));
  int dev_err = 0;
  BCU(cudaMemcpyAsync(&dev_err, b->d_error, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCU(cudaStreamSynchronize(b->stream));
  float ms = 0.f;
  BCU(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->last_ms = ms;
  b->last_launches = launches;
  b->step += n;
  for (aerosim_engine* e : b->eng) {
    e->step_index = b->step;
    e->cur = b->step & 1;
  }
  if (dev_err) return bfail(AEROSIM_ERR_DEVICE, "batch_step: the shared-memory pipeline timed out (device error flag set)");
  return AEROSIM_OK;
}

int aerosim_batch_autotune(aerosim_batch* b, int32_t steps_per_trial, aerosim_batch_tuning* out) {
  if (!b) return bfail(AEROSIM_ERR_ARG, "batch_autotune: NULL batch");
  if (steps_per_trial < 1) return bfail(AEROSIM_ERR_ARG, "batch_autotune: steps_per_trial must be positive");
  BCU(cudaSetDevice(b->device));
  // trials start from fresh flows and a cleared error flag (a step that timed out before
  // the autotune leaves the flag set until the batch is reset)
  int rc0 = batch_reset(b);
  if (rc0) return rc0;
  const aerosim_batch_tuning keep = b->tune;
  aerosim_batch_tuning best = keep;
  best.ms_per_step = 1e300;
  for (int cells : {256, 512, 1024})
    for (int stages = 2; stages <= 6; ++stages)
      for (int c = 1; c <= 3; ++c) {
        aerosim_batch_tuning t{stages, c, 1, cells, 0.0};
        if (batch_apply_tuning(b, t) != AEROSIM_OK) continue;  // does not fit: skip
        int rc = aerosim_batch_step(b, 2);
        if (!rc) rc = aerosim_batch_step(b, steps_per_trial);
        if (rc) return rc;
        const double per = b->last_ms / steps_per_trial;
        if (per < best.ms_per_step) {
          best = t;
          best.ms_per_step = per;
        }
      }
  best.graph_steps = keep.graph_steps;
  int rc = batch_apply_tuning(b, best);
  if (rc) return rc;
  b->tune.ms_per_step = best.ms_per_step;
  rc = batch_reset(b);
  if (rc) return rc;
  if (out) *out = b->tune;
  return AEROSIM_OK;
}

int aerosim_batch_set_pipeline_wait_limit(aerosim_batch* b, int32_t polls) {
  if (!b) return bfail(AEROSIM_ERR_ARG, "batch_set_pipeline_wait_limit: NULL batch");
  BCU(cudaSetDevice(b->device));
  BCU(cudaStreamSynchronize(b->stream));
  b->wait_limit = polls < 0 ? kWaitLimit : polls;
  if (b->graph) {  // the captured launches carry the old limit
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return AEROSIM_OK;
}

int aerosim_batch_set_tuning(aerosim_batch* b, const aerosim_batch_tuning* t) {
  if (!b || !t) return bfail(AEROSIM_ERR_ARG, "batch_set_tuning: NULL argument");
  BCU(cudaSetDevice(b->device));
  return batch_apply_tuning(b, *t);
}

int aerosim_batch_get_tuning(aerosim_batch* b, aerosim_batch_tuning* out) {
  if (!b || !out) return bfail(AEROSIM_ERR_ARG, "batch_get_tuning: NULL argument");
  *out = b->tune;
  return AEROSIM_OK;
}

int aerosim_batch_last_timing(aerosim_batch* b, double* ms, int64_t* kernel_launches) {
  if (!b) return bfail(AEROSIM_ERR_ARG, "batch_last_timing: NULL batch");
  if (ms) *ms = b->last_ms;
  if (kernel_launches) *kernel_launches = b->last_launches;
  return AEROSIM_OK;
}

int aerosim_batch_cells(aerosim_batch* b, int64_t* out) {
  if (!b || !out) return bfail(AEROSIM_ERR_ARG, "batch_cells: NULL argument");
  *out = b->cells;
  return AEROSIM_OK;
}

}  // extern "C"
