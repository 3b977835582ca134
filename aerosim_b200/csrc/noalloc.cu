// aerosim_momentum_exchange_noalloc: the FP64 momentum-exchange force reduction
// over buffers the caller already holds on the device, without any device
// allocation by this library.
//
// Who needs it: hosts that own every byte of device memory through their own
// allocator or arena (a framework's caching allocator, an engine with a fixed VRAM
// budget) and do not let third-party code call cudaMalloc, and frame loops that
// cannot afford cudaMalloc/cudaFree, which may synchronise the device.  The caller
// passes inputs and outputs as device pointers; the reduction's scratch (one row of
// partial sums per CTA and a completion ticket) lives in the file-scope array below.
//
// Limits and sharing: at most kNoAllocMaxBlocks CTAs of 256 threads, i.e. 1 048 576
// boundary cells per call; larger inputs are rejected.  The array exists once per
// device that loads the library and stays allocated until the process exits.  Every
// call on a device uses the same array, so calls whose kernels overlap on the GPU
// (different streams, or several host threads) race and must be serialised by the
// caller; the ticket is cleared on the call's stream before each launch.
//
// Set-up: the first call on each device, with that device current, resolves the
// array's device address with cudaGetSymbolAddress (in host code the array's name is
// only a host-side stand-in, not a device address).  That first call should come
// before any stream capture on the device.  The address is kept with the ID of the
// device's current context: a cudaDeviceReset by the host ends that context and
// unloads the array with it, so the first call in the new context resolves the address
// again instead of using the old one.
//
// Preconditions the kernel does not check: every boundary_cells[b] lies in
// [0, nx * ny * nz), and q holds 18 values per boundary cell in the same order.
#include <cuda.h>  // CUcontext / CUresult types; the driver functions are fetched at run time
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/aerosim.h"
#include "common.cuh"
#include "engine_internal.h"
#include "lbm_kernels.cuh"

namespace aerosim {

namespace {

constexpr int kNoAllocMaxBlocks = 4096;
constexpr size_t kPartialBytes = (size_t)kNoAllocMaxBlocks * 8 * sizeof(double);
constexpr size_t kScratchBytes = kPartialBytes + 256;  // partial sums, then the ticket

// Device scratch of the no-allocation force reduction (256 KB + 256 B per device).
static __device__ __align__(256) unsigned char g_force_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // context ID the address belongs to

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Process-unique ID of the calling thread's current context (CUDA 12.0 cuCtxGetId, taken
// from the driver through the runtime, so the library does not link libcuda); 0 when it
// cannot be read, in which case the address is resolved on every call.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Device address of g_force_scratch on the current device: resolved at the first call
// in each context of the device and kept for the calls that follow.
cudaError_t scratch_address(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned long long ctx = current_context_id();
  if (!g_scratch_addr[device] || ctx == 0 || ctx != g_scratch_ctx[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_force_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = p;
    g_scratch_ctx[device] = ctx;
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace aerosim

using namespace aerosim;

extern "C" int aerosim_momentum_exchange_noalloc(const float* f, const uint8_t* flags, const int32_t* boundary_cells,
                                                 const float* q, int64_t boundary_count, int32_t nx, int32_t ny,
                                                 int32_t nz, double* out, void* stream) {
  auto err = [](int code, const std::string& m) {
    set_global_error("aerosim_momentum_exchange_noalloc: " + m);
    return code;
  };
  if (nx < 1 || ny < 1 || nz < 1) return err(AEROSIM_ERR_ARG, "lattice dimensions must be >= 1");
  const long long N = (long long)nx * ny * nz;
  if (N >= (1LL << 31)) return err(AEROSIM_ERR_ARG, "lattice too large (cell indices are 32-bit)");
  if (boundary_count < 0) return err(AEROSIM_ERR_ARG, "negative boundary_count");
  const long long blocks = (boundary_count + 255) / 256;
  if (blocks > kNoAllocMaxBlocks)
    return err(AEROSIM_ERR_ARG, "boundary_count " + std::to_string(boundary_count) + " exceeds the maximum of " +
                                    std::to_string((long long)kNoAllocMaxBlocks * 256) + " boundary cells");
  if (!out || (boundary_count > 0 && (!f || !flags || !boundary_cells || !q)))
    return err(AEROSIM_ERR_ARG, "null device pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return err(AEROSIM_ERR_CUDA, cudaGetErrorString(e));
  if (device < 0 || device >= kMaxDevices) return err(AEROSIM_ERR_ARG, "device ordinal beyond the supported range");
  if (boundary_count == 0) {
    e = cudaMemsetAsync(out, 0, 8 * sizeof(double), s);
    return e == cudaSuccess ? AEROSIM_OK : err(AEROSIM_ERR_CUDA, cudaGetErrorString(e));
  }
  void* scratch = nullptr;
  e = scratch_address(device, &scratch);
  if (e != cudaSuccess) return err(AEROSIM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  unsigned int* ticket = reinterpret_cast<unsigned int*>(static_cast<unsigned char*>(scratch) + kPartialBytes);
  e = cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return err(AEROSIM_ERR_CUDA, cudaGetErrorString(e));

  ForceArgs a{};
  a.f = f;
  a.cls = flags;  // reference flags 0 / 1 / 2: the class byte's flag bits
  a.bcells = boundary_cells;
  a.q = q;
  a.st = nullptr;
  a.partials = static_cast<double*>(scratch);
  a.ticket = ticket;
  a.out = out;
  // the caller's dense layout f[d * N + idx]: a row pitch of nx, planes of N cells
  a.L = make_reference_layout(nx, ny, nz);
  a.B = boundary_count;
  a.prev_slot = -1;  // no pending rescale: the caller's populations are final
  forces_kernel<StoreF32, MODE_MIRROR><<<(unsigned)blocks, 256, 0, s>>>(a);
  e = cudaGetLastError();
  return e == cudaSuccess ? AEROSIM_OK : err(AEROSIM_ERR_CUDA, cudaGetErrorString(e));
}
