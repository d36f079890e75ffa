// strip_iterate_noalloc: one MLEM iteration that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc -- code that runs inside a
// host framework which owns all device memory through its own pool or caching
// allocator under a fixed budget, and latency-sensitive pipelines that must
// not hit cudaMalloc / cudaFree, which can synchronise the whole device.  They
// pass device buffers for the events and for the image in and out; the only
// other memory this entry point uses is the scratch below.
//
// Scratch: file-scope __device__ arrays of fixed size -- a binary64
// backprojection accumulator and a binary32 sensitivity image, each of
// kNoAllocMaxPixels entries (12 MiB in total).  Every GPU that loads this
// library holds them until the process exits.  In host code the array names
// are host-side stand-ins, not device addresses: the device address is taken
// with cudaGetSymbolAddress, with the device current, on the first call made
// in a CUDA context (so that first call must come before any stream capture),
// cached per device together with the context's unique id, and passed to the
// kernels.  A call in another context of the same device -- after
// cudaDeviceReset, or under a driver-API context other than the primary one --
// finds the id changed and looks the address up again instead of using an
// address of a context that may be gone.
//
// Every call shares the scratch and leaves the last call's contents in it;
// each call clears the accumulator before use.  Calls that overlap on the GPU
// (on different streams, or from different host threads) race on the scratch.
#include <cuda.h>  // CUcontext / CUresult types only; nothing links libcuda
#include <cuda_runtime.h>

#include <mutex>

#include "stripmlem.h"
#include "strip_internal.h"

namespace {

constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_acc[STRIP_NOALLOC_MAX_PIXELS];
__device__ __align__(256) float g_noalloc_sens[STRIP_NOALLOC_MAX_PIXELS];

std::mutex g_setup_mutex;

struct Scratch {
  unsigned long long ctx_id;  // unique id of the context the addresses are of
  double* acc;
  float* sens;
};
Scratch g_scratch[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (0: none, or a driver
// without cuCtxGetId).  The driver functions come through the runtime's entry
// point table, so the library does not link libcuda.
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device addresses of the scratch arrays in the current context of `device`.
int noalloc_scratch(int device, double** acc, float** sens) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  Scratch& c = g_scratch[device];
  const unsigned long long id = current_ctx_id();
  if (id == 0 || id != c.ctx_id) {
    double* a = nullptr;
    float* s = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&a), g_noalloc_acc) !=
            cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&s), g_noalloc_sens) !=
            cudaSuccess) {
      cudaGetLastError();
      c = Scratch{};
      return STRIP_E_CUDA;
    }
    // the lookup makes the runtime's context current if none was; without an
    // id (no driver support) nothing is cached and every call looks up again
    c = Scratch{current_ctx_id(), a, s};
  }
  *acc = c.acc;
  *sens = c.sens;
  return STRIP_OK;
}

}  // namespace

extern "C" int strip_iterate_noalloc(const strip_geometry* g, const float* d_z_u,
                                     const float* d_z_d, const float* d_dl,
                                     int64_t n, const float* d_rho_in,
                                     float* d_rho_out, int mode,
                                     void* stream) {
  using namespace stripmlem;
  if (!g || !d_rho_in || !d_rho_out || n < 0 ||
      (n > 0 && (!d_z_u || !d_z_d || !d_dl)) ||
      (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU))
    return STRIP_E_INVALID;
  if (g->n_y_pixels <= 0 || g->n_z_pixels <= 0 || g->n_y_pixels > 32767 ||
      g->n_z_pixels > 32767 || !(g->pixel_height > 0) ||
      !(g->pixel_width > 0) || !(g->sigma_z > 0) || !(g->sigma_dl > 0) ||
      !(g->radius > 0))
    return STRIP_E_INVALID;
  const int64_t n_pix = (int64_t)g->n_y_pixels * g->n_z_pixels;
  if (n_pix > STRIP_NOALLOC_MAX_PIXELS) return STRIP_E_INVALID;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 ||
      device >= kMaxDevices) {
    cudaGetLastError();
    return STRIP_E_NODEVICE;
  }
  double* acc = nullptr;
  float* sens = nullptr;
  if (int rc = noalloc_scratch(device, &acc, &sens)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  LaunchArgs a{};
  a.s = make_scanner(*g);
  a.k = make_kernel(g->sigma_z, g->sigma_dl, a.s.pw);
  a.zu = d_z_u;
  a.zd = d_z_d;
  a.dl = d_dl;
  a.rho = d_rho_in;
  a.sens = mode == STRIP_MODE_GPU ? sens : nullptr;
  a.acc = acc;
  a.g_begin = 0;
  a.g_count = n;
  cudaError_t e = cudaMemsetAsync(acc, 0, n_pix * sizeof(double), st);
  if (e == cudaSuccess && mode == STRIP_MODE_GPU)
    e = launch_sensitivity(a.s, 1, sens, st);
  if (e == cudaSuccess)
    e = launch_global(OP_MLEM, mode, STRIP_ACCUM_KAHAN, a, st);
  if (e == cudaSuccess) e = launch_update_out(d_rho_in, d_rho_out, acc, n_pix, mlem_weighted(mode), st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? STRIP_E_NOMEM : STRIP_E_CUDA;
  }
  return STRIP_OK;
}
