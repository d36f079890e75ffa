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
// with cudaGetSymbolAddress once per device, with that device current, on the
// first call made on that device (so the first call on a device must come
// before any stream capture), and passed to the kernels.
//
// Every call shares the scratch and leaves the last call's contents in it;
// each call clears the accumulator before use.  Calls that overlap on the GPU
// (on different streams, or from different host threads) race on the scratch.
#include <cuda_runtime.h>

#include <mutex>

#include "stripmlem.h"
#include "strip_internal.h"

namespace {

constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_acc[STRIP_NOALLOC_MAX_PIXELS];
__device__ __align__(256) float g_noalloc_sens[STRIP_NOALLOC_MAX_PIXELS];

std::mutex g_setup_mutex;
double* g_acc_ptr[kMaxDevices] = {};
float* g_sens_ptr[kMaxDevices] = {};

// Device addresses of the scratch arrays on the current device.
int noalloc_scratch(int device, double** acc, float** sens) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_acc_ptr[device]) {
    double* a = nullptr;
    float* s = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&a), g_noalloc_acc) !=
            cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&s), g_noalloc_sens) !=
            cudaSuccess) {
      cudaGetLastError();
      return STRIP_E_CUDA;
    }
    g_acc_ptr[device] = a;
    g_sens_ptr[device] = s;
  }
  *acc = g_acc_ptr[device];
  *sens = g_sens_ptr[device];
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
