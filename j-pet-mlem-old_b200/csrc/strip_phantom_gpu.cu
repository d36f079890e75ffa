// Device generator of seeded synthetic list-mode events
// (strip_generate_events_device, strip_generate_events_image_device in
// include/stripmlem.h): one thread per event, the per-event arithmetic of
// strip_generator.h (compiled with -fmad=false, as the host's
// -ffp-contract=off), written straight into device buffers.
#include <cuda_runtime.h>

#include <vector>

#include "stripmlem.h"
#include "strip_generator.h"

namespace {

template <class Emit>
__global__ void k_generate(stripgen::Params p, Emit emit, int64_t n,
                           float* z_u, float* z_d, float* dl, int* bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (!stripgen::event(p, (uint64_t)i, emit, z_u[i], z_d[i], dl[i]))
      atomicOr(bad, 1);
}

// Device scratch freed on every path.
struct Buffers {
  std::vector<void*> p;
  ~Buffers() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  T* copy(const T* host, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) return nullptr;
    p.push_back(q);
    if (cudaMemcpy(q, host, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
      return nullptr;
    return static_cast<T*>(q);
  }
};

template <class Emit>
int launch(const stripgen::Params& p, const Emit& emit, int64_t n, float* z_u,
           float* z_d, float* dl, Buffers& buf) {
  const int zero = 0;
  int* bad = buf.copy(&zero, 1);
  if (!bad) return STRIP_E_CUDA;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t blocks = (n + 255) / 256;
  const int grid = (int)(blocks < (int64_t)sms * 16 ? blocks : (int64_t)sms * 16);
  k_generate<<<grid, 256>>>(p, emit, n, z_u, z_d, dl, bad);
  int h_bad = 0;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpy(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return STRIP_E_CUDA;
  return h_bad ? STRIP_E_INVALID : STRIP_OK;
}

bool device_ptrs(const float* a, const float* b, const float* c) {
  for (const float* q : {a, b, c}) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, q) != cudaSuccess ||
        at.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      return false;
    }
  }
  return true;
}

}  // namespace

extern "C" int strip_generate_events_device(const strip_geometry* g,
                                            const strip_ellipse* el, int n_el,
                                            uint64_t seed, int64_t n,
                                            float* d_z_u, float* d_z_d,
                                            float* d_dl) {
  if (!g || !el || n_el <= 0 || n < 0 || !(g->radius > 0) ||
      !(g->scintillator_length > 0) || !(g->sigma_z >= 0) || !(g->sigma_dl >= 0))
    return STRIP_E_INVALID;
  if (n == 0) return STRIP_OK;
  if (!device_ptrs(d_z_u, d_z_d, d_dl)) return STRIP_E_INVALID;
  std::vector<stripgen::Region> reg;
  std::vector<double> cdf;
  if (!stripgen::make_regions(el, n_el, reg, cdf)) return STRIP_E_INVALID;
  Buffers buf;
  const stripgen::Region* d_reg = buf.copy(reg.data(), reg.size());
  const double* d_cdf = buf.copy(cdf.data(), cdf.size());
  if (!d_reg || !d_cdf) return STRIP_E_CUDA;
  return launch(stripgen::make_params(g, seed, 0),
                stripgen::EllipseEmitter{d_reg, d_cdf, n_el}, n, d_z_u, d_z_d,
                d_dl, buf);
}

extern "C" int strip_generate_events_image_device(const strip_geometry* g,
                                                  const float* rho,
                                                  uint64_t seed, int64_t n,
                                                  int uniform_angle,
                                                  float* d_z_u, float* d_z_d,
                                                  float* d_dl) {
  if (!stripgen::valid_image_geometry(g) || !rho || n < 0) return STRIP_E_INVALID;
  if (n == 0) return STRIP_OK;
  if (!device_ptrs(d_z_u, d_z_d, d_dl)) return STRIP_E_INVALID;
  std::vector<double> cdf;
  if (!stripgen::make_image_cdf(g, rho, cdf)) return STRIP_E_INVALID;
  Buffers buf;
  const double* d_cdf = buf.copy(cdf.data(), cdf.size());
  const float* d_rho = buf.copy(rho, cdf.size());
  if (!d_cdf || !d_rho) return STRIP_E_CUDA;
  return launch(stripgen::make_params(g, seed, uniform_angle != 0),
                stripgen::image_emitter(g, d_cdf, d_rho), n, d_z_u, d_z_d, d_dl,
                buf);
}
