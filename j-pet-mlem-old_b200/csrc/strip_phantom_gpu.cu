// Device generator of seeded synthetic list-mode events
// (strip_generate_events_device, strip_generate_events_image_device in
// include/stripmlem.h): one thread per event, the per-event arithmetic of
// strip_generator.h (compiled with -fmad=false, as the host's
// -ffp-contract=off), written straight into device buffers.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "stripmlem.h"
#include "strip_generator.h"

namespace {

template <class Emit>
__global__ void k_generate(stripgen::Params p, Emit emit, int64_t n,
                           float* z_u, float* z_d, float* dl, int* bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (stripgen::event(p, (uint64_t)i, emit, z_u[i], z_d[i], dl[i]) !=
        stripgen::kDetected)
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

// Emission histogram on the reference tool's pixel grid (pixel_grid.h:59-69:
// column = floor((z - lower_left_z) / s), row = floor((y - lower_left_y) / s),
// row 0 at the bottom).
struct GridHist {
  uint32_t* img = nullptr;
  int nz = 0, ny = 0;
  double llz = 0, lly = 0, s = 1;
  unsigned long long* count = nullptr;  // per-thread emission counter
  __device__ __forceinline__ void operator()(double pz, double py) const {
    if (count) ++*count;
    if (!img) return;
    const double cz = floor((pz - llz) / s), cy = floor((py - lly) / s);
    if (cz >= 0 && cz < nz && cy >= 0 && cy < ny)
      atomicAdd(reinterpret_cast<unsigned*>(img) + (int64_t)cy * nz + (int64_t)cz, 1u);
  }
};

// One thread per emission index: kDetected events go to (z_u, z_d, dl)[i]
// and set flag[i]; every emission is counted in `emitted`, detected ones in
// `detected`.
template <class Emit>
__global__ void k_simulate(stripgen::Params p, Emit emit, int64_t n,
                           int one_emission, GridHist emitted, GridHist detected,
                           float* z_u, float* z_d, float* dl, int* flag,
                           int* bad, unsigned long long* n_emitted) {
  unsigned long long mine = 0;
  emitted.count = &mine;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double origin[2];
    const int st = stripgen::event(p, (uint64_t)i, emit, z_u[i], z_d[i], dl[i],
                                   one_emission != 0, origin, emitted);
    if (st == stripgen::kDetected) detected(origin[0], origin[1]);
    if (st == stripgen::kFailed) atomicOr(bad, 1);
    if (flag) flag[i] = st == stripgen::kDetected;
  }
  if (mine) atomicAdd(n_emitted, mine);
}

__global__ void k_compact(const int* flag, const int* pos, int64_t n,
                          const float* zu, const float* zd, const float* dl,
                          float* ozu, float* ozd, float* odl) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (flag[i]) {
      const int p = pos[i];
      ozu[p] = zu[i];
      ozd[p] = zd[i];
      odl[p] = dl[i];
    }
}

}  // namespace

extern "C" int strip_simulate_device(const strip_geometry* g,
                                     const strip_region* regions, int n_regions,
                                     const strip_simulation* opt, uint64_t seed,
                                     int64_t n, float* d_z_u, float* d_z_d,
                                     float* d_dl, int64_t* n_written,
                                     int64_t* n_emitted) {
  if (!g || !regions || n_regions <= 0 || !opt || n < 0 || n > INT32_MAX ||
      !(g->radius > 0) || !(g->scintillator_length > 0) || !(g->sigma_z >= 0) ||
      !(g->sigma_dl >= 0))
    return STRIP_E_INVALID;
  if (n_written) *n_written = 0;
  if (n_emitted) *n_emitted = 0;
  if (n == 0) return STRIP_OK;
  if (!device_ptrs(d_z_u, d_z_d, d_dl)) return STRIP_E_INVALID;
  std::vector<stripgen::Region> reg;
  std::vector<double> cdf;
  if (!stripgen::make_regions(regions, n_regions, reg, cdf)) return STRIP_E_INVALID;
  Buffers buf;
  const stripgen::Region* d_reg = buf.copy(reg.data(), reg.size());
  const double* d_cdf = buf.copy(cdf.data(), cdf.size());
  const int zero = 0;
  const unsigned long long zero64 = 0;
  int* bad = buf.copy(&zero, 1);
  unsigned long long* d_count = buf.copy(&zero64, 1);
  if (!d_reg || !d_cdf || !bad || !d_count) return STRIP_E_CUDA;
  GridHist he, hd;
  for (GridHist* h : {&he, &hd}) {
    h->nz = g->n_z_pixels;
    h->ny = g->n_y_pixels;
    h->s = opt->pixel_size;
    h->llz = -opt->pixel_size * g->n_z_pixels / 2.0 + opt->origin_z;
    h->lly = -opt->pixel_size * g->n_y_pixels / 2.0 + opt->origin_y;
  }
  he.img = opt->d_emitted;
  hd.img = opt->d_detected;
  if ((he.img || hd.img) && !(opt->pixel_size > 0)) return STRIP_E_INVALID;
  const bool compact = opt->count_emitted != 0;
  float *tzu = d_z_u, *tzd = d_z_d, *tdl = d_dl;
  int *flag = nullptr, *pos = nullptr;
  if (compact) {
    auto alloc = [&](size_t bytes) -> void* {
      void* q = nullptr;
      if (cudaMalloc(&q, bytes) != cudaSuccess) return nullptr;
      buf.p.push_back(q);
      return q;
    };
    tzu = (float*)alloc(n * sizeof(float));
    tzd = (float*)alloc(n * sizeof(float));
    tdl = (float*)alloc(n * sizeof(float));
    flag = (int*)alloc((n + 1) * sizeof(int));
    pos = (int*)alloc((n + 1) * sizeof(int));
    if (!tzu || !tzd || !tdl || !flag || !pos) return STRIP_E_NOMEM;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 16);
  k_simulate<<<grid, 256>>>(stripgen::make_params(g, seed, opt->uniform_angle != 0),
                            stripgen::RegionEmitter{d_reg, d_cdf, n_regions,
                                                    opt->additive != 0},
                            n, compact ? 1 : 0, he, hd, tzu, tzd, tdl, flag, bad,
                            d_count);
  if (cudaGetLastError() != cudaSuccess) return STRIP_E_CUDA;
  int h_bad = 0;
  unsigned long long h_count = 0;
  if (cudaMemcpy(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&h_count, d_count, sizeof(h_count), cudaMemcpyDeviceToHost) != cudaSuccess)
    return STRIP_E_CUDA;
  if (h_bad) return STRIP_E_INVALID;
  if (n_emitted) *n_emitted = (int64_t)h_count;
  if (!compact) {
    if (n_written) *n_written = n;
    return STRIP_OK;
  }
  // positions of the detected emissions: exclusive sum of the flags
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag, pos, (int)n + 1);
  void* tmp = nullptr;
  if (cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 1)) != cudaSuccess) return STRIP_E_NOMEM;
  buf.p.push_back(tmp);
  if (cudaMemset(flag + n, 0, sizeof(int)) != cudaSuccess ||
      cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flag, pos, (int)n + 1) != cudaSuccess)
    return STRIP_E_CUDA;
  k_compact<<<grid, 256>>>(flag, pos, n, tzu, tzd, tdl, d_z_u, d_z_d, d_dl);
  int total = 0;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpy(&total, pos + n, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return STRIP_E_CUDA;
  if (n_written) *n_written = total;
  return STRIP_OK;
}

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
                stripgen::RegionEmitter{d_reg, d_cdf, n_el, 0}, n, d_z_u, d_z_d,
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

extern "C" int strip_simulate(const strip_geometry* g, const strip_region* regions,
                              int n_regions, const strip_simulation* options,
                              uint64_t seed, int64_t n, int device, float* z_u,
                              float* z_d, float* dl, uint32_t* emitted,
                              uint32_t* detected, int64_t* n_written,
                              int64_t* n_emitted) {
  if (!g || !options || n < 0 || (n > 0 && (!z_u || !z_d || !dl)))
    return STRIP_E_INVALID;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev <= 0) {
    cudaGetLastError();
    return STRIP_E_NODEVICE;
  }
  if (device < 0 || device >= n_dev || cudaSetDevice(device) != cudaSuccess)
    return STRIP_E_INVALID;
  const size_t n_pix = (size_t)std::max(g->n_y_pixels, 0) * (size_t)std::max(g->n_z_pixels, 0);
  const size_t ne = (size_t)std::max<int64_t>(n, 1);
  Buffers buf;
  auto alloc = [&](size_t bytes) -> void* {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(bytes, 1)) != cudaSuccess) return nullptr;
    buf.p.push_back(q);
    return q;
  };
  float* d_zu = (float*)alloc(ne * sizeof(float));
  float* d_zd = (float*)alloc(ne * sizeof(float));
  float* d_dl = (float*)alloc(ne * sizeof(float));
  if (!d_zu || !d_zd || !d_dl) return STRIP_E_NOMEM;
  strip_simulation opt = *options;
  opt.d_emitted = opt.d_detected = nullptr;
  if (emitted || detected) {
    opt.d_emitted = (uint32_t*)alloc(n_pix * sizeof(uint32_t));
    opt.d_detected = (uint32_t*)alloc(n_pix * sizeof(uint32_t));
    if (!opt.d_emitted || !opt.d_detected) return STRIP_E_NOMEM;
    if (cudaMemset(opt.d_emitted, 0, n_pix * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(opt.d_detected, 0, n_pix * sizeof(uint32_t)) != cudaSuccess)
      return STRIP_E_CUDA;
  }
  int64_t written = 0;
  const int rc = strip_simulate_device(g, regions, n_regions, &opt, seed, n, d_zu,
                                       d_zd, d_dl, &written, n_emitted);
  if (rc != STRIP_OK) return rc;
  const size_t wb = (size_t)written * sizeof(float);
  if (written > 0 &&
      (cudaMemcpy(z_u, d_zu, wb, cudaMemcpyDeviceToHost) != cudaSuccess ||
       cudaMemcpy(z_d, d_zd, wb, cudaMemcpyDeviceToHost) != cudaSuccess ||
       cudaMemcpy(dl, d_dl, wb, cudaMemcpyDeviceToHost) != cudaSuccess))
    return STRIP_E_CUDA;
  if (emitted && cudaMemcpy(emitted, opt.d_emitted, n_pix * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost) != cudaSuccess)
    return STRIP_E_CUDA;
  if (detected && cudaMemcpy(detected, opt.d_detected, n_pix * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost) != cudaSuccess)
    return STRIP_E_CUDA;
  if (n_written) *n_written = written;
  return STRIP_OK;
}
