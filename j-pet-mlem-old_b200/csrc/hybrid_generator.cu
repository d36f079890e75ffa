// hybrid_generate_responses (include/hybridmlem.h): the seeded response
// generator of hybrid_generator.h on the host (OpenMP) or on a device (one
// thread per response).  Compiled with -fmad=false so both evaluate the same
// binary64 expressions without contraction.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "hybrid_generator.h"
#include "hybridmlem.h"

using hybridgen::Setup;

namespace {

__global__ void k_generate(const Setup S, const float* __restrict__ poly,
                           const float* __restrict__ cen, uint64_t seed, int64_t n,
                           int16_t* first, int16_t* second, float* z_up, float* z_dn, float* dl,
                           int* failed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!hybridgen::generate(S, poly, cen, seed, i, first[i], second[i], z_up[i], z_dn[i], dl[i]))
      atomicExch(failed, 1);
  }
}

// Detector centres (PolygonalDetector::center(), binary32 running sum / 4)
// and the ring layout: consecutive detectors whose centres share a radius,
// equally spaced in angle in index order.
int make_setup(int32_t n_det, const float* poly, const hybrid_cylinder* ph, int32_t n_cyl,
               double L, double sz, double sdl, Setup& S, std::vector<float>& cen) {
  if (n_det <= 1 || n_det > 32767 || !poly || !ph || n_cyl <= 0 ||
      n_cyl > hybridgen::kMaxCylinders || !(L > 0) || !(sz >= 0) || !(sdl >= 0))
    return STRIP_E_INVALID;
  cen.resize(2 * n_det);
  for (int d = 0; d < n_det; ++d) {
    float cx = 0, cy = 0;
    for (int q = 0; q < 4; ++q) {
      cx += poly[8 * d + 2 * q];
      cy += poly[8 * d + 2 * q + 1];
    }
    cen[2 * d] = cx / 4.0f;
    cen[2 * d + 1] = cy / 4.0f;
  }
  S = Setup{};
  int d = 0;
  while (d < n_det) {
    if (S.n_rings == hybridgen::kMaxRings) return STRIP_E_INVALID;
    const double r0 = std::hypot((double)cen[2 * d], (double)cen[2 * d + 1]);
    int e = d + 1;
    while (e < n_det &&
           std::fabs(std::hypot((double)cen[2 * e], (double)cen[2 * e + 1]) - r0) < 1e-5 * r0)
      ++e;
    hybridgen::Ring& rg = S.ring[S.n_rings++];
    rg.first = d;
    rg.count = e - d;
    rg.radius = r0;
    rg.angle0 = std::atan2((double)cen[2 * d + 1], (double)cen[2 * d]);
    for (int k = d; k < e; ++k) {
      const double want = rg.angle0 + 2.0 * stripgen::kPi * (k - d) / rg.count;
      double diff = std::atan2((double)cen[2 * k + 1], (double)cen[2 * k]) - want;
      diff = std::remainder(diff, 2.0 * stripgen::kPi);
      if (std::fabs(diff) > 1e-3) return STRIP_E_INVALID;
    }
    d = e;
  }
  for (int i = 1; i < S.n_rings; ++i)
    if (S.ring[i].radius < S.ring[i - 1].radius) return STRIP_E_INVALID;
  double total = 0;
  S.n_cyl = n_cyl;
  for (int c = 0; c < n_cyl; ++c) {
    const hybrid_cylinder& h = ph[c];
    if (!(h.radius > 0) || !(h.half_length > 0) || !(h.activity >= 0)) return STRIP_E_INVALID;
    S.cyl[c] = hybridgen::Cylinder{h.x, h.y, h.z, h.radius, h.half_length, h.activity};
    total += stripgen::kPi * h.radius * h.radius * 2 * h.half_length * h.activity;
    S.cum[c] = total;
  }
  if (!(total > 0)) return STRIP_E_INVALID;
  for (int c = 0; c < n_cyl; ++c) S.cum[c] /= total;
  S.L = L;
  S.sigma_z = sz;
  S.sigma_dl = sdl;
  return STRIP_OK;
}

}  // namespace

extern "C" int hybrid_generate_responses(int32_t n_detectors, const float* polygons,
                                         const hybrid_cylinder* phantom, int32_t n_cylinders,
                                         double length, double sigma_z, double sigma_dl,
                                         uint64_t seed, int64_t n, int32_t device,
                                         int16_t* first, int16_t* second, float* z_up,
                                         float* z_dn, float* dl) {
  if (n < 0 || (n > 0 && (!first || !second || !z_up || !z_dn || !dl))) return STRIP_E_INVALID;
  Setup S;
  std::vector<float> cen;
  const int rc = make_setup(n_detectors, polygons, phantom, n_cylinders, length, sigma_z,
                            sigma_dl, S, cen);
  if (rc != STRIP_OK) return rc;
  if (n == 0) return STRIP_OK;
  if (device < 0) {
    int failed = 0;
#pragma omp parallel for schedule(static) reduction(| : failed)
    for (int64_t i = 0; i < n; ++i)
      failed |= !hybridgen::generate(S, polygons, cen.data(), seed, i, first[i], second[i],
                                     z_up[i], z_dn[i], dl[i]);
    return failed ? STRIP_E_INVALID : STRIP_OK;
  }
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev <= 0) {
    cudaGetLastError();
    return STRIP_E_NODEVICE;
  }
  if (device >= n_dev || cudaSetDevice(device) != cudaSuccess) return STRIP_E_INVALID;
  float *d_poly = nullptr, *d_cen = nullptr, *d_zu = nullptr, *d_zd = nullptr, *d_dl = nullptr;
  int16_t *d_a = nullptr, *d_b = nullptr;
  int* d_failed = nullptr;
  int out = STRIP_OK;
  cudaStream_t st = nullptr;
  do {
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) { out = STRIP_E_CUDA; break; }
    if (cudaMalloc(&d_poly, 8 * sizeof(float) * n_detectors) != cudaSuccess ||
        cudaMalloc(&d_cen, 2 * sizeof(float) * n_detectors) != cudaSuccess ||
        cudaMalloc(&d_a, n * sizeof(int16_t)) != cudaSuccess ||
        cudaMalloc(&d_b, n * sizeof(int16_t)) != cudaSuccess ||
        cudaMalloc(&d_zu, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_zd, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_dl, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_failed, sizeof(int)) != cudaSuccess) {
      out = STRIP_E_NOMEM;
      break;
    }
    if (cudaMemcpyAsync(d_poly, polygons, 8 * sizeof(float) * n_detectors,
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_cen, cen.data(), 2 * sizeof(float) * n_detectors,
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(d_failed, 0, sizeof(int), st) != cudaSuccess) {
      out = STRIP_E_CUDA;
      break;
    }
    const int64_t blocks = (n + 255) / 256;
    k_generate<<<(int)(blocks < 148 * 64 ? blocks : 148 * 64), 256, 0, st>>>(
        S, d_poly, d_cen, seed, n, d_a, d_b, d_zu, d_zd, d_dl, d_failed);
    int failed = 0;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(first, d_a, n * sizeof(int16_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(second, d_b, n * sizeof(int16_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(z_up, d_zu, n * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(z_dn, d_zd, n * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(dl, d_dl, n * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&failed, d_failed, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      out = STRIP_E_CUDA;
      break;
    }
    if (failed) out = STRIP_E_INVALID;
  } while (0);
  cudaFree(d_poly);
  cudaFree(d_cen);
  cudaFree(d_a);
  cudaFree(d_b);
  cudaFree(d_zu);
  cudaFree(d_zd);
  cudaFree(d_dl);
  cudaFree(d_failed);
  if (st) cudaStreamDestroy(st);
  return out;
}
