// Set-up kernels of the 3D hybrid path: the 2D sensitivity, the weight
// normalisation and the translation of responses to frame events.  This file
// is compiled with -fmad=false: every binary32 operation of the frame
// translation rounds where the reference's C++ says, so the pixel-info and
// plane ranges of each event equal the reference's bit for bit.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "hybrid_internal.h"

namespace hybridmlem {

namespace {

// calculate_sensitivity (src/3d/hybrid/reconstruction.h:226-237): the sum of
// the weights of every pixel info of each pixel.  Summed in binary64 (the
// reference sums sequentially in binary32; the two agree to the binary32
// rounding of the reference's own sum).
__global__ void k_sens_acc(int32_t nc, const short2* __restrict__ pix,
                           const float* __restrict__ w, int64_t n, double* acc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const short2 p = pix[i];
    atomicAdd(acc + p.x + (int64_t)nc * p.y, (double)w[i]);
  }
}

__global__ void k_sens_round(const double* __restrict__ acc, float* sens, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    sens[i] = (float)acc[i];
}

// normalize_geometry_weights (reconstruction.h:239-261), one plane half.
__global__ void k_normalize(int32_t nc, const short2* __restrict__ pix, float* w,
                            const float* __restrict__ sens, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const short2 p = pix[i];
    w[i] = w[i] / sens[p.x + (int64_t)nc * p.y];
  }
}

// std::lower_bound / std::upper_bound over a sorted binary32 range.
__device__ int64_t lower_bound_f(const float* a, int64_t lo, int64_t hi, float v) {
  int64_t n = hi - lo;
  while (n > 0) {
    const int64_t half = n >> 1;
    if (a[lo + half] < v) {
      lo += half + 1;
      n -= half + 1;
    } else {
      n = half;
    }
  }
  return lo;
}

__device__ int64_t upper_bound_f(const float* a, int64_t lo, int64_t hi, float v) {
  int64_t n = hi - lo;
  while (n > 0) {
    const int64_t half = n >> 1;
    if (!(v < a[lo + half])) {
      lo += half + 1;
      n -= half + 1;
    } else {
      n = half;
    }
  }
  return lo;
}

// Reconstruction::plane (reconstruction.h:149): truncation to short.
__device__ __forceinline__ int16_t plane_of(const GridF& g, float z) {
  return (int16_t)(int)((z - g.z_left) / g.p);
}

// translate_to_frame + bb_intersects_grid_with_positive_weight
// (reconstruction.h:97-161), one response per thread.
__global__ void k_frames(const GridF g, const GeometryDev geo,
                         const int16_t* __restrict__ first, const int16_t* __restrict__ second,
                         const float* __restrict__ z_up, const float* __restrict__ z_dn,
                         const float* __restrict__ dl, int64_t n, Frame* frames,
                         int32_t* keep) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    keep[i] = 0;
    const int64_t a = first[i], b = second[i];
    // LOR::index on the pair as the reference reads it (lor.h:33-35)
    const int64_t li = a * (a + 1) / 2 + b;
    if (a < 0 || b < 0 || li >= geo.n_lors) continue;
    const float R = geo.lor_len[li] / 2;
    // Strip::Response::calculate_tan_y_z (src/2d/strip/response.h:22-37)
    const float zu = z_up[i], zd = z_dn[i], d = dl[i];
    const float tan = (zu - zd) / (2 * R);
    const float up = -0.5f * (d / sqrtf(1 + tan * tan));
    const float right = 0.5f * (zu + zd + (2 * up * tan));
    // GaussianKernel::ellipse_bb (src/2d/strip/gaussian_kernel.h:108-128)
    const float tan_sq = tan * tan;
    const float sec = sqrtf(1 + tan * tan);
    const float A = 4 * sec * sec * g.ipdl + 2 * tan_sq * g.ipz;
    const float B = -4 * tan * g.ipz;
    const float C = 2 * g.ipz;
    const float B_2 = (B / 2) * (B / 2);
    const float half_up = 3 / sqrtf(A - (B_2 / C));
    const float half_right = 3 / sqrtf(C - (B_2 / A));
    const int16_t pl = plane_of(g, right - half_right);
    const int16_t pr = plane_of(g, right + half_right);
    const int16_t pb = pl > 0 ? pl : (int16_t)0;
    const int16_t pe1 = (int16_t)(pr + 1);
    const int16_t pe = pe1 < (int16_t)g.np ? pe1 : (int16_t)g.np;
    const float y_up = up + half_up, y_dn = up - half_up;
    const float t_up = (y_up + R) / (2 * R);
    const float t_dn = (y_dn + R) / (2 * R);
    const int64_t lb = geo.lbeg[li], le = geo.lend[li];
    // upper_bound(t_up) + 1 and lower_bound(t_dn) (reconstruction.h:130-145);
    // the end may reach one info past the LOR's range, as in the reference,
    // and is clamped at the end of the arrays
    int64_t ie = upper_bound_f(geo.pos, lb, le, t_up) + 1;
    const int64_t ib = lower_bound_f(geo.pos, lb, le, t_dn);
    if (ie > geo.n_infos) ie = geo.n_infos;
    if (pe <= 0 || pb >= g.np) continue;
    bool ok = false;
    for (int64_t k = ib; k < ie && !ok; ++k) {
      const short2 p = geo.pix[k];
      ok = p.x >= 0 && p.x < g.nc && p.y >= 0 && p.y < g.nr && geo.w[k] > 0;
    }
    if (!ok) continue;
    Frame f;
    f.lor = (int32_t)li;
    f.info_begin = (int32_t)ib;
    f.info_end = (int32_t)ie;
    f.plane_begin = pb;
    f.plane_end = pe;
    f.up = up;
    f.right = right;
    f.tan = tan;
    f.sec = sec;
    frames[i] = f;
    keep[i] = 1;
  }
}

__global__ void k_compact(const Frame* __restrict__ frames, const int32_t* __restrict__ keep,
                          const int64_t* __restrict__ offs, int64_t n, Frame* out,
                          int64_t* out_index) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!keep[i]) continue;
    out[offs[i]] = frames[i];
    out_index[offs[i]] = i;
  }
}

int grid_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (int)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

}  // namespace

void launch_sensitivity(const GridF& g, const short2* pix, const float* w, int64_t n,
                        double* acc, float* sens, cudaStream_t st) {
  cudaMemsetAsync(acc, 0, sizeof(double) * g.n_pixels, st);
  k_sens_acc<<<grid_for(n), 256, 0, st>>>(g.nc, pix, w, n, acc);
  k_sens_round<<<grid_for(g.n_pixels), 256, 0, st>>>(acc, sens, g.n_pixels);
}

void launch_normalize(const GridF& g, const short2* pix, float* w, const float* sens,
                      int64_t n, cudaStream_t st) {
  k_normalize<<<grid_for(n), 256, 0, st>>>(g.nc, pix, w, sens, n);
}

void launch_frames(const GridF& g, const GeometryDev& geo, const int16_t* first,
                   const int16_t* second, const float* z_up, const float* z_dn,
                   const float* dl, int64_t n, Frame* frames, int32_t* keep,
                   cudaStream_t st) {
  k_frames<<<grid_for(n), 256, 0, st>>>(g, geo, first, second, z_up, z_dn, dl, n, frames,
                                        keep);
}

void launch_compact(const Frame* frames, const int32_t* keep, const int64_t* offs, int64_t n,
                    Frame* out, int64_t* out_index, cudaStream_t st) {
  k_compact<<<grid_for(n), 256, 0, st>>>(frames, keep, offs, n, out, out_index);
}

namespace {
__global__ void k_lor_keys(const Frame* __restrict__ frames, int32_t n, int32_t* keys,
                           int32_t* index) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = frames[i].lor;
    index[i] = i;
  }
}
__global__ void k_gather_frames(const Frame* __restrict__ frames, const int32_t* index,
                                int32_t n, Frame* out) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = frames[index[i]];
}
}  // namespace

cudaError_t order_frames_by_lor(const Frame* frames, int32_t n, int64_t n_lors, Frame* out,
                                cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  int end_bit = 1;
  while (end_bit < 31 && ((int64_t)1 << end_bit) < n_lors) ++end_bit;
  int32_t *keys = nullptr, *index = nullptr;
  void* temp = nullptr;
  size_t temp_bytes = 0;
  cudaError_t e = cudaMalloc(&keys, 4 * (size_t)n * sizeof(int32_t));
  if (e != cudaSuccess) return e;
  index = keys + n;
  int32_t* keys_out = keys + 2 * (size_t)n;
  int32_t* index_out = keys + 3 * (size_t)n;
  k_lor_keys<<<grid_for(n), 256, 0, st>>>(frames, n, keys, index);
  e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys_out, index, index_out, n,
                                      0, end_bit, st);
  if (e == cudaSuccess) e = cudaMalloc(&temp, temp_bytes);
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_out, index, index_out, n,
                                        0, end_bit, st);
  if (e == cudaSuccess) {
    k_gather_frames<<<grid_for(n), 256, 0, st>>>(frames, index_out, n, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(temp);
  cudaFree(keys);
  return e;
}

}  // namespace hybridmlem

// Exclusive scan of the keep flags (CUB), used by hybrid_capi.cu.
extern "C" cudaError_t hybridmlem_scan_keep(const int32_t* keep, int64_t* offs, int64_t n,
                                            void* temp, size_t* temp_bytes, cudaStream_t st) {
  return cub::DeviceScan::ExclusiveSum(temp, *temp_bytes, keep, offs, n, st);
}
