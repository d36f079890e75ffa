// The 3D hybrid MLEM iteration on sm_100a.
//
// One warp per frame event.  The event's voxels are its LOR pixel infos
// [info_begin, info_end) times its planes [plane_begin, plane_end); the warp
// walks them flattened with the plane fastest, so that 32 lanes cover a few
// pixels x consecutive planes.  The volume is held on the device with the
// plane index fastest (z-fast: voxel (x, y, z) at (x + n_c y) n_p + z), so a
// warp's image reads and its accumulator atomics fall on a few contiguous
// sectors instead of 32 scattered ones; the boundary layout (x fastest) is
// restored by launch_from_zfast.
//
// Per voxel (GaussianKernel::normalized, src/2d/strip/gaussian_kernel.h:
// 51-105, in the frame of the event's LOR):
//   K = c / sqrt(a' S a) exp(-b' S b / 2) / sens(z, up),
//   sens = (atan u - atan v) / pi,  weight = K w rho,  D += weight s.
// Everything that depends on the pixel only (a' S a, the b_r term, 1/(R -+ up),
// the LOR weight and the pixel's sensitivity) is computed once per pixel into
// the warp's shared memory; per voxel remain one exp, one atan2 (the
// difference of the two arctangents: atan u - atan v = atan2(u - v, 1 + u v),
// whose sign is that of u - v, as the reference's) and a division.  Pass 1
// keeps each voxel's weight in a per-warp shared cache (first kCache voxels);
// pass 2 scatters weight / D with one red.global.add.f32 per voxel, reading
// the cache or recomputing past it.
#include "hybrid_internal.h"

namespace hybridmlem {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kCache = 2048;        // cached voxel weights per warp
constexpr int kBlocksPerSm = 3;     // 3 x (8 warps x 8.9 KB) of shared memory

struct PixelData {
  float bw[32];   // c / sqrt(a' S a) * w
  float dy[32];   // up_pixel - up
  float brr[32];  // b_r S_dl b_r
  float ra[32];   // 1 / (R - up_pixel)
  float rb[32];   // 1 / (R + up_pixel)
  float s[32];    // sensitivity of the pixel
  int vbase[32];  // z-fast index of the pixel's plane 0
};

struct WarpSmem {
  PixelData px;
  float cache[kCache];
};

// Per-pixel terms of the chunk [c0, c0 + 32) of the event's pixel infos.
__device__ __forceinline__ void load_pixels(const GridF& g, const GeometryDev& geo,
                                            const float* __restrict__ sens, const Frame& f,
                                            float4 md, float R, int c0, int n_pix, int lane,
                                            PixelData& px) {
  const int k = c0 + lane;
  if (k < n_pix) {
    const int64_t info = (int64_t)f.info_begin + k;
    const short2 p = geo.pix[info];
    const float w = geo.w[info];
    // PixelGrid::center_at and projection_relative_middle
    const float cx = g.llc_x + (float)p.x * g.p;
    const float cy = g.llc_y + (float)p.y * g.p;
    const float upp = (cx - md.x) * md.z + (cy - md.y) * md.w;
    const float dy = upp - f.up;
    const float yp = dy + f.up;
    const float sec_sq = f.sec * f.sec;
    const float ap = -(yp - R) * sec_sq;
    const float aq = -(yp + R) * sec_sq;
    const float ar = -2.0f * yp * f.sec * f.tan;
    const float aca = ap * g.ipz * ap + aq * g.ipz * aq + ar * g.ipdl * ar;
    const float br = -2.0f * dy * f.sec;
    const int pidx = p.x + g.nc * p.y;
    px.bw[lane] = g.norm_c / sqrtf(aca) * w;
    px.dy[lane] = dy;
    px.brr[lane] = br * g.ipdl * br;
    px.ra[lane] = 1.0f / (R - upp);
    px.rb[lane] = 1.0f / (R + upp);
    px.s[lane] = sens[pidx];
    px.vbase[lane] = pidx * g.np;
  }
  __syncwarp();
}

// K w (without rho) of voxel (pixel j of the chunk, plane iz); 0 where the
// normalised kernel is not positive.
__device__ __forceinline__ float voxel_kw(const GridF& g, const Frame& f, const PixelData& px,
                                          int j, int iz, float half_L) {
  const float z = ((float)iz + 0.5f) * g.p + g.z_left;
  const float dx = z - f.right;
  const float bpq = dx - px.dy[j] * f.tan;
  const float t = bpq * g.ipz * bpq;
  const float bcb = (t + t) + px.brr[j];
  const float e = __expf(-0.5f * bcb);
  const float ra = px.ra[j], rb = px.rb[j];
  const float u = fminf((half_L - z) * ra, (half_L + z) * rb);
  const float v = fmaxf(-(half_L + z) * ra, (z - half_L) * rb);
  const float th = atan2f(u - v, fmaf(u, v, 1.0f));
  if (!(th > 0.0f)) return 0.0f;
  return px.bw[j] * e * (3.14159265358979f / th);
}

__global__ void __launch_bounds__(kThreads, kBlocksPerSm)
k_mlem(const GridF g, const GeometryDev geo, const float* __restrict__ sens,
       const Frame* __restrict__ frames, int64_t n_frames, const float* __restrict__ rho_t,
       float* acc_t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  WarpSmem& sm = reinterpret_cast<WarpSmem*>(smem_raw)[wib];
  const int64_t n_warps = (int64_t)gridDim.x * kWarps;
  const float half_L = g.L / 2;
  for (int64_t e = (int64_t)blockIdx.x * kWarps + wib; e < n_frames; e += n_warps) {
    const Frame f = frames[e];
    const int n_pix = f.info_end - f.info_begin;
    const int n_pl = f.plane_end - f.plane_begin;
    if (n_pix <= 0 || n_pl <= 0) continue;
    const float4 md = geo.lor_md[f.lor];
    const float R = geo.lor_len[f.lor] / 2;
    const int q = 32 / n_pl, r = 32 - q * n_pl;
    // pass 1: weights and the denominator
    float d = 0.0f;
    for (int c0 = 0; c0 < n_pix; c0 += 32) {
      load_pixels(g, geo, sens, f, md, R, c0, n_pix, lane, sm.px);
      const int cn = min(32, n_pix - c0);
      const int nv = cn * n_pl;
      const int base = c0 * n_pl;
      int j = lane / n_pl, pz = lane - (lane / n_pl) * n_pl;
      for (int v = lane; v < nv; v += 32) {
        const int iz = f.plane_begin + pz;
        float wgt = voxel_kw(g, f, sm.px, j, iz, half_L);
        if (wgt != 0.0f) {
          wgt *= __ldg(rho_t + sm.px.vbase[j] + iz);
          d += wgt * sm.px.s[j];
        }
        if (base + v < kCache) sm.cache[base + v] = wgt;
        j += q;
        pz += r;
        if (pz >= n_pl) {
          pz -= n_pl;
          ++j;
        }
      }
      __syncwarp();
    }
    double dd = d;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dd += __shfl_xor_sync(0xffffffffu, dd, o);
    if (!(dd > 0.0)) continue;
    const float inv = (float)(1.0 / dd);
    // pass 2: scatter weight / D
    for (int c0 = 0; c0 < n_pix; c0 += 32) {
      const int base = c0 * n_pl;
      const int cn = min(32, n_pix - c0);
      const int nv = cn * n_pl;
      const bool cached = base + nv <= kCache;
      if (cached) {
        if (lane < cn) {
          const short2 p = geo.pix[(int64_t)f.info_begin + c0 + lane];
          sm.px.vbase[lane] = (p.x + g.nc * p.y) * g.np;
        }
        __syncwarp();
      } else {
        load_pixels(g, geo, sens, f, md, R, c0, n_pix, lane, sm.px);
      }
      int j = lane / n_pl, pz = lane - (lane / n_pl) * n_pl;
      for (int v = lane; v < nv; v += 32) {
        const int iz = f.plane_begin + pz;
        const int vi = sm.px.vbase[j] + iz;
        float wgt;
        if (base + v < kCache) {
          wgt = sm.cache[base + v];
        } else {
          wgt = voxel_kw(g, f, sm.px, j, iz, half_L);
          if (wgt != 0.0f) wgt *= __ldg(rho_t + vi);
        }
        if (wgt != 0.0f) atomicAdd(acc_t + vi, wgt * inv);
        j += q;
        pz += r;
        if (pz >= n_pl) {
          pz -= n_pl;
          ++j;
        }
      }
      __syncwarp();
    }
  }
}

// Boundary layout (x fastest, plane slowest) <-> z-fast layout.
__global__ void k_to_zfast(const GridF g, const float* __restrict__ rho, float* rho_t) {
  const int64_t n = (int64_t)g.n_pixels * g.np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pidx = i % g.n_pixels, z = i / g.n_pixels;
    rho_t[pidx * g.np + z] = rho[i];
  }
}

__global__ void k_from_zfast(const GridF g, const float* __restrict__ rho_t, float* rho) {
  const int64_t n = (int64_t)g.n_pixels * g.np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pidx = i % g.n_pixels, z = i / g.n_pixels;
    rho[i] = rho_t[pidx * g.np + z];
  }
}

__global__ void k_event_counts(const Frame* __restrict__ frames, int64_t n,
                               unsigned long long* out2) {
  unsigned long long a = 0, b = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const Frame f = frames[i];
    const int np = f.info_end - f.info_begin, nz = f.plane_end - f.plane_begin;
    a += np > 0 ? np : 0;
    b += (np > 0 && nz > 0) ? (unsigned long long)np * nz : 0ull;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out2, a);
    atomicAdd(out2 + 1, b);
  }
}

int grid_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (int)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

}  // namespace

int mlem_blocks_per_sm() { return kBlocksPerSm; }

void launch_to_zfast(const GridF& g, const float* rho, float* rho_t, cudaStream_t st) {
  k_to_zfast<<<grid_for((int64_t)g.n_pixels * g.np), 256, 0, st>>>(g, rho, rho_t);
}

void launch_from_zfast(const GridF& g, const float* rho_t, float* rho, cudaStream_t st) {
  k_from_zfast<<<grid_for((int64_t)g.n_pixels * g.np), 256, 0, st>>>(g, rho_t, rho);
}

void launch_mlem(const GridF& g, const GeometryDev& geo, const float* sens,
                 const Frame* frames, int64_t n_frames, const float* rho_t, float* acc_t,
                 int n_blocks, cudaStream_t st) {
  const int smem = (int)sizeof(WarpSmem) * kWarps;
  cudaFuncSetAttribute(k_mlem, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  k_mlem<<<n_blocks, kThreads, smem, st>>>(g, geo, sens, frames, n_frames, rho_t, acc_t);
}

void launch_event_counts(const Frame* frames, int64_t n, unsigned long long* out2,
                         cudaStream_t st) {
  cudaMemsetAsync(out2, 0, 2 * sizeof(unsigned long long), st);
  k_event_counts<<<grid_for(n), 256, 0, st>>>(frames, n, out2);
}

}  // namespace hybridmlem
