// The 3D hybrid MLEM iteration on sm_100a.
//
// One warp per frame event.  The event's voxels are its LOR pixel infos
// [info_begin, info_end) times its planes [plane_begin, plane_end); the warp
// walks them flattened with the plane fastest.  The volume is held on the
// device with the plane index fastest (z-fast: voxel (x, y, z) at
// (x + n_c y) n_p + z), so a warp's image reads and accumulator atomics fall
// on a few contiguous sectors; the boundary layout (x fastest) is restored
// by launch_from_zfast.
//
// Per voxel (GaussianKernel::normalized, src/2d/strip/gaussian_kernel.h:
// 51-105, in the frame of the event's LOR):
//   K = c / sqrt(a' S a) exp(-b' S b / 2) / sens(z, up),
//   sens = (atan u - atan v) / pi,  weight = K w rho,  D += weight s.
// Everything that depends on the pixel only (c / sqrt(a' S a) w, (up_p - up)
// tan, the b_r term, 1 / (R -+ up_p), the pixel's sensitivity and its base
// index) is computed once per pixel into the warp's shared memory; per voxel
// remain z, the two ratios of the sensitivity (from z exactly as the
// reference forms them, so the decisions sens <= 0 at z = +-L/2 are the
// reference's), one exp2, the arctangent difference atan u - atan v =
// atan2(u - v, 1 + u v) by atan2_pos below, and an image load.  (A table of
// 1 / sens per pixel info and plane -- it depends on the LOR, the pixel and
// the plane only -- was slower: 414 against 252 ms per iteration on the
// big-barrel workload, the walk waiting on its HBM loads; with the events in
// LOR order, so that the rows in use stay in L2, still 279 against 204 ms.)
// Pass 1 keeps each
// voxel's weight in a per-warp shared cache (first kCache voxels) and the
// next kSpill in a per-warp slab of global memory (written and read back by
// the same warp within microseconds, so it stays in L2); pass 2
// scatters weight / D with one red.global.add.f32 per voxel, reading the
// cache or recomputing past it.
#include "hybrid_internal.h"

namespace hybridmlem {

namespace {

// Launch shape and per-warp cache (compile-time tuning constants).
#ifndef HYBRID_WARPS
#define HYBRID_WARPS 8
#endif
#ifndef HYBRID_CACHE
#define HYBRID_CACHE 2048
#endif
#ifndef HYBRID_BLOCKS_PER_SM
#define HYBRID_BLOCKS_PER_SM 3
#endif
#ifndef HYBRID_SPILL
#define HYBRID_SPILL 16384
#endif
#ifndef HYBRID_UNROLL
#define HYBRID_UNROLL 1
#endif
#ifndef HYBRID_UNROLL2
#define HYBRID_UNROLL2 1
#endif
constexpr int kWarps = HYBRID_WARPS;
constexpr int kThreads = kWarps * 32;
constexpr int kCache = HYBRID_CACHE;          // cached voxel weights per warp
constexpr int kSpill = HYBRID_SPILL;          // further weights per warp in global memory
constexpr int kBlocksPerSm = HYBRID_BLOCKS_PER_SM;
constexpr int kUnroll = HYBRID_UNROLL;           // pass-1 voxel-loop unroll
constexpr int kUnroll2 = HYBRID_UNROLL2;         // pass-2 voxel-loop unroll

// atan2(a, b) for a > 0, in (0, pi): the quotient of the smaller by the
// larger of a and |b| (fast division) folded into [0, 1], an odd polynomial
// t P(t^2) of degree 15 for atan on [0, 1], then the quadrant.  The
// coefficients come from tests/golden/fit_atan.py: Lawson's iteratively
// reweighted least squares toward the minimax absolute error (3.75e-8 in
// exact arithmetic, 1.2e-7 evaluated in binary32), rounded to binary32.
// The reference's atanf(u) - atanf(v) carries about the same binary32
// rounding.
__device__ __forceinline__ float atan2_pos(float a, float b) {
  const float ab = fabsf(b);
  const float mx = fmaxf(a, ab), mn = fminf(a, ab);
  const float t = __fdividef(mn, mx);
  const float s = t * t;
  float p = -0.0040545654483139515f;
  p = fmaf(p, s, 0.021862952038645744f);
  p = fmaf(p, s, -0.0559123195707798f);
  p = fmaf(p, s, 0.0964219719171524f);
  p = fmaf(p, s, -0.1390862911939621f);
  p = fmaf(p, s, 0.19946566224098206f);
  p = fmaf(p, s, -0.33329859375953674f);
  p = fmaf(p, s, 0.9999993443489075f);
  float r = t * p;
  if (a > ab) r = 1.5707963267948966f - r;
  if (b < 0.0f) r = 3.14159265358979f - r;
  return r;
}

// z of plane iz (VoxelGrid::center_z_at, voxel_grid.h:38-40).
__device__ __forceinline__ float plane_z(const GridF& g, int iz) {
  return ((float)iz + 0.5f) * g.p + g.z_left;
}

// pi / (pi sens) of a voxel at z for a pixel at up_p in a LOR of half length
// R (GaussianKernel::sensitivity, gaussian_kernel.h:139-148, with the two
// quotients as products by 1 / (R -+ up_p)); 0 where sens <= 0.  The signs
// of the two ratios, hence the decision sens <= 0, are the reference's.
__device__ __forceinline__ float inv_sens(float half_L, float z, float ra, float rb) {
  const float lmz = half_L - z, lpz = half_L + z;
  const float u = fminf(lmz * ra, lpz * rb);
  const float v = fmaxf(-lpz * ra, -lmz * rb);
  const float a = u - v;
  if (!(a > 0.0f)) return 0.0f;
  return __fdividef(3.14159265358979f, atan2_pos(a, fmaf(u, v, 1.0f)));
}

__device__ __forceinline__ float proj_up(const GridF& g, short2 p, float4 md) {
  const float cx = g.llc_x + (float)p.x * g.p;
  const float cy = g.llc_y + (float)p.y * g.p;
  return (cx - md.x) * md.z + (cy - md.y) * md.w;
}

// Event-dependent pixel terms of one chunk of 32 pixel infos.
struct PixelData {
  float4 t[32];    // c / sqrt(a' S a) w, (up_p - up) tan, b_r S_dl b_r, s
  float2 r[32];    // 1 / (R - up_p), 1 / (R + up_p)
  int base[32];    // z-fast index of plane 0
};

struct WarpSmem {
  PixelData px;
  float cache[kCache];
};

__device__ __forceinline__ void load_pixels(const GridF& g, const GeometryDev& geo,
                                            const float* __restrict__ sens, const Frame& f,
                                            float4 md, float R, int c0, int n_pix, int lane,
                                            PixelData& px) {
  const int k = c0 + lane;
  if (k < n_pix) {
    const int64_t info = (int64_t)f.info_begin + k;
    const short2 p = geo.pix[info];
    const float w = geo.w[info];
    const float upp = proj_up(g, p, md);
    const float dy = upp - f.up;
    const float yp = dy + f.up;
    const float sec_sq = f.sec * f.sec;
    const float ap = -(yp - R) * sec_sq;
    const float aq = -(yp + R) * sec_sq;
    const float ar = -2.0f * yp * f.sec * f.tan;
    const float aca = ap * g.ipz * ap + aq * g.ipz * aq + ar * g.ipdl * ar;
    const float br = -2.0f * dy * f.sec;
    const int pidx = p.x + g.nc * p.y;
    px.t[lane] = make_float4(g.norm_c * rsqrtf(aca) * w, dy * f.tan, br * g.ipdl * br,
                             sens[pidx]);
    px.r[lane] = make_float2(__frcp_rn(R - upp), __frcp_rn(R + upp));
    px.base[lane] = pidx * g.np;
  }
  __syncwarp();
}

// K w (without rho) of voxel (pixel j of the chunk, plane iz).
__device__ __forceinline__ float voxel_kw(const GridF& g, const Frame& f, const PixelData& px,
                                          int j, int iz, float half_L) {
  const float4 t4 = px.t[j];
  const float z = plane_z(g, iz);
  const float2 r = px.r[j];
  const float is = inv_sens(half_L, z, r.x, r.y);
  if (is == 0.0f) return 0.0f;
  const float bpq = (z - f.right) - t4.y;
  const float t = bpq * g.ipz * bpq;
  const float bcb = (t + t) + t4.z;
  return t4.x * exp2f(-0.7213475204444817f * bcb) * is;  // exp(-bcb / 2)
}

__global__ void __launch_bounds__(kThreads, kBlocksPerSm)
k_mlem(const GridF g, const GeometryDev geo, const float* __restrict__ sens,
       const Frame* __restrict__ frames, int64_t n_frames,
       const float* __restrict__ rho_t, float* acc_t, float* spill) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  WarpSmem& sm = reinterpret_cast<WarpSmem*>(smem_raw)[wib];
  float* slab = spill + ((int64_t)blockIdx.x * kWarps + wib) * kSpill;
  const float half_L = g.L / 2;
  // grid-stride over the events (in LOR order: the warps resident at one
  // time work on a few LORs, whose pixel infos and image lines stay in L2)
  const int64_t n_warps = (int64_t)gridDim.x * kWarps;
  for (int64_t e = (int64_t)blockIdx.x * kWarps + wib; e < n_frames; e += n_warps) {
    const Frame f = frames[e];
    const int n_pix = f.info_end - f.info_begin;
    const int n_pl = f.plane_end - f.plane_begin;
    if (n_pix <= 0 || n_pl <= 0) continue;
    const float4 md = geo.lor_md[f.lor];
    const float R = geo.lor_len[f.lor] / 2;
    const int q = 32 / n_pl, r = 32 - q * n_pl;
    const int j0 = lane / n_pl, pz0 = lane - j0 * n_pl;
    // pass 1: weights and the denominator
    float d = 0.0f;
    for (int c0 = 0; c0 < n_pix; c0 += 32) {
      load_pixels(g, geo, sens, f, md, R, c0, n_pix, lane, sm.px);
      const int nv = min(32, n_pix - c0) * n_pl;
      const int base = c0 * n_pl;
      int j = j0, pz = pz0;
#pragma unroll kUnroll
      for (int v = lane; v < nv; v += 32) {
        const int iz = f.plane_begin + pz;
        // the image load goes out first; the kernel arithmetic hides it
        const float rho = __ldg(rho_t + sm.px.base[j] + iz);
        float wgt = voxel_kw(g, f, sm.px, j, iz, half_L);
        if (wgt != 0.0f) {
          wgt *= rho;
          d = fmaf(wgt, sm.px.t[j].w, d);
        }
        const int fv = base + v;
        if (fv < kCache)
          sm.cache[fv] = wgt;
        else if (fv < kCache + kSpill)
          slab[fv - kCache] = wgt;
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
      const int nv = min(32, n_pix - c0) * n_pl;
      if (base + nv <= kCache + kSpill) {
        if (c0 + lane < n_pix) {
          const short2 p = geo.pix[(int64_t)f.info_begin + c0 + lane];
          sm.px.base[lane] = (p.x + g.nc * p.y) * g.np;
        }
        __syncwarp();
      } else {
        load_pixels(g, geo, sens, f, md, R, c0, n_pix, lane, sm.px);
      }
      int j = j0, pz = pz0;
#pragma unroll kUnroll2
      for (int v = lane; v < nv; v += 32) {
        const int iz = f.plane_begin + pz;
        const int vi = sm.px.base[j] + iz;
        const int fv = base + v;
        float wgt;
        if (fv < kCache) {
          wgt = sm.cache[fv];
        } else if (fv < kCache + kSpill) {
          wgt = slab[fv - kCache];
        } else {
          const float rho = __ldg(rho_t + vi);
          wgt = voxel_kw(g, f, sm.px, j, iz, half_L) * rho;
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

size_t mlem_spill_floats(int n_blocks) { return (size_t)n_blocks * kWarps * kSpill; }

void launch_mlem(const GridF& g, const GeometryDev& geo, const float* sens, const Frame* frames,
                 int64_t n_frames, const float* rho_t, float* acc_t, float* spill, int n_blocks,
                 cudaStream_t st) {
  const int smem = (int)sizeof(WarpSmem) * kWarps;
  cudaFuncSetAttribute(k_mlem, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  k_mlem<<<n_blocks, kThreads, smem, st>>>(g, geo, sens, frames, n_frames, rho_t, acc_t, spill);
}

void launch_event_counts(const Frame* frames, int64_t n, unsigned long long* out2,
                         cudaStream_t st) {
  cudaMemsetAsync(out2, 0, 2 * sizeof(unsigned long long), st);
  k_event_counts<<<grid_for(n), 256, 0, st>>>(frames, n, out2);
}

namespace {
// The kernel's arctangent (which = 0) or CUDA's atan2f (which = 1) on n
// argument pairs: the test hook that bounds atan2_pos's error.
__global__ void k_atan2_probe(const float* a, const float* b, int64_t n, int which,
                              float* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = which == 0 ? atan2_pos(a[i], b[i]) : atan2f(a[i], b[i]);
}
}  // namespace

cudaError_t launch_atan2_probe(const float* a, const float* b, int64_t n, int which,
                               float* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_atan2_probe<<<grid_for(n), 256, 0, st>>>(a, b, n, which, out);
  return cudaGetLastError();
}

}  // namespace hybridmlem
