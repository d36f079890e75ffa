// Internal types and launchers of the 3D hybrid path (include/hybridmlem.h).
// Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hybridmlem {

// The voxel grid and scanner constants in binary32 / int16 as the reference
// holds them: PixelGrid (src/2d/geometry/pixel_grid.h:22-37), VoxelGrid
// (src/3d/geometry/voxel_grid.h:19-24), GaussianKernel<float> members
// (src/2d/strip/gaussian_kernel.h:27-33).
struct GridF {
  int32_t nc, nr, np;
  float p;        // pixel size = plane thickness
  float z_left;
  float llc_x;    // lower_left_center
  float llc_y;
  float L;        // barrel length
  float ipz;      // 1 / sigma_z^2
  float ipdl;     // 1 / sigma_dl^2
  float norm_c;   // 1 / (2 pi^2) sqrt(ipz^2 ipdl)
  int32_t n_pixels;
};

// One kept frame event (FrameEvent, src/3d/hybrid/reconstruction.h:53-63),
// 32 bytes: the LOR, its pixel-info range, its plane range and the strip
// frame's (up, right, tan, sec).
struct __align__(16) Frame {
  int32_t lor;
  int32_t info_begin;
  int32_t info_end;
  int16_t plane_begin;
  int16_t plane_end;
  float up;
  float right;
  float tan;
  float sec;
};
static_assert(sizeof(Frame) == 32, "Frame is 32 bytes");

// Device view of the flattened geometry (GeometrySOA, geometry_soa.h:270-284).
struct GeometryDev {
  const float4* lor_md;     // per LOR: mid x, mid y, direction x, direction y
  const float* lor_len;     // per LOR: segment length
  const short2* pix;        // per info: pixel (x, y)
  const float* pos;         // per info: position along the LOR
  const float* w;           // per info: weight (normalised after the sensitivity)
  const int64_t* lbeg;      // per LOR
  const int64_t* lend;
  int64_t n_lors;
  int64_t n_infos;
};

// hybrid_setup.cu (compiled without FMA contraction: the frame arithmetic
// rounds as the reference's binary32 C++).
void launch_sensitivity(const GridF& g, const short2* pix, const float* w, int64_t n,
                        double* acc, float* sens, cudaStream_t st);
void launch_normalize(const GridF& g, const short2* pix, float* w, const float* sens,
                      int64_t n, cudaStream_t st);
void launch_frames(const GridF& g, const GeometryDev& geo, const int16_t* first,
                   const int16_t* second, const float* z_up, const float* z_dn,
                   const float* dl, int64_t n, Frame* frames, int32_t* keep,
                   cudaStream_t st);
void launch_compact(const Frame* frames, const int32_t* keep, const int64_t* offs, int64_t n,
                    Frame* out, int64_t* out_index, cudaStream_t st);
// The frame events in LOR order (stable: response order within a LOR), for
// the iteration kernel; synchronises the stream.
cudaError_t order_frames_by_lor(const Frame* frames, int32_t n, int64_t n_lors, Frame* out,
                                cudaStream_t st);

// hybrid_kernels.cu
void launch_to_zfast(const GridF& g, const float* rho, float* rho_t, cudaStream_t st);
void launch_from_zfast(const GridF& g, const float* rho_t, float* rho, cudaStream_t st);
// spill: mlem_spill_floats(n_blocks) floats of scratch for the per-warp
// weight slabs.
void launch_mlem(const GridF& g, const GeometryDev& geo, const float* sens, const Frame* frames,
                 int64_t n_frames, const float* rho_t, float* acc_t, float* spill, int n_blocks,
                 cudaStream_t st);
size_t mlem_spill_floats(int n_blocks);
int mlem_blocks_per_sm();
void launch_event_counts(const Frame* frames, int64_t n, unsigned long long* out2,
                         cudaStream_t st);
cudaError_t launch_atan2_probe(const float* a, const float* b, int64_t n, int which,
                               float* out, cudaStream_t st);

}  // namespace hybridmlem
