/*
 * TEST INFRASTRUCTURE ONLY -- the oracle for the 3D hybrid list-mode TOF MLEM
 * path.  A CPU restatement of the reference (JPETTomography/j-pet-mlem-old,
 * src/3d/hybrid/reconstruction.h and the 2D barrel / strip headers it uses)
 * in C++.  Only tests/, bench.py's reference arm and __graft_entry__.smoke()
 * may load it, and only as the checker; the product never links or calls it.
 *
 * Two arithmetic flavours of the iteration:
 *   hyb_mlem_f32  binary32 in the reference's operation order (compiled with
 *                 -ffp-contract=off): reproduces the reference binary's
 *                 images bit for bit at one thread (pinned against
 *                 oracle/_ref/3d_hybrid_reconstruction_nocontract);
 *   hyb_mlem_f64  the same algorithm in binary64 from the same binary32
 *                 inputs: the "FP64 oracle" device images are held to.
 *
 * Layouts (as the reference's GeometrySOA, src/2d/barrel/geometry_soa.h):
 *   seg      per LOR 9 floats: start x y, end x y, mid x y, direction x y,
 *            length (LineSegment, src/2d/geometry/line_segment.h:18-27)
 *   pix      per pixel info 2 int16 (x = column, y = row)
 *   pos/w    per pixel info position along the LOR (0 at start) and weight
 *   lbeg/lend per LOR the [begin, end) pixel-info range
 *   volume   x fastest, then y, then plane (VoxelGrid::index,
 *            src/3d/geometry/voxel_grid.h:56-61)
 */
#ifndef HYBRID_ORACLE_H
#define HYBRID_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The voxel grid and scanner constants, narrowed to float as the reference
 * narrows its options (reconstruction_cmd.cpp:415-447). */
typedef struct hyb_setup {
  int32_t n_columns;
  int32_t n_rows;
  int32_t n_planes;
  float pixel_size;
  float z_left;
  float length;
  float sigma_z;
  float sigma_dl;
} hyb_setup;

typedef struct hyb_frame {
  int32_t lor_index;
  int16_t plane_begin;
  int16_t plane_end;
  int64_t info_begin;
  int64_t info_end;
  float up;
  float right;
  float tan;
  float sec;
} hyb_frame;

typedef struct hyb_stats {
  int64_t used_events;
  int64_t used_pixels;
  int64_t used_voxels;
} hyb_stats;

/* GeometrySOA(matrix, detector centers, grid, inactive)
 * (geometry_soa.h:72-180): sorts the matrix elements by LOR then pixel,
 * writes per LOR its segment between the detector centers and its pixel
 * infos sorted by position along the LOR (std::sort, as the reference).
 * Returns the number of pixel infos, or -1 on invalid input. */
int64_t hyb_soa_from_matrix(const hyb_setup* s, int32_t n_detectors,
                            const float* centers_xy, int64_t n_elements,
                            const uint16_t* lor_a, const uint16_t* lor_b,
                            const uint16_t* px, const uint16_t* py,
                            const uint32_t* hits, uint32_t n_emissions,
                            const int16_t* inactive, int32_t n_inactive,
                            float* seg, int16_t* pix, float* pos, float* w,
                            int64_t* lbeg, int64_t* lend);

/* Reconstruction::calculate_sensitivity (reconstruction.h:226-237) and
 * normalize_geometry_weights (reconstruction.h:239-261), one plane half. */
void hyb_sensitivity(const hyb_setup* s, int64_t n_infos, const int16_t* pix,
                     const float* w, float* sens);
void hyb_normalize(int64_t n_infos, const hyb_setup* s, const int16_t* pix,
                   float* w, const float* sens);

/* translate_to_frame + bb_intersects_grid_with_positive_weight
 * (reconstruction.h:97-161) for each response; kept frames are written in
 * input order.  keep[i] = 1 when response i is kept.  Returns the count. */
int64_t hyb_frame_events(const hyb_setup* s, int64_t n_lors, const float* seg,
                         const int16_t* pix, const float* pos, const float* w,
                         const int64_t* lbeg, const int64_t* lend,
                         int64_t n_infos, int64_t n_events,
                         const int16_t* first, const int16_t* second,
                         const float* z_up, const float* z_dn,
                         const float* dl, hyb_frame* frames, uint8_t* keep);

/* n_iter iterations of Reconstruction::operator() (reconstruction.h:263-386)
 * with the 2D sensitivity; rho (n_columns * n_rows * n_planes) in/out. */
void hyb_mlem_f32(const hyb_setup* s, const float* seg, const int16_t* pix,
                  const float* w, const float* sens, const hyb_frame* frames,
                  int64_t n_frames, float* rho, int32_t n_iter,
                  hyb_stats* stats);
void hyb_mlem_f64(const hyb_setup* s, const float* seg, const int16_t* pix,
                  const float* w, const float* sens, const hyb_frame* frames,
                  int64_t n_frames, double* rho, int32_t n_iter,
                  hyb_stats* stats);

/* The normalized strip kernel times nothing else (GaussianKernel::normalized,
 * src/2d/strip/gaussian_kernel.h:93-105 with sensitivity :139-148), for unit
 * tests of the voxel arithmetic. */
float hyb_kernel_f32(const hyb_setup* s, float right, float up, float tan,
                     float sec, float R, float z, float up_pixel);

#ifdef __cplusplus
}
#endif

#endif
