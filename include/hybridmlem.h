/*
 * hybridmlem.h -- C ABI of the B200 (sm_100a) 3D hybrid list-mode TOF MLEM.
 *
 * Drop-in boundary for the 3D hybrid reconstruction of
 * JPETTomography/j-pet-mlem-old (2D barrel LOR geometry x strip TOF kernel
 * along z).  The reference has no FFI; its operator API is
 *   (1) the C++ template PET3D::Hybrid::Reconstruction<Scanner, Kernel2D>
 *       built from a GeometrySOA, with calculate_sensitivity /
 *       set_sensitivity_to_one / normalize_geometry_weights, operator<< for
 *       responses and operator()() for one iteration
 *                                  (src/3d/hybrid/reconstruction.h:31-386)
 *   (2) the GPU entry point PET3D::Hybrid::GPU::Reconstruction::run(geometry,
 *       sensitivity, events, n_events, sigma_z, sigma_dl, grid, length,
 *       n_blocks, n_iterations_in_block, rho, start_iteration, output_cb,
 *       progress_cb, device, cuda_blocks, cuda_threads, device_name_cb)
 *                                  (src/3d/hybrid/cuda/reconstruction.cu:31-190)
 *   (3) the 3d_hybrid_reconstruction CLI with --system, --detector-file,
 *       --sens-to-one, --sensitivity, --inactive
 *                                  (src/3d/hybrid/reconstruction_cmd.cpp:147-680)
 * Each entry point below names the piece it replaces.
 *
 * Conventions as stripmlem.h: every function returns STRIP_OK (0) or a
 * negative STRIP_E* code, never throws or aborts; the caller owns every host
 * buffer; one context per host thread; device work is ordered on the
 * context's own stream and every call returns after it is done.
 *
 * Volume layout at the boundary: binary32, x (column) fastest, then y (row),
 * then plane -- VoxelGrid::index (src/3d/geometry/voxel_grid.h:56-61).
 * Units are the caller's (the reference CLI works in metres).
 */
#ifndef HYBRIDMLEM_H
#define HYBRIDMLEM_H

#include <stddef.h>
#include <stdint.h>

#include "stripmlem.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The voxel grid and scanner constants.  Replaces PixelGrid(n, n, s_pixel),
 * VoxelGrid(grid2d, z_left, n_planes), Scanner(barrel, length) and
 * set_sigmas (reconstruction_cmd.cpp:415-447); narrowed to binary32 / int16
 * as the reference narrows them.  The grid is centred on the origin. */
typedef struct hybrid_setup {
  int32_t n_columns;   /* pixels along x                                    */
  int32_t n_rows;      /* pixels along y                                    */
  int32_t n_planes;    /* voxel planes along z                              */
  int32_t reserved;
  double pixel_size;   /* pixel edge and plane thickness                    */
  double z_left;       /* z of the first plane's lower edge                 */
  double length;       /* barrel length L (the strip frame's sensitivity)   */
  double sigma_z;      /* TOF sigma along z                                 */
  double sigma_dl;     /* TOF sigma of delta-l                              */
} hybrid_setup;

typedef struct hybrid_ctx hybrid_ctx;

typedef struct hybrid_stats {
  int64_t n_responses;    /* responses passed to hybrid_set_responses        */
  int64_t n_events;       /* kept frame events (the reference's n_events())  */
  int64_t n_lors;         /* (n_detectors + 1) * n_detectors / 2             */
  int64_t n_pixel_infos;  /* flattened LOR pixel infos                       */
  int64_t used_pixels;    /* pixel infos walked by the last iteration        */
  int64_t used_voxels;    /* voxels walked by the last iteration             */
  int32_t iterations;     /* iterations run so far                           */
  int32_t reserved;
  double last_iteration_ms; /* device time of the last iteration            */
} hybrid_stats;

/* Sensitivity source (run_reconstruction, reconstruction_cmd.cpp:503-522). */
enum hybrid_sensitivity_mode {
  HYBRID_SENS_CALCULATE = 0, /* calculate_sensitivity: sum of LOR weights   */
  HYBRID_SENS_ONE = 1,       /* --sens-to-one                               */
  HYBRID_SENS_EXTERNAL = 2,  /* --sensitivity: caller's 2D map              */
  HYBRID_SENS_GIVEN = 3      /* caller's 2D map, weights already normalised
                                (the GPU run()'s inputs)                    */
};

typedef void (*hybrid_progress_cb)(int32_t iteration, int32_t finished, void* user);

/* Creates a context on `device`; the image starts at 1 everywhere
 * (Reconstruction's rho(..., 1), reconstruction.h:70-75). */
int hybrid_ctx_create(const hybrid_setup* setup, int32_t device, hybrid_ctx** out);
int hybrid_ctx_destroy(hybrid_ctx* ctx);
const char* hybrid_last_error(const hybrid_ctx* ctx);

/* Builds the flattened LOR geometry from a full 2D barrel system matrix and
 * the detector centres.  Replaces GeometrySOA(sparse_matrix, c_detectors,
 * grid, inactive, n_inactive) (src/2d/barrel/geometry_soa.h:72-180):
 * elements sorted by LOR then pixel, weight = hits / n_emissions, elements
 * of inactive detectors dropped, per LOR the segment from the centre of
 * detector `second` to that of `first` and its pixel infos sorted by
 * position along it (std::sort, as the reference).  Element i is the pixel
 * (px[i], py[i]) of LOR (lor_a[i], lor_b[i]) (either order) with hits[i].
 * centers_xy holds 2 floats per detector: PolygonalDetector::center() of
 * the detector's vertices (src/2d/geometry/polygon.h:57-68).  The grid must
 * be square (n_columns == n_rows == the matrix's pixels in a row). */
int hybrid_set_geometry_from_matrix(hybrid_ctx* ctx, int32_t n_detectors,
                                    const float* centers_xy, int64_t n_elements,
                                    const uint16_t* lor_a, const uint16_t* lor_b,
                                    const uint16_t* px, const uint16_t* py,
                                    const uint32_t* hits, uint32_t n_emissions,
                                    const int16_t* inactive, int32_t n_inactive);

/* Takes a flattened geometry as the reference's GPU entry point receives it
 * (GeometrySOA, src/2d/barrel/geometry_soa.h:270-284): per LOR index
 * first * (first + 1) / 2 + second its segment (start x, y, end x, y; the
 * mid point, direction and length are derived as LineSegment's constructor
 * does, line_segment.h:18-27) and [lor_begin, lor_end) into the pixel-info
 * arrays; per pixel info its pixel (x, y), position along the LOR and
 * weight.  Use HYBRID_SENS_GIVEN when the weights are normalised already. */
int hybrid_set_geometry_soa(hybrid_ctx* ctx, int32_t n_detectors, const float* segments,
                            int64_t n_infos, const int16_t* pixels, const float* positions,
                            const float* weights, const uint64_t* lor_begin,
                            const uint64_t* lor_end);

/* Copies the flattened geometry back (sizes from hybrid_get_stats):
 * seg 9 floats per LOR (start xy, end xy, mid xy, direction xy, length),
 * pix 2 int16 per info, pos / weight per info (weights as normalised by
 * hybrid_set_sensitivity once it ran), lbeg / lend per LOR.  Any pointer
 * may be null. */
int hybrid_get_geometry(hybrid_ctx* ctx, float* seg, int16_t* pix, float* pos,
                        float* weight, int64_t* lbeg, int64_t* lend);

/* Sensitivity and weight normalisation: calculate_sensitivity /
 * set_sensitivity_to_one / an external 2D map, then
 * normalize_geometry_weights (reconstruction.h:226-261).  `external`
 * (n_columns * n_rows) is read for HYBRID_SENS_EXTERNAL only.  Runs on the
 * device; must follow the geometry and precede the responses. */
int hybrid_set_sensitivity(hybrid_ctx* ctx, int32_t mode, const float* external);
int hybrid_get_sensitivity(hybrid_ctx* ctx, float* sens /* n_columns*n_rows */);

/* Loads responses (LOR pair, z_up, z_dn, dl) and translates them to frame
 * events on the device: translate_to_frame then
 * bb_intersects_grid_with_positive_weight (reconstruction.h:97-161,
 * fast_load_txt_events / operator<< :163-212).  The pair is used as stored
 * (index first * (first + 1) / 2 + second, as the reference reads it);
 * responses whose index falls outside the LOR table are dropped.  Replaces
 * the previous responses. */
int hybrid_set_responses(hybrid_ctx* ctx, const int16_t* first, const int16_t* second,
                         const float* z_up, const float* z_dn, const float* dl,
                         int64_t n);

/* Takes frame events as the reference's GPU entry point receives them
 * (Reconstruction::FrameEvent, reconstruction.h:53-63: the LOR's index,
 * [pixel_info_begin, pixel_info_end), [plane_begin, plane_end), up, right,
 * tan, sec), already translated and filtered by the caller.  Replaces the
 * previous responses or frames. */
int hybrid_set_frames(hybrid_ctx* ctx, int64_t n, const int32_t* lor, const int64_t* info_begin,
                      const int64_t* info_end, const int16_t* plane_begin,
                      const int16_t* plane_end, const float* up, const float* right,
                      const float* tan, const float* sec);

/* Frame events of kept responses in input order, for parity checks:
 * per event its LOR index, [info_begin, info_end), [plane_begin,
 * plane_end) and the kept responses' input indices.  Any pointer may be
 * null; sizes n_events from hybrid_get_stats. */
int hybrid_get_frames(hybrid_ctx* ctx, int32_t* lor_index, int64_t* info_begin,
                      int64_t* info_end, int16_t* plane_begin, int16_t* plane_end,
                      int64_t* response_index);

/* n_iterations of Reconstruction::operator()() (reconstruction.h:263-386) /
 * the GPU run loop (cuda/reconstruction.cu:121-182):
 *   rho'_v = sum_e K_ev w_v rho_v / D_e,  D_e = sum_v K_ev w_v rho_v s_v
 * with K the strip GaussianKernel::normalized in the LOR's frame, w the
 * normalised LOR pixel weight, s the 2D sensitivity; events with D_e <= 0
 * contribute nothing.  progress may be null. */
int hybrid_iterate(hybrid_ctx* ctx, int32_t n_iterations, hybrid_progress_cb progress,
                   void* user);

/* One iteration split for event-sharded runs (one process per GPU, each
 * holding a shard of the responses and the whole image): hybrid_accumulate
 * back-projects this context's events into the accumulator (zeroed first;
 * the caller's device buffer of n_voxels floats when hybrid_set_accumulator
 * gave one, else the context's own), the caller sums the accumulators over
 * the ranks (e.g. an NCCL all-reduce), and hybrid_update makes the summed
 * accumulator the image -- the reference's sum of its per-thread images
 * (reconstruction.h:369-376) taken across processes.  The accumulator is in
 * the library's internal voxel order (the same on every rank); null
 * restores the context's own. */
int hybrid_set_accumulator(hybrid_ctx* ctx, float* device_acc);
int hybrid_accumulate(hybrid_ctx* ctx);
int hybrid_update(hybrid_ctx* ctx);

/* The current image (n_columns * n_rows * n_planes), VoxelGrid order. */
int hybrid_set_image(hybrid_ctx* ctx, const float* rho);
int hybrid_get_image(hybrid_ctx* ctx, float* rho);

int hybrid_get_stats(hybrid_ctx* ctx, hybrid_stats* out);

/* Text responses "first second z_up z_dn dl", one per '\n'-terminated line
 * (an unterminated last line is not read), parsed with the arithmetic of the
 * reference's fast text parser (util::text_parser, text_parser.h:82-175, as
 * Reconstruction::fast_load_txt_events uses it, reconstruction.h:163-186) so
 * the binary32 values are the reference's; the detector indices keep their
 * low 16 bits as the reference's short fields do.  `text` holds `length`
 * bytes; up to `capacity` lines are stored and *n_lines receives the number
 * of complete lines (call with capacity 0 to count them).  On a malformed
 * number returns STRIP_E_INVALID with *n_lines = the line's index.  Host
 * only. */
int hybrid_parse_responses_text(const char* text, int64_t length, int64_t capacity,
                                int16_t* first, int16_t* second, float* z_up, float* z_dn,
                                float* dl, int64_t* n_lines);

/* Adds the converter's Gaussian errors to n converted responses in place:
 * for each response in order, z_up += N(0, sigma_z), z_dn += N(0, sigma_z),
 * dl += N(0, sigma_dl), drawn from std::normal_distribution<double> (one
 * for z, one for dl) over one std::mt19937_64(seed) -- 3d_tool_convert
 * --warsaw's smearing (src/3d/tool/convert_cmd.cpp:92-95,149-151), value for
 * value with the same C++ standard library.  Host only. */
int hybrid_smear_responses(int64_t seed, double sigma_z, double sigma_dl, int64_t n,
                           double* z_up, double* z_dn, double* dl);

/* Test hook: evaluates, on CUDA device `device`, the arctangent the MLEM
 * kernel uses for the strip frame's angular sensitivity (which = 0: atan2(a, b)
 * for a > 0 by an odd degree-15 polynomial) or CUDA's atan2f (which = 1) on
 * n host argument pairs; out receives n values.  The reference calls
 * std::atan (gaussian_kernel.h:139-148); this bounds the replacement. */
int hybrid_debug_atan2(int32_t device, const float* a, const float* b, int64_t n,
                       int32_t which, float* out);

/* A z-cylinder of a synthetic phantom: centre, radius, half length along z,
 * activity. */
typedef struct hybrid_cylinder {
  double x, y, z;
  double radius;
  double half_length;
  double activity;
} hybrid_cylinder;

/* Seeded synthetic responses, a stand-in for 3d_hybrid_phantom
 * (src/3d/hybrid/phantom_cmd.cpp) on a ring barrel: emissions uniform in the
 * cylinders (chosen by volume x activity, overlaps exclusive with the first
 * cylinder on top), isotropic directions, each photon taken by the first
 * detector its 2D line crosses (rings inwards out) at the projection of the
 * detector's centre, kept when both points lie within |z| <= length / 2;
 * first = the larger detector index, dl = l_up - l_dn of the 3D path
 * lengths, z_up, z_dn, dl smeared with N(0, sigma_z), N(0, sigma_dl)
 * (Scanner::response_w_error, src/3d/hybrid/scanner.h:215-225).  `polygons`
 * holds 4 vertices (x, y) per detector, rings of equal centre radius in
 * index order, equally spaced in angle, radii increasing.  Response i
 * depends only on (seed, i).  device < 0 generates on the host (OpenMP),
 * otherwise on that device; the outputs are host arrays of n. */
int hybrid_generate_responses(int32_t n_detectors, const float* polygons,
                              const hybrid_cylinder* phantom, int32_t n_cylinders,
                              double length, double sigma_z, double sigma_dl,
                              uint64_t seed, int64_t n, int32_t device,
                              int16_t* first, int16_t* second, float* z_up,
                              float* z_dn, float* dl);

#ifdef __cplusplus
}
#endif

#endif
