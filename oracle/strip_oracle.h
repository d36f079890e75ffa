/*
 * TEST INFRASTRUCTURE ONLY -- the oracle for the 2D strip list-mode TOF MLEM
 * path.  A CPU restatement of the reference (JPETTomography/j-pet-mlem-old,
 * src/2d/strip/) in plain C.  Only tests/, bench.py's cpu_baseline / reference
 * arm and __graft_entry__.smoke() may load it, and only as the checker; the
 * product (the CUDA library) never links or calls it.
 *
 * Two arithmetic flavours:
 *   *_f32  binary32, the reference's own operation order, compiled with
 *          -ffp-contract=off: pixel sets and images are reproduced bit for bit
 *          (pinned against the reference binary built under oracle/_ref).
 *   *_f64  binary64 restatement (the reference templates instantiated with
 *          double): the "FP64 oracle" every image error is stated against.
 *
 * Kernel modes (see the *_mlem_* functions):
 *   ORC_MODE_CPU  GaussianKernel, no sensitivity      (reconstruction.h:220-298)
 *   ORC_MODE_GPU  AnalyticKernel, 5-point pixel sensitivity in the
 *                 denominator                         (warp_granularity.cuh:20-154)
 */
#ifndef STRIP_ORACLE_H
#define STRIP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_MODE_CPU = 0, ORC_MODE_GPU = 1 };

/* Scanner parameters as the CLI parses them (doubles), before the reference
 * narrows them to Scanner<float, short> (options.h:42-50, scanner.h:39-67). */
typedef struct orc_geometry {
  double radius;
  double scintillator_length;
  int32_t n_y_pixels;
  int32_t n_z_pixels;
  double pixel_height;
  double pixel_width;
  double sigma_z;
  double sigma_dl;
  double center_y;
  double center_z;
} orc_geometry;

/* --- per-event geometry --------------------------------------------------- */

/* box[0..5] = center pixel (x=z, y), clamped top-left (x, y), clamped
 * bottom-right (x, y); the scan visits y in [tl.y, br.y), z in [tl.x, br.x). */
void orc_event_box_f32(const orc_geometry* g, float z_u, float z_d, float dl,
                       int32_t box[6]);
void orc_event_box_f64(const orc_geometry* g, double z_u, double z_d,
                       double dl, int32_t box[6]);

/* Writes the event's in-ellipse pixel indices (y * n_z + z) in scan order;
 * returns the count (indices beyond cap are counted, not written). */
int64_t orc_pixel_set_f32(const orc_geometry* g, float z_u, float z_d,
                          float dl, int32_t* idx, int64_t cap);

/* Per event: bbox pixels tested, in-ellipse pixels, and an order-free 64-bit
 * digest of the set (sum over pixels of mix64(index)).  OpenMP parallel. */
void orc_pixel_set_stats_f32(const orc_geometry* g, const float* z_u,
                             const float* z_d, const float* dl, int64_t n,
                             int32_t* n_bb, int32_t* n_in, uint64_t* digest);
uint64_t orc_mix64(uint64_t x);

/* --- MLEM ----------------------------------------------------------------- */

/* Exact restatement of Reconstruction<float, GaussianKernel<float>>::operator()
 * with one thread (reconstruction.h:109-154, 220-298); ORC_MODE_GPU follows
 * the warp kernel's arithmetic (AnalyticKernel, sensitivity-weighted
 * denominator) with the CPU's zero-denominator rule.  rho is updated in place. */
void orc_mlem_f32(const orc_geometry* g, const float* z_u, const float* z_d,
                  const float* dl, int64_t n, float* rho, int n_iter, int mode);

/* FP64 oracle.  sets_f32 = 1 uses the binary32 pixel sets (the reference's
 * sets), 0 recomputes the sets in binary64.  n_subsets > 1 runs list-mode
 * OSEM: subset s holds events e with e % n_subsets == s, and each subset
 * update is rho_j <- n_subsets * rho_j * sum_{e in s} K_ej / D_e.
 * n_threads <= 0 uses all OpenMP threads. */
void orc_mlem_f64(const orc_geometry* g, const float* z_u, const float* z_d,
                  const float* dl, int64_t n, double* rho, int n_iter,
                  int mode, int n_subsets, int sets_f32, int n_threads);

/* --- projections and gradients (FP64, pixel sets from binary32) ------------ */

/* y_e = sum_j P_ej rho_j with P = K (cpu mode) or K * s (gpu mode); the kernel
 * uses (sigma_z, sigma_dl) while the pixel set stays the one the geometry's
 * sigmas define. */
void orc_forward_f64(const orc_geometry* g, const float* z_u, const float* z_d,
                     const float* dl, int64_t n, const double* rho,
                     double sigma_z, double sigma_dl, int mode, double* y);
/* g_j = sum_e P_ej w_e */
void orc_adjoint_f64(const orc_geometry* g, const float* z_u, const float* z_d,
                     const float* dl, int64_t n, const double* w,
                     double sigma_z, double sigma_dl, int mode, double* out);
/* d/dsigma of sum_e w_e y_e  (cpu mode: GaussianKernel) */
void orc_grad_sigma_f64(const orc_geometry* g, const float* z_u,
                        const float* z_d, const float* dl, int64_t n,
                        const double* rho, const double* w, double sigma_z,
                        double sigma_dl, double* d_sigma_z,
                        double* d_sigma_dl);

/* --- scalar pieces (golden-value tests) ----------------------------------- */

float orc_gaussian_kernel_f32(float sigma_z, float sigma_dl, float y, float tan,
                              float sec, float R, float dz, float dy);
double orc_gaussian_kernel_f64(double sigma_z, double sigma_dl, double y,
                               double tan, double sec, double R, double dz,
                               double dy);
float orc_analytic_kernel_f32(float sigma_z, float sigma_dl, float y, float tan,
                              float sec, float R, float dz, float dy);
double orc_analytic_kernel_f64(double sigma_z, double sigma_dl, double y,
                               double tan, double sec, double R, double dz,
                               double dy);
double orc_bb_y_f64(double A, double C, double B_2);
double orc_bb_z_f64(double A, double C, double B_2);
double orc_sensitivity_f64(const orc_geometry* g, double z, double y);
float orc_sensitivity_f32(const orc_geometry* g, float z, float y);
float orc_pixel_sensitivity_f32(const orc_geometry* g, int32_t px, int32_t py);
/* out[n_y * n_z]; five_point = 1: pixel_sensitivity, 0: center value */
void orc_sensitivity_image_f32(const orc_geometry* g, int five_point,
                               float* out);
void orc_pixel_at_f64(const orc_geometry* g, double z, double y, int32_t px[2]);
void orc_pixel_center_f64(const orc_geometry* g, int32_t px, int32_t py,
                          double pt[2]);
void orc_to_projection_tan_f64(double R, double y, double z, double tan,
                               double out[3]);
void orc_from_projection_tan_f64(double R, double z_u, double z_d, double dl,
                                 double out[3]);

/* --- synthetic events (strip_events.c) ----------------------------------- */

/* n seeded events of the benchmark's generator from ellipses given as
 * n_ellipses rows of (z, y, a, b, angle in degrees, activity); returns 0, or
 * -1 on bad arguments or an event no attempt could detect. */
int orc_generate_events(const orc_geometry* g, const double* ellipses,
                        int n_ellipses, uint64_t seed, int64_t n, float* z_u,
                        float* z_d, float* dl);

#ifdef __cplusplus
}
#endif

#endif
