/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the 2D strip list-mode TOF MLEM
 * path (see strip_oracle.h).  A plain-C restatement of the reference
 * JPETTomography/j-pet-mlem-old, src/2d/strip/.  Every function cites the
 * reference lines it follows.  Compiled with -ffp-contract=off: each binary32
 * expression below rounds exactly where the reference's C++ source rounds, in
 * the same order, so pixel sets (and single-thread images) are bit-identical
 * to the reference built with FMA contraction off.
 *
 * Parity pin: tests/test_oracle_ref.py runs the reference's own
 * 2d_strip_reconstruction (compiled from its sources into oracle/_ref by
 * oracle/Makefile) on the same event files and requires identical output
 * bytes; tests/test_oracle_golden.py checks the reference's unit-test golden
 * values (gaussian_kernel_test.cpp, kernel_test.cpp, scanner_test.cpp,
 * response_test.cpp).
 */
#define _GNU_SOURCE
#include "strip_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_1_PI
#define M_1_PI 0.31830988618379067154
#endif

/* ------------------------------------------------------------------------- */
/* Integer conversions with the semantics GCC gives the reference on x86-64:  */
/* float/double -> int via cvtts{s,d}2si (out of range or NaN -> INT32_MIN),  */
/* int -> short keeps the low 16 bits, int arithmetic wraps.                   */
/* ------------------------------------------------------------------------- */
static inline int32_t f2i(float x) {
  if (x >= -2147483648.0f && x < 2147483648.0f) return (int32_t)x;
  return INT32_MIN;
}
static inline int32_t d2i(double x) {
  if (x > -2147483649.0 && x < 2147483648.0) return (int32_t)x;
  return INT32_MIN;
}
static inline int16_t i2s(int32_t v) { return (int16_t)(uint16_t)(uint32_t)v; }
static inline int32_t wadd(int32_t a, int32_t b) {
  return (int32_t)((uint32_t)a + (uint32_t)b);
}
static inline int32_t wsub(int32_t a, int32_t b) {
  return (int32_t)((uint32_t)a - (uint32_t)b);
}
static inline int16_t smin(int16_t a, int16_t b) { return b < a ? b : a; }
static inline int16_t smax(int16_t a, int16_t b) { return a < b ? b : a; }

uint64_t orc_mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}

/* ========================================================================= */
/* binary32 scanner + kernel state                                           */
/* ========================================================================= */

/* Scanner<float, short> members (scanner.h:50-67, 271-290) and
 * GaussianKernel<float> constants (gaussian_kernel.h:27-33). */
typedef struct {
  float R, L;
  int16_t n_y, n_z;
  float pw, ph, sz, sdl, cy, cz;
  float size_y, size_z, tl_y, tl_z, tl_y_half_h, tl_z_half_w, half_L;
  float ipsz, ipsdl, kc;
} sf_t;

static void sf_init(sf_t* s, const orc_geometry* g) {
  s->R = (float)g->radius;
  s->L = (float)g->scintillator_length;
  s->n_y = i2s(g->n_y_pixels);
  s->n_z = i2s(g->n_z_pixels);
  s->ph = (float)g->pixel_height;
  s->pw = (float)g->pixel_width;
  s->sz = (float)g->sigma_z;
  s->sdl = (float)g->sigma_dl;
  s->cy = (float)g->center_y;
  s->cz = (float)g->center_z;
  s->size_y = (float)s->n_y * s->ph;          /* scanner.h:61 */
  s->size_z = (float)s->n_z * s->pw;          /* scanner.h:62 */
  s->tl_y = s->cy + s->size_y / 2.0f;         /* scanner.h:63 */
  s->tl_z = s->cz - s->size_z / 2.0f;         /* scanner.h:64 */
  s->tl_y_half_h = s->tl_y - s->ph / 2.0f;    /* scanner.h:65 */
  s->tl_z_half_w = s->tl_z + s->pw / 2.0f;    /* scanner.h:66 */
  s->half_L = s->L / 2.0f;                    /* scanner.h:67 */
  s->ipsz = 1.0f / (s->sz * s->sz);           /* gaussian_kernel.h:28 */
  s->ipsdl = 1.0f / (s->sdl * s->sdl);        /* gaussian_kernel.h:29 */
  /* gaussian_kernel.h:30-33: double constant times a float sqrt, narrowed */
  s->kc = (float)((1.0 / (2.0 * M_PI * M_PI)) *
                  (double)sqrtf((s->ipsz * s->ipsz) * s->ipsdl));
}

/* Event setup: Response::calculate_tan_y_z (response.h:22-37) followed by
 * GaussianKernel::ellipse_bb (gaussian_kernel.h:108-128, 159-160), pixel_at
 * (scanner.h:142-144), n_pixels_in_line (reconstruction.h:216-218) and the
 * clamped box (reconstruction.h:237-246, pixel.h:51-54). */
typedef struct {
  float tan, y, z, sec, A, B, C;
  int16_t cx, cy, tlx, tly, brx, bry;
} ef_t;

static inline void ef_setup(const sf_t* s, float z_u, float z_d, float dl,
                            ef_t* e) {
  float tan = (z_u - z_d) / (2.0f * s->R);
  float y = -0.5f * (dl / sqrtf(1.0f + tan * tan));
  float z = 0.5f * ((z_u + z_d) + ((2.0f * y) * tan));
  float tan_sq = tan * tan;
  float sec = sqrtf(1.0f + tan * tan);
  float A = (((4.0f * sec) * sec) * s->ipsdl) + ((2.0f * tan_sq) * s->ipsz);
  float B = (-4.0f * tan) * s->ipsz;
  float C = 2.0f * s->ipsz;
  float B_2 = (B / 2.0f) * (B / 2.0f);
  float bb_y = 3.0f / sqrtf(A - (B_2 / C));
  float bb_z = 3.0f / sqrtf(C - (B_2 / A));
  int16_t cx = i2s(f2i((z - s->tl_z) / s->pw));
  int16_t cy = i2s(f2i((s->tl_y - y) / s->ph));
  int32_t hw = f2i(bb_z / s->pw + 0.5f);
  int32_t hh = f2i(bb_y / s->ph + 0.5f);
  int16_t tlx = i2s(wsub(cx, hw)), tly = i2s(wsub(cy, hh));
  int16_t brx = i2s(wadd(cx, hw)), bry = i2s(wadd(cy, hh));
  int16_t mx = i2s((int32_t)s->n_z - 1), my = i2s((int32_t)s->n_y - 1);
  tlx = smin(mx, smax(0, tlx));
  tly = smin(my, smax(0, tly));
  brx = smin(mx, smax(0, brx));
  bry = smin(my, smax(0, bry));
  e->tan = tan;
  e->y = y;
  e->z = z;
  e->sec = sec;
  e->A = A;
  e->B = B;
  e->C = C;
  e->cx = cx;
  e->cy = cy;
  e->tlx = tlx;
  e->tly = tly;
  e->brx = brx;
  e->bry = bry;
}

/* pixel_center (scanner.h:136-139) then in_ellipse (gaussian_kernel.h:131-137);
 * dz/dy are also the kernel's `distance` (reconstruction.h:265). */
static inline int ef_in(const sf_t* s, const ef_t* e, int iz, int iy,
                        float* dz_out, float* dy_out) {
  float pz = s->tl_z_half_w + (float)iz * s->pw;
  float py = s->tl_y_half_h - (float)iy * s->ph;
  float dy = py - e->y;
  float dz = pz - e->z;
  *dz_out = dz;
  *dy_out = dy;
  return ((((e->A * dy) * dy) + ((e->B * dy) * dz)) + ((e->C * dz) * dz)) <=
         9.0f;
}

static inline float mic_f(float ipsz, float ipsdl, float ap, float aq, float ar,
                          float bp, float bq, float br) {
  /* multiply_inv_cor_mat, gaussian_kernel.h:152-156 */
  return (((ap * ipsz) * bp) + ((aq * ipsz) * bq)) + ((ar * ipsdl) * br);
}

/* GaussianKernel::operator() (gaussian_kernel.h:51-79) */
static inline float gk_f(float ipsz, float ipsdl, float kc, float y, float tan,
                         float sec, float R, float dz, float dy) {
  float sec_sq = sec * sec;
  float yp = dy + y;
  float ap = -(yp - R) * sec_sq;
  float aq = -(yp + R) * sec_sq;
  float ar = ((-2.0f * yp) * sec) * tan;
  float bpq = dz - (dy * tan);
  float br = (-2.0f * dy) * sec;
  float a_ic_a = mic_f(ipsz, ipsdl, ap, aq, ar, ap, aq, ar);
  float b_ic_b = mic_f(ipsz, ipsdl, bpq, bpq, br, bpq, bpq, br);
  float norm = a_ic_a;
  float before = kc / sqrtf(norm);
  float arg = -0.5f * b_ic_b;
  return before * expf(arg);
}

/* AnalyticKernel::operator() (analytic_kernel.h:28-62) */
static inline float ak_f(float ipsz, float ipsdl, float kc, float y, float tan,
                         float sec, float R, float dz, float dy) {
  float sec_sq = sec * sec;
  float yp = dy + y;
  float ap = -(yp - R) * sec_sq;
  float aq = -(yp + R) * sec_sq;
  float ar = ((-2.0f * yp) * sec) * tan;
  float op = ap * tan, oq = aq * tan;
  float orr = ((-yp) * sec) * (1.0f + ((2.0f * tan) * tan));
  float bpq = dz - (dy * tan);
  float br = (-2.0f * dy) * sec;
  float a_ic_a = mic_f(ipsz, ipsdl, ap, aq, ar, ap, aq, ar);
  float b_ic_a = mic_f(ipsz, ipsdl, bpq, bpq, br, ap, aq, ar);
  float b_ic_b = mic_f(ipsz, ipsdl, bpq, bpq, br, bpq, bpq, br);
  float o_ic_b = mic_f(ipsz, ipsdl, op, oq, orr, bpq, bpq, br);
  float norm = a_ic_a + 2.0f * o_ic_b;
  float before = kc / sqrtf(norm);
  float arg = -0.5f * (b_ic_b - ((b_ic_a * b_ic_a) / norm));
  return before * expf(arg);
}

/* Scanner::sensitivity (scanner.h:147-171), binary32 */
static inline float sens_f(const sf_t* s, float px, float py) {
  float L_plus = s->half_L + px;
  float L_minus = s->half_L - px;
  float R_plus = s->R + py;
  float R_minus = s->R - py;
  if (R_plus <= 0) R_plus = 1;
  if (R_minus <= 0) R_minus = 1;
  float a = L_minus / R_minus, b = L_plus / R_plus;
  float c = -L_plus / R_minus, d = -L_minus / R_plus;
  float mn = b < a ? b : a;   /* std::min(a, b) */
  float mx = c < d ? d : c;   /* std::max(c, d) */
  return (float)M_1_PI * (atanf(mn) - atanf(mx));
}

/* Scanner::pixel_sensitivity (scanner.h:174-185), binary32 */
static inline float pixel_sens_f(const sf_t* s, int px, int py) {
  float cz = s->tl_z_half_w + (float)px * s->pw;
  float cy = s->tl_y_half_h - (float)py * s->ph;
  float hx = s->pw / 2.0f, hy = s->ph / 2.0f;
  float nhx = -s->pw / 2.0f;
  return sens_f(s, cz, cy) / 3.0f + sens_f(s, cz + hx, cy + hy) / 6.0f +
         sens_f(s, cz - hx, cy - hy) / 6.0f +
         sens_f(s, cz + nhx, cy + hy) / 6.0f +
         sens_f(s, cz - nhx, cy - hy) / 6.0f;
}

/* ========================================================================= */
/* binary64 scanner + kernel state (Scanner<double, short>)                  */
/* ========================================================================= */
typedef struct {
  double R, L;
  int16_t n_y, n_z;
  double pw, ph, sz, sdl, cy, cz;
  double size_y, size_z, tl_y, tl_z, tl_y_half_h, tl_z_half_w, half_L;
  double ipsz, ipsdl, kc;
} sd_t;

static void sd_init_sigma(sd_t* s, const orc_geometry* g, double sz,
                          double sdl) {
  s->R = g->radius;
  s->L = g->scintillator_length;
  s->n_y = i2s(g->n_y_pixels);
  s->n_z = i2s(g->n_z_pixels);
  s->ph = g->pixel_height;
  s->pw = g->pixel_width;
  s->sz = sz;
  s->sdl = sdl;
  s->cy = g->center_y;
  s->cz = g->center_z;
  s->size_y = (double)s->n_y * s->ph;
  s->size_z = (double)s->n_z * s->pw;
  s->tl_y = s->cy + s->size_y / 2.0;
  s->tl_z = s->cz - s->size_z / 2.0;
  s->tl_y_half_h = s->tl_y - s->ph / 2.0;
  s->tl_z_half_w = s->tl_z + s->pw / 2.0;
  s->half_L = s->L / 2.0;
  s->ipsz = 1.0 / (sz * sz);
  s->ipsdl = 1.0 / (sdl * sdl);
  s->kc = (1.0 / (2.0 * M_PI * M_PI)) * sqrt((s->ipsz * s->ipsz) * s->ipsdl);
}
static void sd_init(sd_t* s, const orc_geometry* g) {
  sd_init_sigma(s, g, g->sigma_z, g->sigma_dl);
}

typedef struct {
  double tan, y, z, sec, A, B, C;
  int16_t cx, cy, tlx, tly, brx, bry;
} ed_t;

static inline void ed_setup(const sd_t* s, double z_u, double z_d, double dl,
                            ed_t* e) {
  double tan = (z_u - z_d) / (2.0 * s->R);
  double y = -0.5 * (dl / sqrt(1.0 + tan * tan));
  double z = 0.5 * ((z_u + z_d) + ((2.0 * y) * tan));
  double tan_sq = tan * tan;
  double sec = sqrt(1.0 + tan * tan);
  double A = (((4.0 * sec) * sec) * s->ipsdl) + ((2.0 * tan_sq) * s->ipsz);
  double B = (-4.0 * tan) * s->ipsz;
  double C = 2.0 * s->ipsz;
  double B_2 = (B / 2.0) * (B / 2.0);
  double bb_y = 3.0 / sqrt(A - (B_2 / C));
  double bb_z = 3.0 / sqrt(C - (B_2 / A));
  int16_t cx = i2s(d2i((z - s->tl_z) / s->pw));
  int16_t cy = i2s(d2i((s->tl_y - y) / s->ph));
  int32_t hw = d2i(bb_z / s->pw + 0.5);
  int32_t hh = d2i(bb_y / s->ph + 0.5);
  int16_t tlx = i2s(wsub(cx, hw)), tly = i2s(wsub(cy, hh));
  int16_t brx = i2s(wadd(cx, hw)), bry = i2s(wadd(cy, hh));
  int16_t mx = i2s((int32_t)s->n_z - 1), my = i2s((int32_t)s->n_y - 1);
  tlx = smin(mx, smax(0, tlx));
  tly = smin(my, smax(0, tly));
  brx = smin(mx, smax(0, brx));
  bry = smin(my, smax(0, bry));
  e->tan = tan;
  e->y = y;
  e->z = z;
  e->sec = sec;
  e->A = A;
  e->B = B;
  e->C = C;
  e->cx = cx;
  e->cy = cy;
  e->tlx = tlx;
  e->tly = tly;
  e->brx = brx;
  e->bry = bry;
}

static inline int ed_in(const sd_t* s, const ed_t* e, int iz, int iy,
                        double* dz_out, double* dy_out) {
  double pz = s->tl_z_half_w + (double)iz * s->pw;
  double py = s->tl_y_half_h - (double)iy * s->ph;
  double dy = py - e->y;
  double dz = pz - e->z;
  *dz_out = dz;
  *dy_out = dy;
  return ((((e->A * dy) * dy) + ((e->B * dy) * dz)) + ((e->C * dz) * dz)) <=
         9.0;
}

static inline double mic_d(double ipsz, double ipsdl, double ap, double aq,
                           double ar, double bp, double bq, double br) {
  return (((ap * ipsz) * bp) + ((aq * ipsz) * bq)) + ((ar * ipsdl) * br);
}

static inline double gk_d(double ipsz, double ipsdl, double kc, double y,
                          double tan, double sec, double R, double dz,
                          double dy) {
  double sec_sq = sec * sec;
  double yp = dy + y;
  double ap = -(yp - R) * sec_sq;
  double aq = -(yp + R) * sec_sq;
  double ar = ((-2.0 * yp) * sec) * tan;
  double bpq = dz - (dy * tan);
  double br = (-2.0 * dy) * sec;
  double a_ic_a = mic_d(ipsz, ipsdl, ap, aq, ar, ap, aq, ar);
  double b_ic_b = mic_d(ipsz, ipsdl, bpq, bpq, br, bpq, bpq, br);
  return kc / sqrt(a_ic_a) * exp(-0.5 * b_ic_b);
}

static inline double ak_d(double ipsz, double ipsdl, double kc, double y,
                          double tan, double sec, double R, double dz,
                          double dy) {
  double sec_sq = sec * sec;
  double yp = dy + y;
  double ap = -(yp - R) * sec_sq;
  double aq = -(yp + R) * sec_sq;
  double ar = ((-2.0 * yp) * sec) * tan;
  double op = ap * tan, oq = aq * tan;
  double orr = ((-yp) * sec) * (1.0 + ((2.0 * tan) * tan));
  double bpq = dz - (dy * tan);
  double br = (-2.0 * dy) * sec;
  double a_ic_a = mic_d(ipsz, ipsdl, ap, aq, ar, ap, aq, ar);
  double b_ic_a = mic_d(ipsz, ipsdl, bpq, bpq, br, ap, aq, ar);
  double b_ic_b = mic_d(ipsz, ipsdl, bpq, bpq, br, bpq, bpq, br);
  double o_ic_b = mic_d(ipsz, ipsdl, op, oq, orr, bpq, bpq, br);
  double norm = a_ic_a + 2.0 * o_ic_b;
  return kc / sqrt(norm) * exp(-0.5 * (b_ic_b - ((b_ic_a * b_ic_a) / norm)));
}

static inline double sens_d(const sd_t* s, double px, double py) {
  double L_plus = s->half_L + px;
  double L_minus = s->half_L - px;
  double R_plus = s->R + py;
  double R_minus = s->R - py;
  if (R_plus <= 0) R_plus = 1;
  if (R_minus <= 0) R_minus = 1;
  double a = L_minus / R_minus, b = L_plus / R_plus;
  double c = -L_plus / R_minus, d = -L_minus / R_plus;
  double mn = b < a ? b : a;
  double mx = c < d ? d : c;
  return M_1_PI * (atan(mn) - atan(mx));
}

static inline double pixel_sens_d(const sd_t* s, int px, int py) {
  double cz = s->tl_z_half_w + (double)px * s->pw;
  double cy = s->tl_y_half_h - (double)py * s->ph;
  double hx = s->pw / 2.0, hy = s->ph / 2.0;
  return sens_d(s, cz, cy) / 3.0 + sens_d(s, cz + hx, cy + hy) / 6.0 +
         sens_d(s, cz - hx, cy - hy) / 6.0 +
         sens_d(s, cz - hx, cy + hy) / 6.0 +
         sens_d(s, cz + hx, cy - hy) / 6.0;
}

/* ========================================================================= */
/* Per-event geometry API                                                     */
/* ========================================================================= */

void orc_event_box_f32(const orc_geometry* g, float z_u, float z_d, float dl,
                       int32_t box[6]) {
  sf_t s;
  ef_t e;
  sf_init(&s, g);
  ef_setup(&s, z_u, z_d, dl, &e);
  box[0] = e.cx;
  box[1] = e.cy;
  box[2] = e.tlx;
  box[3] = e.tly;
  box[4] = e.brx;
  box[5] = e.bry;
}

void orc_event_box_f64(const orc_geometry* g, double z_u, double z_d,
                       double dl, int32_t box[6]) {
  sd_t s;
  ed_t e;
  sd_init(&s, g);
  ed_setup(&s, z_u, z_d, dl, &e);
  box[0] = e.cx;
  box[1] = e.cy;
  box[2] = e.tlx;
  box[3] = e.tly;
  box[4] = e.brx;
  box[5] = e.bry;
}

int64_t orc_pixel_set_f32(const orc_geometry* g, float z_u, float z_d,
                          float dl, int32_t* idx, int64_t cap) {
  sf_t s;
  ef_t e;
  sf_init(&s, g);
  ef_setup(&s, z_u, z_d, dl, &e);
  int64_t n = 0;
  for (int iy = e.tly; iy < e.bry; ++iy)
    for (int iz = e.tlx; iz < e.brx; ++iz) {
      float dz, dy;
      if (ef_in(&s, &e, iz, iy, &dz, &dy)) {
        if (n < cap) idx[n] = iy * (int32_t)s.n_z + iz;
        ++n;
      }
    }
  return n;
}

void orc_pixel_set_stats_f32(const orc_geometry* g, const float* z_u,
                             const float* z_d, const float* dl, int64_t n,
                             int32_t* n_bb, int32_t* n_in, uint64_t* digest) {
  sf_t s;
  sf_init(&s, g);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < n; ++i) {
    ef_t e;
    ef_setup(&s, z_u[i], z_d[i], dl[i], &e);
    int32_t cnt = 0;
    uint64_t h = 0;
    for (int iy = e.tly; iy < e.bry; ++iy)
      for (int iz = e.tlx; iz < e.brx; ++iz) {
        float dz, dy;
        if (ef_in(&s, &e, iz, iy, &dz, &dy)) {
          ++cnt;
          h += orc_mix64((uint64_t)(iy * (int32_t)s.n_z + iz) + 1u);
        }
      }
    int32_t w = e.brx - e.tlx, hgt = e.bry - e.tly;
    if (n_bb) n_bb[i] = (w > 0 && hgt > 0) ? w * hgt : 0;
    if (n_in) n_in[i] = cnt;
    if (digest) digest[i] = h;
  }
}

/* ========================================================================= */
/* MLEM                                                                       */
/* ========================================================================= */

/* Reconstruction::operator() + bb_update with one OpenMP thread
 * (reconstruction.h:109-154, 220-298).  ORC_MODE_GPU swaps in the warp
 * kernel's arithmetic: AnalyticKernel and denominator += K*rho*s
 * (warp_granularity.cuh:347-357), scatter K*rho*inv (:397-399). */
void orc_mlem_f32(const orc_geometry* g, const float* z_u, const float* z_d,
                  const float* dl, int64_t n, float* rho, int n_iter,
                  int mode) {
  sf_t s;
  sf_init(&s, g);
  const int64_t total = (int64_t)s.n_y * s.n_z;
  float* out = (float*)malloc(sizeof(float) * (size_t)total);
  float* sens = NULL;
  if (mode == ORC_MODE_GPU) {
    sens = (float*)malloc(sizeof(float) * (size_t)total);
    for (int y = 0; y < s.n_y; ++y)
      for (int x = 0; x < s.n_z; ++x)
        sens[(int64_t)y * s.n_z + x] = pixel_sens_f(&s, x, y);
  }
  /* per-event caches, as the reference's alloca buffers */
  int64_t cap = 1 << 16;
  int32_t* cache_idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
  float* cache_val = (float*)malloc(sizeof(float) * (size_t)cap);

  for (int it = 0; it < n_iter; ++it) {
    memset(out, 0, sizeof(float) * (size_t)total);
    for (int64_t i = 0; i < n; ++i) {
      ef_t e;
      ef_setup(&s, z_u[i], z_d[i], dl[i], &e);
      int64_t bb = (int64_t)(e.brx - e.tlx) * (e.bry - e.tly);
      if (bb > cap) {
        cap = bb;
        cache_idx = (int32_t*)realloc(cache_idx, sizeof(int32_t) * (size_t)cap);
        cache_val = (float*)realloc(cache_val, sizeof(float) * (size_t)cap);
      }
      int64_t m = 0;
      float den = 0;
      for (int iy = e.tly; iy < e.bry; ++iy)
        for (int iz = e.tlx; iz < e.brx; ++iz) {
          float dz, dy;
          if (!ef_in(&s, &e, iz, iy, &dz, &dy)) continue;
          int32_t pi = iy * (int32_t)s.n_z + iz;
          float kv, kr;
          if (mode == ORC_MODE_GPU) {
            kv = ak_f(s.ipsz, s.ipsdl, s.kc, e.y, e.tan, e.sec, s.R, dz, dy);
            kr = kv * rho[pi];
            den += kr * sens[pi];
          } else {
            kv = gk_f(s.ipsz, s.ipsdl, s.kc, e.y, e.tan, e.sec, s.R, dz, dy);
            kr = kv * rho[pi];
            den += kr;
            kr = kr / 1.0f; /* kernel_mul_rho / pixel_sensitivity (== 1) */
          }
          cache_idx[m] = pi;
          cache_val[m] = kr;
          ++m;
        }
      float inv = (den > 0) ? 1.0f / den : 0.0f;
      for (int64_t p = 0; p < m; ++p) out[cache_idx[p]] += cache_val[p] * inv;
    }
    /* rho.assign(0); rho[i] += thread_rho[i]  (reconstruction.h:143-149) */
    for (int64_t j = 0; j < total; ++j) rho[j] = 0.0f + out[j];
  }
  free(cache_idx);
  free(cache_val);
  free(sens);
  free(out);
}

/* One event's contribution in binary64: visits the event's pixel set (from
 * binary32 or binary64 geometry) and returns the count.  The callback-free
 * form keeps the hot oracle loops plain. */
typedef struct {
  int32_t pi;
  double k;
} kd_t;

static int64_t event_kernels_d(const sf_t* sf, const sd_t* sd, int sets_f32,
                               int mode, float zu, float zd, float dlv,
                               kd_t** buf, int64_t* cap) {
  ed_t ed;
  ed_setup(sd, (double)zu, (double)zd, (double)dlv, &ed);
  int16_t tlx = ed.tlx, tly = ed.tly, brx = ed.brx, bry = ed.bry;
  ef_t ef;
  if (sets_f32) {
    ef_setup(sf, zu, zd, dlv, &ef);
    tlx = ef.tlx;
    tly = ef.tly;
    brx = ef.brx;
    bry = ef.bry;
  }
  int64_t bb = (int64_t)(brx - tlx) * (bry - tly);
  if (bb <= 0) return 0;
  if (bb > *cap) {
    *cap = bb;
    *buf = (kd_t*)realloc(*buf, sizeof(kd_t) * (size_t)bb);
  }
  int64_t m = 0;
  for (int iy = tly; iy < bry; ++iy)
    for (int iz = tlx; iz < brx; ++iz) {
      double dz, dy;
      int in;
      if (sets_f32) {
        float fz, fy;
        in = ef_in(sf, &ef, iz, iy, &fz, &fy);
        dz = sd->tl_z_half_w + (double)iz * sd->pw - ed.z;
        dy = sd->tl_y_half_h - (double)iy * sd->ph - ed.y;
      } else {
        in = ed_in(sd, &ed, iz, iy, &dz, &dy);
      }
      if (!in) continue;
      double kv = (mode == ORC_MODE_GPU)
                      ? ak_d(sd->ipsz, sd->ipsdl, sd->kc, ed.y, ed.tan, ed.sec,
                             sd->R, dz, dy)
                      : gk_d(sd->ipsz, sd->ipsdl, sd->kc, ed.y, ed.tan, ed.sec,
                             sd->R, dz, dy);
      (*buf)[m].pi = iy * (int32_t)sd->n_z + iz;
      (*buf)[m].k = kv;
      ++m;
    }
  return m;
}

static double* sens_image_d(const sd_t* sd) {
  int64_t total = (int64_t)sd->n_y * sd->n_z;
  double* sens = (double*)malloc(sizeof(double) * (size_t)total);
  for (int y = 0; y < sd->n_y; ++y)
    for (int x = 0; x < sd->n_z; ++x)
      sens[(int64_t)y * sd->n_z + x] = pixel_sens_d(sd, x, y);
  return sens;
}

void orc_mlem_f64(const orc_geometry* g, const float* z_u, const float* z_d,
                  const float* dl, int64_t n, double* rho, int n_iter,
                  int mode, int n_subsets, int sets_f32, int n_threads) {
  sf_t sf;
  sd_t sd;
  sf_init(&sf, g);
  sd_init(&sd, g);
  if (n_subsets < 1) n_subsets = 1;
  const int64_t total = (int64_t)sd.n_y * sd.n_z;
  double* sens = (mode == ORC_MODE_GPU) ? sens_image_d(&sd) : NULL;
  int nt = 1;
#ifdef _OPENMP
  nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#endif
  double* acc = (double*)calloc((size_t)nt * (size_t)total, sizeof(double));

  for (int it = 0; it < n_iter; ++it) {
    for (int sub = 0; sub < n_subsets; ++sub) {
      memset(acc, 0, sizeof(double) * (size_t)nt * (size_t)total);
      int64_t n_sub = (n - sub + n_subsets - 1) / n_subsets;
#pragma omp parallel num_threads(nt)
      {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double* my = acc + (int64_t)t * total;
        kd_t* buf = NULL;
        int64_t cap = 0;
#pragma omp for schedule(dynamic, 256)
        for (int64_t k = 0; k < n_sub; ++k) {
          int64_t i = sub + k * n_subsets;
          int64_t m = event_kernels_d(&sf, &sd, sets_f32, mode, z_u[i], z_d[i],
                                      dl[i], &buf, &cap);
          double den = 0;
          for (int64_t p = 0; p < m; ++p) {
            double w = buf[p].k * rho[buf[p].pi];
            if (sens) w *= sens[buf[p].pi];
            den += w;
          }
          double inv = den > 0 ? 1.0 / den : 0.0;
          for (int64_t p = 0; p < m; ++p) my[buf[p].pi] += buf[p].k * inv;
        }
        free(buf);
      }
      for (int64_t j = 0; j < total; ++j) {
        double gsum = 0;
        for (int t = 0; t < nt; ++t) gsum += acc[(int64_t)t * total + j];
        rho[j] = rho[j] * gsum * (double)n_subsets;
      }
    }
  }
  free(acc);
  free(sens);
}

/* ========================================================================= */
/* Projections and gradients (binary64; pixel sets from binary32)            */
/* ========================================================================= */

void orc_forward_f64(const orc_geometry* g, const float* z_u, const float* z_d,
                     const float* dl, int64_t n, const double* rho,
                     double sigma_z, double sigma_dl, int mode, double* y) {
  sf_t sf;
  sd_t sd;
  sf_init(&sf, g);
  sd_init_sigma(&sd, g, sigma_z, sigma_dl);
  double* sens = (mode == ORC_MODE_GPU) ? sens_image_d(&sd) : NULL;
#pragma omp parallel
  {
    kd_t* buf = NULL;
    int64_t cap = 0;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
      int64_t m = event_kernels_d(&sf, &sd, 1, mode, z_u[i], z_d[i], dl[i],
                                  &buf, &cap);
      double acc = 0;
      for (int64_t p = 0; p < m; ++p) {
        double w = buf[p].k * rho[buf[p].pi];
        if (sens) w *= sens[buf[p].pi];
        acc += w;
      }
      y[i] = acc;
    }
    free(buf);
  }
  free(sens);
}

void orc_adjoint_f64(const orc_geometry* g, const float* z_u, const float* z_d,
                     const float* dl, int64_t n, const double* w,
                     double sigma_z, double sigma_dl, int mode, double* out) {
  sf_t sf;
  sd_t sd;
  sf_init(&sf, g);
  sd_init_sigma(&sd, g, sigma_z, sigma_dl);
  const int64_t total = (int64_t)sd.n_y * sd.n_z;
  double* sens = (mode == ORC_MODE_GPU) ? sens_image_d(&sd) : NULL;
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  double* acc = (double*)calloc((size_t)nt * (size_t)total, sizeof(double));
#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    double* my = acc + (int64_t)t * total;
    kd_t* buf = NULL;
    int64_t cap = 0;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
      int64_t m = event_kernels_d(&sf, &sd, 1, mode, z_u[i], z_d[i], dl[i],
                                  &buf, &cap);
      for (int64_t p = 0; p < m; ++p) my[buf[p].pi] += buf[p].k * w[i];
    }
    free(buf);
  }
  for (int64_t j = 0; j < total; ++j) {
    double s = 0;
    for (int t = 0; t < nt; ++t) s += acc[(int64_t)t * total + j];
    out[j] = sens ? s * sens[j] : s;
  }
  free(acc);
  free(sens);
}

/* d K / d sigma for the GaussianKernel (gaussian_kernel.h:51-79):
 *   log K = log(1/(2 pi^2)) - 2 log sz - log sdl - log(norm)/2 - b_ic_b/2
 * with norm = (ap^2+aq^2)/sz^2 + ar^2/sdl^2, b_ic_b = 2 bpq^2/sz^2 + br^2/sdl^2 */
void orc_grad_sigma_f64(const orc_geometry* g, const float* z_u,
                        const float* z_d, const float* dl, int64_t n,
                        const double* rho, const double* w, double sigma_z,
                        double sigma_dl, double* d_sigma_z,
                        double* d_sigma_dl) {
  sf_t sf;
  sd_t sd;
  sf_init(&sf, g);
  sd_init_sigma(&sd, g, sigma_z, sigma_dl);
  double gz = 0, gdl = 0;
  const double sz = sigma_z, sdl = sigma_dl;
  const double sz3 = sz * sz * sz, sdl3 = sdl * sdl * sdl;
#pragma omp parallel reduction(+ : gz, gdl)
  {
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
      ef_t ef;
      ed_t ed;
      ef_setup(&sf, z_u[i], z_d[i], dl[i], &ef);
      ed_setup(&sd, (double)z_u[i], (double)z_d[i], (double)dl[i], &ed);
      double ez = 0, edl = 0;
      for (int iy = ef.tly; iy < ef.bry; ++iy)
        for (int iz = ef.tlx; iz < ef.brx; ++iz) {
          float fz, fy;
          if (!ef_in(&sf, &ef, iz, iy, &fz, &fy)) continue;
          double dz = sd.tl_z_half_w + (double)iz * sd.pw - ed.z;
          double dy = sd.tl_y_half_h - (double)iy * sd.ph - ed.y;
          double sec_sq = ed.sec * ed.sec, yp = dy + ed.y;
          double ap = -(yp - sd.R) * sec_sq, aq = -(yp + sd.R) * sec_sq;
          double ar = -2.0 * yp * ed.sec * ed.tan;
          double bpq = dz - dy * ed.tan, br = -2.0 * dy * ed.sec;
          double apq2 = ap * ap + aq * aq, bpq2 = 2.0 * bpq * bpq;
          double norm = apq2 * sd.ipsz + ar * ar * sd.ipsdl;
          double k = gk_d(sd.ipsz, sd.ipsdl, sd.kc, ed.y, ed.tan, ed.sec, sd.R,
                          dz, dy);
          double dlz = -2.0 / sz + apq2 / (sz3 * norm) + bpq2 / sz3;
          double dld = -1.0 / sdl + ar * ar / (sdl3 * norm) + br * br / sdl3;
          double kr = k * rho[iy * (int32_t)sd.n_z + iz];
          ez += kr * dlz;
          edl += kr * dld;
        }
      gz += w[i] * ez;
      gdl += w[i] * edl;
    }
  }
  *d_sigma_z = gz;
  *d_sigma_dl = gdl;
}

/* ========================================================================= */
/* Scalar pieces                                                              */
/* ========================================================================= */

float orc_gaussian_kernel_f32(float sigma_z, float sigma_dl, float y, float tan,
                              float sec, float R, float dz, float dy) {
  float ipsz = 1.0f / (sigma_z * sigma_z), ipsdl = 1.0f / (sigma_dl * sigma_dl);
  float kc = (float)((1.0 / (2.0 * M_PI * M_PI)) *
                     (double)sqrtf((ipsz * ipsz) * ipsdl));
  return gk_f(ipsz, ipsdl, kc, y, tan, sec, R, dz, dy);
}

double orc_gaussian_kernel_f64(double sigma_z, double sigma_dl, double y,
                               double tan, double sec, double R, double dz,
                               double dy) {
  double ipsz = 1.0 / (sigma_z * sigma_z), ipsdl = 1.0 / (sigma_dl * sigma_dl);
  double kc = (1.0 / (2.0 * M_PI * M_PI)) * sqrt((ipsz * ipsz) * ipsdl);
  return gk_d(ipsz, ipsdl, kc, y, tan, sec, R, dz, dy);
}

float orc_analytic_kernel_f32(float sigma_z, float sigma_dl, float y, float tan,
                              float sec, float R, float dz, float dy) {
  float ipsz = 1.0f / (sigma_z * sigma_z), ipsdl = 1.0f / (sigma_dl * sigma_dl);
  float kc = (float)((1.0 / (2.0 * M_PI * M_PI)) *
                     (double)sqrtf((ipsz * ipsz) * ipsdl));
  return ak_f(ipsz, ipsdl, kc, y, tan, sec, R, dz, dy);
}

double orc_analytic_kernel_f64(double sigma_z, double sigma_dl, double y,
                               double tan, double sec, double R, double dz,
                               double dy) {
  double ipsz = 1.0 / (sigma_z * sigma_z), ipsdl = 1.0 / (sigma_dl * sigma_dl);
  double kc = (1.0 / (2.0 * M_PI * M_PI)) * sqrt((ipsz * ipsz) * ipsdl);
  return ak_d(ipsz, ipsdl, kc, y, tan, sec, R, dz, dy);
}

/* GaussianKernel::bb_y / bb_z (gaussian_kernel.h:159-160) */
double orc_bb_y_f64(double A, double C, double B_2) {
  return 3.0 / sqrt(A - (B_2 / C));
}
double orc_bb_z_f64(double A, double C, double B_2) {
  return 3.0 / sqrt(C - (B_2 / A));
}

double orc_sensitivity_f64(const orc_geometry* g, double z, double y) {
  sd_t s;
  sd_init(&s, g);
  return sens_d(&s, z, y);
}

float orc_sensitivity_f32(const orc_geometry* g, float z, float y) {
  sf_t s;
  sf_init(&s, g);
  return sens_f(&s, z, y);
}

float orc_pixel_sensitivity_f32(const orc_geometry* g, int32_t px,
                                int32_t py) {
  sf_t s;
  sf_init(&s, g);
  return pixel_sens_f(&s, px, py);
}

void orc_sensitivity_image_f32(const orc_geometry* g, int five_point,
                               float* out) {
  sf_t s;
  sf_init(&s, g);
  for (int y = 0; y < s.n_y; ++y)
    for (int x = 0; x < s.n_z; ++x) {
      float v;
      if (five_point) {
        v = pixel_sens_f(&s, x, y);
      } else {
        float cz = s.tl_z_half_w + (float)x * s.pw;
        float cy = s.tl_y_half_h - (float)y * s.ph;
        v = sens_f(&s, cz, cy);
      }
      out[(int64_t)y * s.n_z + x] = v;
    }
}

/* pixel_at / pixel_center of Scanner<double, short> (scanner.h:136-144) */
void orc_pixel_at_f64(const orc_geometry* g, double z, double y,
                      int32_t px[2]) {
  sd_t s;
  sd_init(&s, g);
  px[0] = i2s(d2i((z - s.tl_z) / s.pw));
  px[1] = i2s(d2i((s.tl_y - y) / s.ph));
}

void orc_pixel_center_f64(const orc_geometry* g, int32_t px, int32_t py,
                          double pt[2]) {
  sd_t s;
  sd_init(&s, g);
  pt[0] = s.tl_z_half_w + (double)i2s(px) * s.pw;
  pt[1] = s.tl_y_half_h - (double)i2s(py) * s.ph;
}

/* Scanner::to_projection_space_tan (scanner.h:107-113): out = z_u, z_d, dl */
void orc_to_projection_tan_f64(double R, double y, double z, double tan,
                               double out[3]) {
  out[0] = z + (R - y) * tan;
  out[1] = z - (R + y) * tan;
  out[2] = -2.0 * y * sqrt(tan * tan + 1.0);
}

/* Response::calculate_tan_y_z (response.h:22-37): out = tan, y, z */
void orc_from_projection_tan_f64(double R, double z_u, double z_d, double dl,
                                 double out[3]) {
  double tan = (z_u - z_d) / (2.0 * R);
  double y = -0.5 * (dl / sqrt(1.0 + tan * tan));
  double z = 0.5 * ((z_u + z_d) + ((2.0 * y) * tan));
  out[0] = tan;
  out[1] = y;
  out[2] = z;
}
