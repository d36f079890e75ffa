// Device-side geometry of the strip scanner: the binary32 arithmetic that
// decides which pixels belong to an event, written with explicitly rounded
// intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, __fsqrt_rn) in the reference's
// operation order, so nvcc cannot contract or reorder it and the pixel sets
// equal the reference CPU's bit for bit.  The kernel *values* (which only need
// the 1e-4 image tolerance) are evaluated separately with FMA and MUFU
// approximations (strip_kernel_eval.cuh).
#pragma once

#include <climits>
#include <cstdint>

namespace stripmlem {

// Scanner<float, short> constants (scanner.h:50-67) plus the
// GaussianKernel<float> constants that shape the 3-sigma ellipse
// (gaussian_kernel.h:27-33).  Filled on the host by make_scanner().
struct ScannerF {
  float R, L, pw, ph, sz, sdl, cy, cz;
  float tl_y, tl_z, tl_y_half_h, tl_z_half_w, half_L;
  float ipsz, ipsdl, kc;
  int n_y, n_z;  // after narrowing to int16, as Scanner<float, short>
  // launch constants of the closed-form row runs (not part of the exact
  // set arithmetic): 1 / pw, sigma_z^2 / 2, and the smallest closed-form
  // half width (pixels) whose run ends two exact tests settle
  float inv_pw, inv2z, min_closed_hw;
};

// One event after Response::calculate_tan_y_z (response.h:22-37) and
// GaussianKernel::ellipse_bb (gaussian_kernel.h:108-128), with the clamped
// bounding box of bb_update (reconstruction.h:225-246).  The scan visits rows
// [tly, bry) and columns [tlx, brx) -- half-open, as the reference's loops.
struct EventF {
  float tan, y, z, sec, A, B, C;
  int tlx, tly, brx, bry;
};

// float -> int32 as x86-64 cvttss2si (GCC's code for the reference): in-range
// values truncate toward zero, out-of-range and NaN give INT32_MIN.
__device__ __forceinline__ int f2i_x86(float x) {
  return (x >= -2147483648.0f && x < 2147483648.0f) ? (int)x : INT_MIN;
}
// int -> int16 keeping the low 16 bits (the reference's Pixel<short> fields).
__device__ __forceinline__ int i2s(int v) {
  return ((v & 0xFFFF) ^ 0x8000) - 0x8000;
}
__device__ __forceinline__ int wrap_add(int a, int b) {
  return (int)((unsigned)a + (unsigned)b);
}
__device__ __forceinline__ int wrap_sub(int a, int b) {
  return (int)((unsigned)a - (unsigned)b);
}

// Response::calculate_tan_y_z + GaussianKernel::ellipse_bb + Scanner::pixel_at
// + n_pixels_in_line + Pixel::clamp, in binary32 (see the file comment).
__device__ __forceinline__ void event_setup(const ScannerF& s, float z_u,
                                            float z_d, float dl, EventF& e) {
  // response.h:29-37
  const float tan = __fdiv_rn(__fsub_rn(z_u, z_d), __fmul_rn(2.0f, s.R));
  const float tt = __fmul_rn(tan, tan);
  const float y = __fmul_rn(-0.5f, __fdiv_rn(dl, __fsqrt_rn(__fadd_rn(1.0f, tt))));
  const float z = __fmul_rn(
      0.5f, __fadd_rn(__fadd_rn(z_u, z_d), __fmul_rn(__fmul_rn(2.0f, y), tan)));
  // gaussian_kernel.h:117-127
  const float sec = __fsqrt_rn(__fadd_rn(1.0f, tt));
  const float A = __fadd_rn(
      __fmul_rn(__fmul_rn(__fmul_rn(4.0f, sec), sec), s.ipsdl),
      __fmul_rn(__fmul_rn(2.0f, tt), s.ipsz));
  const float B = __fmul_rn(__fmul_rn(-4.0f, tan), s.ipsz);
  const float C = __fmul_rn(2.0f, s.ipsz);
  const float hb = __fdiv_rn(B, 2.0f);
  const float B_2 = __fmul_rn(hb, hb);
  const float bb_y = __fdiv_rn(3.0f, __fsqrt_rn(__fsub_rn(A, __fdiv_rn(B_2, C))));
  const float bb_z = __fdiv_rn(3.0f, __fsqrt_rn(__fsub_rn(C, __fdiv_rn(B_2, A))));
  // scanner.h:142-144 (float -> short)
  const int cx = i2s(f2i_x86(__fdiv_rn(__fsub_rn(z, s.tl_z), s.pw)));
  const int cy = i2s(f2i_x86(__fdiv_rn(__fsub_rn(s.tl_y, y), s.ph)));
  // reconstruction.h:216-218, 227-228
  const int hw = f2i_x86(__fadd_rn(__fdiv_rn(bb_z, s.pw), 0.5f));
  const int hh = f2i_x86(__fadd_rn(__fdiv_rn(bb_y, s.ph), 0.5f));
  // reconstruction.h:237-246, pixel.h:51-54
  int tlx = i2s(wrap_sub(cx, hw)), tly = i2s(wrap_sub(cy, hh));
  int brx = i2s(wrap_add(cx, hw)), bry = i2s(wrap_add(cy, hh));
  const int mx = i2s(s.n_z - 1), my = i2s(s.n_y - 1);
  tlx = min(mx, max(0, tlx));
  tly = min(my, max(0, tly));
  brx = min(mx, max(0, brx));
  bry = min(my, max(0, bry));
  e.tan = tan;
  e.y = y;
  e.z = z;
  e.sec = sec;
  e.A = A;
  e.B = B;
  e.C = C;
  e.tlx = tlx;
  e.tly = tly;
  e.brx = brx;
  e.bry = bry;
}

// Row part of GaussianKernel::in_ellipse (gaussian_kernel.h:131-137) for the
// pixel centre of row iy (scanner.h:136-139): dy, (A*dy)*dy and B*dy are the
// same binary32 values the reference computes for every pixel of the row.
struct RowSet {
  float dy, Ady2, Bdy;
};
__device__ __forceinline__ RowSet row_set(const ScannerF& s, const EventF& e,
                                          int iy) {
  RowSet r;
  const float py = __fsub_rn(s.tl_y_half_h, __fmul_rn((float)iy, s.ph));
  r.dy = __fsub_rn(py, e.y);
  r.Ady2 = __fmul_rn(__fmul_rn(e.A, r.dy), r.dy);
  r.Bdy = __fmul_rn(e.B, r.dy);
  return r;
}
// Column part: dz of pixel column iz.
__device__ __forceinline__ float col_dz(const ScannerF& s, const EventF& e,
                                        int iz) {
  const float pz = __fadd_rn(s.tl_z_half_w, __fmul_rn((float)iz, s.pw));
  return __fsub_rn(pz, e.z);
}
// (A*dy*dy) + (B*dy*dz) + (C*dz*dz), summed left to right; in the ellipse
// when <= 9.
__device__ __forceinline__ float row_q(const RowSet& r, float C, float dz) {
  return __fadd_rn(__fadd_rn(r.Ady2, __fmul_rn(r.Bdy, dz)),
                   __fmul_rn(__fmul_rn(C, dz), dz));
}
__device__ __forceinline__ bool in_ellipse(const RowSet& r, float C, float dz) {
  return row_q(r, C, dz) <= 9.0f;
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}

}  // namespace stripmlem
