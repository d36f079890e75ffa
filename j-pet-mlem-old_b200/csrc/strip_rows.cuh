// Row-interval enumeration of an event's pixel set.
//
// The reference tests every pixel of the clamped bounding box with
// GaussianKernel::in_ellipse (reconstruction.h:255-264).  Along one row the
// tested quantity q(dz) = (A dy dy) + (B dy dz) + (C dz dz) is a parabola in
// dz with curvature C = 2/sigma_z^2, so the pixels with q <= 9 form one
// contiguous run of columns: two pixels that pass with a failing pixel
// between them would need q to dip by C * p^2 (>= 0.03 for every geometry
// here) between samples, while binary32 rounding moves q by ~1e-5.  Each row's
// run is therefore found from the closed form of the ellipse (for the
// reference's A, B, C: dz = dy tan +- sqrt((9 - 4 sec^2 dy^2 / s_dl^2) s_z^2 / 2))
// and its two ends are settled with the *exact* binary32 predicate
// (strip_device.cuh), so the pixel set is the reference's bit for bit while
// only 2 pixels per row are tested instead of the whole row.
//
// One warp handles one event.  build_rows() gives each lane one row of a
// 32-row block, computes the row's exact run [lo, lo + len), its kernel row
// constants, and a warp prefix sum of the run lengths into per-warp shared
// tables; the runs are then walked as one flattened pixel list split evenly
// across the 32 lanes (walk_*), so every lane gets the same number of pixels.
#pragma once

#include "strip_device.cuh"
#include "strip_kernel_eval.cuh"

namespace stripmlem {

constexpr unsigned kWarpMask = 0xffffffffu;

// Per-warp shared-memory row tables for up to `cap` rows (a multiple of 32).
//   start[r]   flattened index of the first pixel of row r (start[0] = 0)
//   lo[r]      first column of row r's run
//   c[j][r]    kernel row constants (GaussRow: pref, c0, dytan; AnalyticRow:
//              n0, n1, u0, u1, cr, dytan)
struct RowTables {
  int* start;
  int* lo;
  float* c;
  int cap;
  __device__ __forceinline__ float& k(int j, int r) const { return c[j * cap + r]; }
};

constexpr int kRowConsts = 6;

__host__ __device__ inline int row_table_bytes(int cap) {
  return (cap + 1) * 4 + cap * 4 + kRowConsts * cap * 4;
}

__device__ __forceinline__ RowTables row_tables_at(char* base, int cap) {
  RowTables t;
  t.start = reinterpret_cast<int*>(base);
  t.lo = t.start + cap + 1;
  t.c = reinterpret_cast<float*>(t.lo + cap);
  t.cap = cap;
  return t;
}

// Event constants of the closed-form row runs.
struct EventRows {
  float k4;       // 4 sec^2 / s_dl^2   (u = 9 - k4 dy^2)
  float inv2z;    // s_z^2 / 2          (half width^2 = u * inv2z)
  float x0;       // (z - tl_z_half_w) / pw : column of the event centre
  float inv_pw;
};

__device__ __forceinline__ EventRows event_rows(const ScannerF& s,
                                                const EventF& e) {
  EventRows r;
  r.k4 = 4.0f * e.sec * e.sec * s.ipsdl;
  r.inv2z = s.inv2z;
  r.inv_pw = s.inv_pw;
  r.x0 = (e.z - s.tl_z_half_w) * r.inv_pw;
  return r;
}

__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Rows whose closed form is usable: the closed form locates each run end
// within ~1e-4 px (binary32 rounding of q is <= ~1e-4 even for the most
// tilted ellipses here, k = |B| / (2 sqrt(A C)) <= 0.93).  A column d >= 1/2
// pixel beyond an end has q - 9 = C pw^2 (d^2 + 2 d hw) >= C pw^2 (1/4 + hw)
// (hw the half width in pixels), far above that rounding whenever
// hw >= s.min_closed_hw (0 for sigma_z <= ~22 pixels: every row, the
// ellipse's tips and the empty rows of the box included).  So with m the
// column nearest to the closed-form end xl, every column left of m is
// outside and every column right of m up to the centre inside: the exact
// test of m alone decides the end (lo = m or m + 1), and likewise at xh --
// two exact tests per row, no loop, no divergence.  Other rows take the
// general search.
// Exact run of row iy within the box columns [tlx, brx): returns len, sets lo.
// CLOSED_ONLY: the geometry lets the closed form settle every row
// (s.min_closed_hw == 0), so the general search is compiled out; a row whose
// centre column is not finite or lies 1e7 columns away is empty (its ellipse
// cannot reach the box), as the general search finds.
template <bool CLOSED_ONLY = false>
__device__ __forceinline__ int row_run(const ScannerF& s, const EventF& e,
                                       const EventRows& er, const RowSet& rs,
                                       int& lo_out) {
  const int cmin = e.tlx, cmax = e.brx - 1;
  const float u = fmaf(-er.k4 * rs.dy, rs.dy, 9.0f);
  const float hw = sqrt_approx(fmaxf(u, 0.0f) * er.inv2z) * er.inv_pw;
  const float xv = fmaf(e.tan * rs.dy, er.inv_pw, er.x0);
  float xl = xv - hw, xh = xv + hw;
  int lo, hi;
  if (CLOSED_ONLY || (hw >= s.min_closed_hw && fabsf(xv) < 1e7f)) {
    if (CLOSED_ONLY && !(fabsf(xv) < 1e7f)) {
      lo_out = cmin;
      return 0;
    }
    const int ml = __float2int_rn(xl), mh = __float2int_rn(xh);
    const float ql = row_q(rs, e.C, col_dz(s, e, ml));
    const float qh = row_q(rs, e.C, col_dz(s, e, mh));
    lo = ql <= 9.0f ? ml : ml + 1;
    hi = qh <= 9.0f ? mh : mh - 1;
    lo = max(lo, cmin);
    hi = min(hi, cmax);
    lo_out = lo;
    return hi >= lo ? hi - lo + 1 : 0;
  }
  if (!(fabsf(xl) < 1e8f) || !(fabsf(xh) < 1e8f)) {
    lo = cmin;  // unusable closed form: scan the whole row
    hi = cmax;
  } else {
    xl = fminf(fmaxf(xl, (float)cmin - 2.0f), (float)cmax + 2.0f);
    xh = fminf(fmaxf(xh, (float)cmin - 2.0f), (float)cmax + 2.0f);
    lo = max((int)ceilf(xl) - 1, cmin);
    hi = min((int)floorf(xh) + 1, cmax);
  }
  while (lo <= hi && !in_ellipse(rs, e.C, col_dz(s, e, lo))) ++lo;
  while (hi >= lo && !in_ellipse(rs, e.C, col_dz(s, e, hi))) --hi;
  if (lo <= hi) {
    while (lo > cmin && in_ellipse(rs, e.C, col_dz(s, e, lo - 1))) --lo;
    while (hi < cmax && in_ellipse(rs, e.C, col_dz(s, e, hi + 1))) ++hi;
  }
  lo_out = lo;
  return hi >= lo ? hi - lo + 1 : 0;
}

// Builds the tables of rows [row0, row0 + nrows) (nrows <= cap) of event e.
// KC: 0 = no kernel constants, 1 = GaussRow, 2 = AnalyticRow.  Returns the
// number of pixels in those rows (same value in every lane).  Ends with a
// __syncwarp(); the caller must __syncwarp() before rebuilding.
template <int KC, bool CLOSED_ONLY = false>
__device__ __forceinline__ int build_rows(const ScannerF& s, const KernelF& k,
                                          const EventF& e, const EventRows& er,
                                          int row0, int nrows,
                                          const RowTables& T, int lane) {
  int base = 0;
  if (lane == 0) T.start[0] = 0;
  for (int b = 0; b < nrows; b += 32) {
    const int r = b + lane;
    int len = 0;
    if (r < nrows) {
      const RowSet rs = row_set(s, e, row0 + r);
      int lo;
      len = row_run<CLOSED_ONLY>(s, e, er, rs, lo);
      T.lo[r] = lo;
      if (KC == 1) {
        GaussRow g;
        g.init(k, s.R, e.y, e.tan, e.sec, rs.dy);
        T.k(0, r) = g.pref;
        T.k(1, r) = g.c0;
        T.k(2, r) = g.dytan;
      } else if (KC == 2) {
        AnalyticRow g;
        g.init(k, s.R, e.y, e.tan, e.sec, rs.dy);
        T.k(0, r) = g.n0;
        T.k(1, r) = g.n1;
        T.k(2, r) = g.u0;
        T.k(3, r) = g.u1;
        T.k(4, r) = g.cr;
        T.k(5, r) = g.dytan;
      }
    }
    // inclusive warp scan of the run lengths
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(kWarpMask, incl, o);
      if (lane >= o) incl += v;
    }
    if (r < nrows) T.start[r + 1] = base + incl;
    base += __shfl_sync(kWarpMask, incl, 31);
  }
  __syncwarp();
  return base;
}

// The lane's share [f0, f1) of the flattened pixel list of n pixels and the
// row holding f0 (largest r with start[r] <= f0).
__device__ __forceinline__ int lane_share(const RowTables& T, int nrows, int n,
                                          int lane, int& f0, int& f1) {
  f0 = (int)(((long long)n * lane) >> 5);
  f1 = (int)(((long long)n * (lane + 1)) >> 5);
  int a = 0, b = nrows;
  while (b - a > 1) {
    const int m = (a + b) >> 1;
    if (T.start[m] <= f0) a = m; else b = m;
  }
  return a;
}

}  // namespace stripmlem
