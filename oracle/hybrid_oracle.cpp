// TEST INFRASTRUCTURE ONLY -- CPU restatement of the reference's 3D hybrid
// list-mode MLEM (src/3d/hybrid/reconstruction.h) for the parity tests.  The
// product never links this file.  Compiled with -ffp-contract=off so each
// binary32 operation rounds where the reference's C++ source says.
#include "hybrid_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr int kSeg = 9;  // start xy, end xy, mid xy, direction xy, length

// LOR<S>::index, src/2d/barrel/lor.h:33-35 (first >= second).
inline int64_t lor_index(int64_t first, int64_t second) {
  return first * (first + 1) / 2 + second;
}

// PixelGrid(n, n, size): lower_left = (-size * n / 2, ...), the pixel centre
// lower_left + size/2 + index * size (src/2d/geometry/pixel_grid.h:22-50).
struct Grid {
  float llc_x, llc_y, p;
  int32_t nc, nr, np;
  float z_left;
  explicit Grid(const hyb_setup* s)
      : p(s->pixel_size), nc(s->n_columns), nr(s->n_rows), np(s->n_planes),
        z_left(s->z_left) {
    const float llx = -p * (float)nc / 2;
    const float lly = -p * (float)nr / 2;
    llc_x = llx + p / 2;
    llc_y = lly + p / 2;
  }
  float cx(int x) const { return llc_x + (float)x * p; }
  float cy(int y) const { return llc_y + (float)y * p; }
  bool contains(int x, int y) const { return x >= 0 && x < nc && y >= 0 && y < nr; }
  // VoxelGrid::center_z_at (voxel_grid.h:38-40)
  float center_z(int iz) const { return ((float)iz + 0.5f) * p + z_left; }
  // Reconstruction::plane (reconstruction.h:149): truncation to short
  int16_t plane(float z) const { return (int16_t)(int)((z - z_left) / p); }
};

// LineSegment(start, end), src/2d/geometry/line_segment.h:18-27.
void make_segment(float sx, float sy, float ex, float ey, float* o) {
  const float vx = ex - sx, vy = ey - sy;
  const float l = std::sqrt(vx * vx + vy * vy);
  o[0] = sx;
  o[1] = sy;
  o[2] = ex;
  o[3] = ey;
  o[4] = (sx + ex) / 2;
  o[5] = (sy + ey) / 2;
  o[6] = vx / l;
  o[7] = vy / l;
  o[8] = std::sqrt(vx * vx + vy * vy);
}

// GaussianKernel<F>, src/2d/strip/gaussian_kernel.h.
template <typename F> struct Kernel {
  F ipz, ipdl, norm_c;
  Kernel(float sigma_z, float sigma_dl) {
    const F sz = (F)sigma_z, sdl = (F)sigma_dl;
    ipz = 1 / (sz * sz);
    ipdl = 1 / (sdl * sdl);
    norm_c = (F)(1 / (2 * M_PI * M_PI) * std::sqrt(ipz * ipz * ipdl));
  }
  // operator()(y, tan, sec, R, distance), gaussian_kernel.h:51-79
  F value(F y, F tan, F sec, F R, F dx, F dy) const {
    const F sec_sq = sec * sec;
    const F yp = dy + y;
    const F ap = -(yp - R) * sec_sq;
    const F aq = -(yp + R) * sec_sq;
    const F ar = -2 * yp * sec * tan;
    const F bpq = dx - dy * tan;
    const F br = -2 * dy * sec;
    const F a_ic_a = ap * ipz * ap + aq * ipz * aq + ar * ipdl * ar;
    const F b_ic_b = bpq * ipz * bpq + bpq * ipz * bpq + br * ipdl * br;
    const F before = norm_c / std::sqrt(a_ic_a);
    const F arg = -F(0.5) * (b_ic_b);
    return before * std::exp(arg);
  }
  // sensitivity(p, R, L), gaussian_kernel.h:139-148
  static F sensitivity(F px, F py, F R, F L) {
    const F L2 = L / 2;
    const F tmax = std::atan(std::min((L2 - px) / (R - py), (L2 + px) / (R + py)));
    const F tmin = std::atan(std::max(-(L2 + px) / (R - py), (-L2 + px) / (R + py)));
    const F sens = tmax - tmin;
    return sens / (F)M_PI;
  }
  // normalized(event, tan, sec, R, L, p), gaussian_kernel.h:93-105
  F normalized(F ev_x, F ev_y, F tan, F sec, F R, F L, F px, F py) const {
    const F dx = px - ev_x, dy = py - ev_y;
    const F un = value(ev_y, tan, sec, R, dx, dy);
    const F sens = sensitivity(px, py, R, L);
    return un / sens;
  }
};

template <typename F>
void mlem(const hyb_setup* s, const float* seg, const int16_t* pix, const float* w,
          const float* sens, const hyb_frame* frames, int64_t n_frames, F* rho,
          int32_t n_iter, hyb_stats* stats) {
  const Grid g(s);
  const Kernel<F> kernel(s->sigma_z, s->sigma_dl);
  const int64_t n_pixels = (int64_t)g.nc * g.nr;
  const int64_t n_voxels = n_pixels * g.np;
  std::vector<F> out(n_voxels), cache(n_voxels);
  hyb_stats st{0, 0, 0};
  for (int32_t it = 0; it < n_iter; ++it) {
    std::fill(out.begin(), out.end(), F(0));
    std::fill(cache.begin(), cache.end(), F(0));
    st = hyb_stats{0, 0, 0};
    for (int64_t i = 0; i < n_frames; ++i) {
      const hyb_frame& ev = frames[i];
      st.used_events++;
      const float* sg = seg + (int64_t)ev.lor_index * kSeg;
      const F R = (F)(sg[8] / 2);
      F denominator = 0;
      for (int64_t info = ev.info_begin; info < ev.info_end; ++info) {
        st.used_pixels++;
        const int x = pix[2 * info], y = pix[2 * info + 1];
        const F pixel_weight = (F)w[info];
        const int64_t pidx = x + (int64_t)g.nc * y;
        // projection_relative_middle (line_segment.h:58-60), in float
        const float cx = g.cx(x), cy = g.cy(y);
        const F up = (F)((cx - sg[4]) * sg[6] + (cy - sg[5]) * sg[7]);
        for (int iz = ev.plane_begin; iz < ev.plane_end; ++iz) {
          st.used_voxels++;
          const int64_t vidx = pidx + (int64_t)iz * n_pixels;
          const F z = (F)g.center_z(iz);
          const F k2d = kernel.normalized((F)ev.right, (F)ev.up, (F)ev.tan, (F)ev.sec, R,
                                          (F)s->length, z, up);
          if (k2d <= 0) {
            cache[vidx] = 0;
            continue;
          }
          const F weight = k2d * pixel_weight * rho[vidx];
          denominator += weight * (F)sens[pidx];
          cache[vidx] = weight;
        }
      }
      if (!(denominator > 0)) continue;
      const F inv = 1 / denominator;
      for (int64_t info = ev.info_begin; info < ev.info_end; ++info) {
        const int x = pix[2 * info], y = pix[2 * info + 1];
        const int64_t pidx = x + (int64_t)g.nc * y;
        for (int iz = ev.plane_begin; iz < ev.plane_end; ++iz) {
          const int64_t vidx = pidx + (int64_t)iz * n_pixels;
          out[vidx] += cache[vidx] * inv;
        }
      }
    }
    std::copy(out.begin(), out.end(), rho);
  }
  if (stats) *stats = st;
}

}  // namespace

extern "C" {

int64_t hyb_soa_from_matrix(const hyb_setup* s, int32_t n_detectors, const float* centers_xy,
                            int64_t n_elements, const uint16_t* lor_a, const uint16_t* lor_b,
                            const uint16_t* px, const uint16_t* py, const uint32_t* hits,
                            uint32_t n_emissions, const int16_t* inactive, int32_t n_inactive,
                            float* seg, int16_t* pix, float* pos, float* w, int64_t* lbeg,
                            int64_t* lend) {
  if (n_detectors <= 0 || n_elements <= 0) return -1;
  const int64_t n_lors = lor_index(n_detectors, 0);
  struct El {
    int16_t first, second, x, y;
    uint32_t hits;
  };
  std::vector<El> el(n_elements);
  for (int64_t i = 0; i < n_elements; ++i) {
    const int16_t a = (int16_t)lor_a[i], b = (int16_t)lor_b[i];
    el[i] = El{std::max(a, b), std::min(a, b), (int16_t)px[i], (int16_t)py[i], hits[i]};
    if (lor_index(el[i].first, el[i].second) >= n_lors) return -1;
  }
  // SortByLORNPositionNPixel (sparse_matrix.h:585-593), position 0
  std::sort(el.begin(), el.end(), [](const El& a, const El& b) {
    if (a.first != b.first) return a.first < b.first;
    if (a.second != b.second) return a.second < b.second;
    if (a.y != b.y) return a.y < b.y;
    return a.x < b.x;
  });
  std::vector<char> off(n_detectors > 0 ? 65536 : 1, 0);
  for (int32_t i = 0; i < n_inactive; ++i) off[(uint16_t)inactive[i]] = 1;
  std::fill(lbeg, lbeg + n_lors, 0);
  std::fill(lend, lend + n_lors, 0);
  int64_t cur = -1, index = 0;
  for (const El& e : el) {
    const int64_t li = lor_index(e.first, e.second);
    if (li != cur) {
      if (cur >= 0) lend[cur] = index;
      cur = li;
      lbeg[cur] = index;
    }
    if (n_inactive > 0 && (off[(uint16_t)e.first] || off[(uint16_t)e.second])) continue;
    pix[2 * index] = e.x;
    pix[2 * index + 1] = e.y;
    w[index] = (float)e.hits / (float)n_emissions;
    ++index;
  }
  lend[cur] = index;
  // per LOR: segment between the detector centres, positions, sort by position
  const Grid g(s);
  std::vector<int64_t> indices;
  std::vector<int16_t> sp;
  std::vector<float> sw, spos;
  for (int64_t first = 0; first < n_detectors; ++first) {
    for (int64_t second = 0; second <= first; ++second) {
      const int64_t li = lor_index(first, second);
      make_segment(centers_xy[2 * second], centers_xy[2 * second + 1], centers_xy[2 * first],
                   centers_xy[2 * first + 1], seg + li * kSeg);
      const float* sg = seg + li * kSeg;
      const int64_t b = lbeg[li], e = lend[li], n = e - b;
      if (!n) continue;
      indices.resize(n);
      for (int64_t i = 0; i < n; ++i) {
        const int64_t k = b + i;
        const float cx = g.cx(pix[2 * k]), cy = g.cy(pix[2 * k + 1]);
        // projection_scaled (line_segment.h:56)
        pos[k] = ((cx - sg[0]) * sg[6] + (cy - sg[1]) * sg[7]) / sg[8];
        indices[i] = k;
      }
      std::sort(indices.begin(), indices.end(),
                [pos](const int64_t a, const int64_t c) { return pos[a] < pos[c]; });
      sp.resize(2 * n);
      sw.resize(n);
      spos.resize(n);
      for (int64_t i = 0; i < n; ++i) {
        sp[2 * i] = pix[2 * indices[i]];
        sp[2 * i + 1] = pix[2 * indices[i] + 1];
        sw[i] = w[indices[i]];
        spos[i] = pos[indices[i]];
      }
      std::memcpy(pix + 2 * b, sp.data(), sizeof(int16_t) * 2 * n);
      std::memcpy(w + b, sw.data(), sizeof(float) * n);
      std::memcpy(pos + b, spos.data(), sizeof(float) * n);
    }
  }
  return index;
}

void hyb_sensitivity(const hyb_setup* s, int64_t n_infos, const int16_t* pix, const float* w,
                     float* sens) {
  const int64_t n_pixels = (int64_t)s->n_columns * s->n_rows;
  std::fill(sens, sens + n_pixels, 0.0f);
  for (int64_t i = 0; i < n_infos; ++i)
    sens[pix[2 * i] + (int64_t)s->n_columns * pix[2 * i + 1]] += w[i];
}

void hyb_normalize(int64_t n_infos, const hyb_setup* s, const int16_t* pix, float* w,
                   const float* sens) {
  for (int64_t i = 0; i < n_infos; ++i)
    w[i] /= sens[pix[2 * i] + (int64_t)s->n_columns * pix[2 * i + 1]];
}

int64_t hyb_frame_events(const hyb_setup* s, int64_t n_lors, const float* seg,
                         const int16_t* pix, const float* pos, const float* w,
                         const int64_t* lbeg, const int64_t* lend, int64_t n_infos,
                         int64_t n_events, const int16_t* first, const int16_t* second,
                         const float* z_up, const float* z_dn, const float* dl,
                         hyb_frame* frames, uint8_t* keep) {
  const Grid g(s);
  const Kernel<float> kernel(s->sigma_z, s->sigma_dl);
  int64_t n_kept = 0;
  for (int64_t i = 0; i < n_events; ++i) {
    keep[i] = 0;
    // the reference reads the pair as stored (Response(istream), no reordering)
    const int64_t li = lor_index(first[i], second[i]);
    if (first[i] < 0 || second[i] < 0 || li < 0 || li >= n_lors) continue;
    const float* sg = seg + li * kSeg;
    const float R = sg[8] / 2;
    // Strip::Response::calculate_tan_y_z (src/2d/strip/response.h:22-37)
    const float zu = z_up[i], zd = z_dn[i], d = dl[i];
    const float tan = (zu - zd) / (2 * R);
    const float up = -0.5f * (d / std::sqrt(1 + tan * tan));
    const float right = 0.5f * (zu + zd + (2 * up * tan));
    // GaussianKernel::ellipse_bb (gaussian_kernel.h:108-128)
    const float tan_sq = tan * tan;
    const float sec = std::sqrt(1 + tan * tan);
    const float A = 4 * sec * sec * kernel.ipdl + 2 * tan_sq * kernel.ipz;
    const float B = -4 * tan * kernel.ipz;
    const float C = 2 * kernel.ipz;
    const float B_2 = (B / 2) * (B / 2);
    const float half_up = 3 / std::sqrt(A - (B_2 / C));
    const float half_right = 3 / std::sqrt(C - (B_2 / A));
    const float z_l = right - half_right, z_r = right + half_right;
    const int16_t pb = std::max((int16_t)0, g.plane(z_l));
    const int16_t pe = std::min((int16_t)(g.plane(z_r) + 1), (int16_t)g.np);
    const float y_up = up + half_up, y_dn = up - half_up;
    const float t_up = (y_up + R) / (2 * R);
    const float t_dn = (y_dn + R) / (2 * R);
    const float* pb_ptr = pos + lbeg[li];
    const float* pe_ptr = pos + lend[li];
    // upper_bound(t_up) + 1 and lower_bound(t_dn) (reconstruction.h:130-145);
    // the "+ 1" end can reach one info past the LOR's own range; at the very
    // end of the arrays it is clamped (the reference would read past them).
    int64_t ie = (std::upper_bound(pb_ptr, pe_ptr, t_up) - pos) + 1;
    const int64_t ib = std::lower_bound(pb_ptr, pe_ptr, t_dn) - pos;
    if (ie > n_infos) ie = n_infos;
    hyb_frame f{(int32_t)li, pb, pe, ib, ie, up, right, tan, sec};
    // bb_intersects_grid_with_positive_weight (reconstruction.h:151-161)
    if (f.plane_end <= 0 || f.plane_begin >= g.np) continue;
    bool ok = false;
    for (int64_t k = ib; k < ie && !ok; ++k)
      ok = g.contains(pix[2 * k], pix[2 * k + 1]) && w[k] > 0;
    if (!ok) continue;
    keep[i] = 1;
    frames[n_kept++] = f;
  }
  return n_kept;
}

void hyb_mlem_f32(const hyb_setup* s, const float* seg, const int16_t* pix, const float* w,
                  const float* sens, const hyb_frame* frames, int64_t n_frames, float* rho,
                  int32_t n_iter, hyb_stats* stats) {
  mlem<float>(s, seg, pix, w, sens, frames, n_frames, rho, n_iter, stats);
}

void hyb_mlem_f64(const hyb_setup* s, const float* seg, const int16_t* pix, const float* w,
                  const float* sens, const hyb_frame* frames, int64_t n_frames, double* rho,
                  int32_t n_iter, hyb_stats* stats) {
  mlem<double>(s, seg, pix, w, sens, frames, n_frames, rho, n_iter, stats);
}

float hyb_kernel_f32(const hyb_setup* s, float right, float up, float tan, float sec, float R,
                     float z, float up_pixel) {
  const Kernel<float> kernel(s->sigma_z, s->sigma_dl);
  return kernel.normalized(right, up, tan, sec, R, s->length, z, up_pixel);
}

}  // extern "C"
