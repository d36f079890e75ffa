// Host generator of seeded synthetic list-mode events (strip_generate_events,
// strip_generate_events_image in include/stripmlem.h); the per-event
// arithmetic is strip_generator.h, shared with the device generator.
#include <cmath>
#include <cstdint>
#include <vector>

#include "stripmlem.h"
#include "strip_generator.h"

namespace {

bool valid_geometry(const strip_geometry* g) {
  return g && g->radius > 0 && g->scintillator_length > 0 && g->sigma_z >= 0 &&
         g->sigma_dl >= 0;
}

template <class Emit>
int generate(const stripgen::Params& p, int64_t n, float* z_u, float* z_d,
             float* dl, const Emit& emit) {
  int bad = 0;
#pragma omp parallel for schedule(static, 4096) reduction(| : bad)
  for (int64_t i = 0; i < n; ++i)
    if (stripgen::event(p, (uint64_t)i, emit, z_u[i], z_d[i], dl[i]) !=
        stripgen::kDetected)
      bad = 1;
  return bad ? STRIP_E_INVALID : STRIP_OK;
}

}  // namespace

namespace stripgen {

Params make_params(const strip_geometry* g, uint64_t seed, int uniform_angle) {
  Params p;
  p.R = g->radius;
  p.hL = g->scintillator_length / 2.0;
  p.tmax = g->scintillator_length / (2.0 * g->radius);
  p.sigma_z = g->sigma_z;
  p.sigma_dl = g->sigma_dl;
  p.k0 = (uint32_t)seed;
  p.k1 = (uint32_t)(seed >> 32);
  p.uniform_angle = uniform_angle;
  return p;
}

// Regions and their cumulative weights (area x activity); false when an
// ellipse is invalid or the total weight is zero.
bool make_regions(const strip_region* rg, int n_rg, std::vector<Region>& reg,
                  std::vector<double>& cdf) {
  reg.resize((size_t)n_rg);
  cdf.resize((size_t)n_rg);
  double acc = 0;
  for (int i = 0; i < n_rg; ++i) {
    const strip_region& q = rg[i];
    if (!(q.intensity >= 0) || !std::isfinite(q.z) || !std::isfinite(q.y)) return false;
    Region r{};
    r.kind = q.kind;
    r.z = q.z;
    r.y = q.y;
    if (q.kind == STRIP_REGION_ELLIPSE) {
      if (!(q.a > 0) || !(q.b > 0)) return false;
      const double ang = q.angle_deg * kPi / 180.0;
      r.a = q.a;
      r.b = q.b;
      r.c = std::cos(ang);
      r.s = std::sin(ang);
      r.w = kPi * q.a * q.b * q.intensity;
    } else if (q.kind == STRIP_REGION_RECTANGLE) {
      if (!(q.a > 0) || !(q.b > 0)) return false;
      r.a = q.a;
      r.b = q.b;
      r.w = 4.0 * q.a * q.b * q.intensity;
    } else if (q.kind == STRIP_REGION_POINT) {
      r.w = q.intensity;
    } else {
      return false;
    }
    reg[i] = r;
    acc += r.w;
    cdf[i] = acc;
  }
  if (!(acc > 0)) return false;
  for (auto& c : cdf) c /= acc;
  return true;
}

bool make_regions(const strip_ellipse* el, int n_el, std::vector<Region>& reg,
                  std::vector<double>& cdf) {
  std::vector<strip_region> rg((size_t)n_el);
  for (int i = 0; i < n_el; ++i)
    rg[i] = strip_region{STRIP_REGION_ELLIPSE, 0, el[i].z, el[i].y, el[i].a,
                         el[i].b, el[i].angle_deg, el[i].activity};
  return make_regions(rg.data(), n_el, reg, cdf);
}

// Cumulative pixel weights of an activity image; false when a pixel is
// negative or not finite or the image is all zero.
bool make_image_cdf(const strip_geometry* g, const float* rho,
                    std::vector<double>& cdf) {
  const int64_t np = (int64_t)g->n_y_pixels * g->n_z_pixels;
  cdf.resize((size_t)np);
  double acc = 0;
  for (int64_t j = 0; j < np; ++j) {
    if (!(rho[j] >= 0) || !std::isfinite(rho[j])) return false;
    acc += rho[j];
    cdf[(size_t)j] = acc;
  }
  if (!(acc > 0)) return false;
  for (auto& c : cdf) c /= acc;
  return true;
}

ImageEmitter image_emitter(const strip_geometry* g, const double* cdf,
                           const float* rho) {
  ImageEmitter e;
  e.cdf = cdf;
  e.rho = rho;
  e.np = (int64_t)g->n_y_pixels * g->n_z_pixels;
  e.nz = g->n_z_pixels;
  e.tl_y = g->center_y + g->n_y_pixels * g->pixel_height / 2.0;
  e.tl_z = g->center_z - g->n_z_pixels * g->pixel_width / 2.0;
  e.ph = g->pixel_height;
  e.pw = g->pixel_width;
  return e;
}

bool valid_image_geometry(const strip_geometry* g) {
  return valid_geometry(g) && g->n_y_pixels > 0 && g->n_z_pixels > 0 &&
         g->pixel_height > 0 && g->pixel_width > 0;
}

}  // namespace stripgen

extern "C" int strip_generate_events(const strip_geometry* g,
                                     const strip_ellipse* el, int n_el,
                                     uint64_t seed, int64_t n, float* z_u,
                                     float* z_d, float* dl) {
  if (!valid_geometry(g) || !el || n_el <= 0 || n < 0 ||
      (n > 0 && (!z_u || !z_d || !dl)))
    return STRIP_E_INVALID;
  std::vector<stripgen::Region> reg;
  std::vector<double> cdf;
  if (!stripgen::make_regions(el, n_el, reg, cdf)) return STRIP_E_INVALID;
  const stripgen::RegionEmitter emit{reg.data(), cdf.data(), n_el, 0};
  return generate(stripgen::make_params(g, seed, 0), n, z_u, z_d, dl, emit);
}

extern "C" int strip_generate_events_image(const strip_geometry* g,
                                           const float* rho, uint64_t seed,
                                           int64_t n, int uniform_angle,
                                           float* z_u, float* z_d, float* dl) {
  if (!stripgen::valid_image_geometry(g) || !rho || n < 0 ||
      (n > 0 && (!z_u || !z_d || !dl)))
    return STRIP_E_INVALID;
  std::vector<double> cdf;
  if (!stripgen::make_image_cdf(g, rho, cdf)) return STRIP_E_INVALID;
  return generate(stripgen::make_params(g, seed, uniform_angle != 0), n, z_u, z_d,
                  dl, stripgen::image_emitter(g, cdf.data(), rho));
}
