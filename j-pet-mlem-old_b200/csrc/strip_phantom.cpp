// Seeded synthetic list-mode events for the strip scanner (strip_generate_events
// in include/stripmlem.h).  Follows the reference's phantom Monte Carlo
// semantics -- region chosen by area x activity (phantom.h:120-133), point
// uniform in the region, rejected when an earlier-listed region contains it
// (phantom.h:193-204), detection when both hits land on the strips
// (scanner.h:196-214, to_projection_space_tan scanner.h:107-113), Gaussian
// smearing after detection (scanner.h:257-267) -- with tan(theta) drawn
// uniformly over the strip acceptance instead of the reference's uniform
// angle (phantom.h:213), and a counter-based RNG so event i is a pure
// function of (seed, i): Philox-4x32-10 (Salmon et al., SC'11).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "stripmlem.h"

namespace {

struct Philox {
  static inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi,
                             uint32_t& lo) {
    const uint64_t p = (uint64_t)a * b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
  }
  // Philox-4x32 with 10 rounds: multipliers 0xD2511F53, 0xCD9E8D57 and Weyl
  // key increments 0x9E3779B9, 0xBB67AE85 (the published constants).
  static inline void block(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
      uint32_t hi0, lo0, hi1, lo1;
      mulhilo(0xD2511F53u, ctr[0], hi0, lo0);
      mulhilo(0xCD9E8D57u, ctr[2], hi1, lo1);
      const uint32_t c0 = hi1 ^ ctr[1] ^ k0;
      const uint32_t c2 = hi0 ^ ctr[3] ^ k1;
      ctr[0] = c0;
      ctr[1] = lo1;
      ctr[2] = c2;
      ctr[3] = lo0;
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
  }
};

// (0, 1), never 0 or 1
inline double u01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

struct Region {
  double z, y, a, b, c, s, w;  // centre, axes, cos/sin of the rotation, weight
  bool contains(double pz, double py) const {
    const double dz = pz - z, dy = py - y;
    const double u = dz * c + dy * s, v = -dz * s + dy * c;
    return (u * u) / (a * a) + (v * v) / (b * b) <= 1.0;
  }
};

// Detection and smearing shared by the generators.  `emit(c, pz, py)` fills
// the emission point from the first three words of the attempt's Philox block
// c and returns false when the attempt is rejected; c[3] draws tan(theta),
// uniform over the acceptance or (uniform_angle) from an angle uniform in
// (-pi/2, pi/2) as the reference's phantom generator (phantom.h:213).
template <class Emit>
int generate(const strip_geometry* g, uint64_t seed, int64_t n, float* z_u,
             float* z_d, float* dl, const Emit& emit, bool uniform_angle = false) {
  const double R = g->radius, hL = g->scintillator_length / 2.0;
  const double tmax = g->scintillator_length / (2.0 * R);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const int kMaxAttempts = 1 << 20;
  int bad = 0;

#pragma omp parallel for schedule(static, 4096) reduction(| : bad)
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t ilo = (uint32_t)i, ihi = (uint32_t)((uint64_t)i >> 32);
    double pz = 0, py = 0, t = 0;
    bool ok = false;
    for (uint32_t att = 0; att < (uint32_t)kMaxAttempts && !ok; ++att) {
      uint32_t c[4] = {ilo, ihi, att, 0u};
      Philox::block(c, k0, k1);
      if (!emit(c, pz, py)) continue;
      t = uniform_angle ? std::tan(M_PI * (u01(c[3]) - 0.5))
                        : tmax * (2.0 * u01(c[3]) - 1.0);
      const double zu = pz + (R - py) * t, zd = pz - (R + py) * t;
      ok = std::fabs(zu) < hL && std::fabs(zd) < hL;
    }
    if (!ok) {
      bad = 1;
      continue;
    }
    uint32_t c[4] = {ilo, ihi, 0xFFFFFFFFu, 1u};
    Philox::block(c, k0, k1);
    // Box-Muller: two normal pairs from four uniforms
    const double r0 = std::sqrt(-2.0 * std::log(u01(c[0]))), a0 = 2.0 * M_PI * u01(c[1]);
    const double r1 = std::sqrt(-2.0 * std::log(u01(c[2]))), a1 = 2.0 * M_PI * u01(c[3]);
    const double n0 = r0 * std::cos(a0), n1 = r0 * std::sin(a0), n2 = r1 * std::cos(a1);
    const double zu = pz + (R - py) * t;
    const double zd = pz - (R + py) * t;
    const double d = -2.0 * py * std::sqrt(t * t + 1.0);
    z_u[i] = (float)(zu + g->sigma_z * n0);
    z_d[i] = (float)(zd + g->sigma_z * n1);
    dl[i] = (float)(d + g->sigma_dl * n2);
  }
  return bad ? STRIP_E_INVALID : STRIP_OK;
}

bool valid_geometry(const strip_geometry* g) {
  return g && g->radius > 0 && g->scintillator_length > 0 && g->sigma_z >= 0 &&
         g->sigma_dl >= 0;
}

}  // namespace

extern "C" int strip_generate_events(const strip_geometry* g,
                                     const strip_ellipse* el, int n_el,
                                     uint64_t seed, int64_t n, float* z_u,
                                     float* z_d, float* dl) {
  if (!valid_geometry(g) || !el || n_el <= 0 || n < 0 ||
      (n > 0 && (!z_u || !z_d || !dl)))
    return STRIP_E_INVALID;
  std::vector<Region> reg((size_t)n_el);
  std::vector<double> cdf((size_t)n_el);
  double acc = 0;
  for (int i = 0; i < n_el; ++i) {
    if (!(el[i].a > 0) || !(el[i].b > 0) || !(el[i].activity >= 0))
      return STRIP_E_INVALID;
    const double ang = el[i].angle_deg * M_PI / 180.0;
    reg[i] = Region{el[i].z, el[i].y, el[i].a, el[i].b, std::cos(ang),
                    std::sin(ang), M_PI * el[i].a * el[i].b * el[i].activity};
    acc += reg[i].w;
    cdf[i] = acc;
  }
  if (!(acc > 0)) return STRIP_E_INVALID;
  for (auto& c : cdf) c /= acc;
  return generate(g, seed, n, z_u, z_d, dl,
                  [&](const uint32_t* c, double& pz, double& py) {
                    const double ur = u01(c[0]);
                    int r = 0;
                    while (r < n_el - 1 && ur > cdf[r]) ++r;
                    const Region& q = reg[r];
                    const double rad = std::sqrt(u01(c[1])), phi = 2.0 * M_PI * u01(c[2]);
                    const double lu = q.a * rad * std::cos(phi), lv = q.b * rad * std::sin(phi);
                    pz = q.z + lu * q.c - lv * q.s;
                    py = q.y + lu * q.s + lv * q.c;
                    for (int j = 0; j < r; ++j)
                      if (reg[j].contains(pz, py)) return false;
                    return true;
                  });
}

extern "C" int strip_generate_events_image(const strip_geometry* g,
                                           const float* rho, uint64_t seed,
                                           int64_t n, int uniform_angle,
                                           float* z_u, float* z_d, float* dl) {
  if (!valid_geometry(g) || !rho || g->n_y_pixels <= 0 || g->n_z_pixels <= 0 ||
      !(g->pixel_height > 0) || !(g->pixel_width > 0) || n < 0 ||
      (n > 0 && (!z_u || !z_d || !dl)))
    return STRIP_E_INVALID;
  const int64_t np = (int64_t)g->n_y_pixels * g->n_z_pixels;
  std::vector<double> cdf((size_t)np);
  double acc = 0;
  for (int64_t j = 0; j < np; ++j) {
    if (!(rho[j] >= 0) || !std::isfinite(rho[j])) return STRIP_E_INVALID;
    acc += rho[j];
    cdf[(size_t)j] = acc;
  }
  if (!(acc > 0)) return STRIP_E_INVALID;
  for (auto& c : cdf) c /= acc;
  const double tl_y = g->center_y + g->n_y_pixels * g->pixel_height / 2.0;
  const double tl_z = g->center_z - g->n_z_pixels * g->pixel_width / 2.0;
  const int nz = g->n_z_pixels;
  return generate(g, seed, n, z_u, z_d, dl,
                  [&](const uint32_t* c, double& pz, double& py) {
                    const double ur = u01(c[0]);
                    int64_t j = std::lower_bound(cdf.begin(), cdf.end(), ur) - cdf.begin();
                    if (j >= np) j = np - 1;
                    while (rho[j] <= 0) --j;  // ur rounded past the end: last non-empty pixel
                    const int64_t iy = j / nz, iz = j - iy * nz;
                    pz = tl_z + ((double)iz + u01(c[1])) * g->pixel_width;
                    py = tl_y - ((double)iy + u01(c[2])) * g->pixel_height;
                    return true;
                  },
                  uniform_angle != 0);
}
