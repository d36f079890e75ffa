// Seeded synthetic list-mode events for the strip scanner, one definition for
// the host generator (strip_phantom.cpp, OpenMP) and the device generator
// (strip_phantom_gpu.cu, one thread per event).  Follows the reference's
// phantom Monte Carlo semantics -- region chosen by area x activity
// (phantom.h:120-133), point uniform in the region, rejected when an
// earlier-listed region contains it (phantom.h:193-204), detection when both
// hits land on the strips (scanner.h:196-214, to_projection_space_tan
// scanner.h:107-113), Gaussian smearing after detection (scanner.h:257-267)
// -- with tan(theta) drawn uniformly over the strip acceptance (or, on
// request, from a uniform angle as phantom.h:213 does), and a counter-based
// RNG so event i is a pure function of (seed, i): Philox-4x32-10 (Salmon et
// al., SC'11).  Both builds evaluate the same binary64 expressions without
// contraction (host -ffp-contract=off, device -fmad=false); they can differ
// only where the math library's log / sin / cos / tan round differently.
#pragma once

#include <math.h>
#include <stdint.h>

#include <vector>

#include "stripmlem.h"

#ifdef __CUDACC__
#define STRIP_HD __host__ __device__ __forceinline__
#else
#define STRIP_HD inline
#endif

namespace stripgen {

constexpr double kPi = 3.14159265358979323846;
constexpr uint32_t kMaxAttempts = 1u << 20;

// Philox-4x32 with 10 rounds: multipliers 0xD2511F53, 0xCD9E8D57 and Weyl key
// increments 0x9E3779B9, 0xBB67AE85 (the published constants).
STRIP_HD void philox(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
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

// (0, 1), never 0 or 1
STRIP_HD double u01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

// A phantom region (phantom.h:32-95): ellipse (axes a, b rotated by the
// angle whose cosine / sine are c, s), rectangle (half sides a, b, not
// rotated) or point; w = its weight, area x intensity (intensity alone for a
// point).
struct Region {
  int kind;  // STRIP_REGION_ELLIPSE / _RECTANGLE / _POINT
  double z, y, a, b, c, s, w;
  STRIP_HD bool contains(double pz, double py) const {
    const double dz = pz - z, dy = py - y;
    if (kind == STRIP_REGION_RECTANGLE) return fabs(dz) <= a && fabs(dy) <= b;
    if (kind == STRIP_REGION_POINT) return pz == z && py == y;
    const double u = dz * c + dy * s, v = -dz * s + dy * c;
    return (u * u) / (a * a) + (v * v) / (b * b) <= 1.0;
  }
  // a point uniform in the region from two uniforms
  STRIP_HD void point(double u1, double u2, double& pz, double& py) const {
    if (kind == STRIP_REGION_RECTANGLE) {
      pz = z + a * (2.0 * u1 - 1.0);
      py = y + b * (2.0 * u2 - 1.0);
    } else if (kind == STRIP_REGION_POINT) {
      pz = z;
      py = y;
    } else {
      const double rad = sqrt(u1), phi = 2.0 * kPi * u2;
      const double lu = a * rad * cos(phi), lv = b * rad * sin(phi);
      pz = z + lu * c - lv * s;
      py = y + lu * s + lv * c;
    }
  }
};

struct Params {
  double R, hL, tmax, sigma_z, sigma_dl;
  uint32_t k0, k1;
  int uniform_angle;
};

// Emission from regions: r = region by cdf, point uniform in it; unless the
// regions are additive, rejected when an earlier region covers the point
// (phantom.h:193-204).
struct RegionEmitter {
  const Region* reg;
  const double* cdf;
  int n;
  int additive;
  STRIP_HD bool operator()(const uint32_t* c, double& pz, double& py) const {
    const double ur = u01(c[0]);
    int r = 0;
    while (r < n - 1 && ur > cdf[r]) ++r;
    reg[r].point(u01(c[1]), u01(c[2]), pz, py);
    if (additive) return true;
    for (int j = 0; j < r; ++j)
      if (reg[j].contains(pz, py)) return false;
    return true;
  }
};

// Emission from an activity image: pixel j = the first with cdf[j] >= u,
// point uniform in the pixel.
struct ImageEmitter {
  const double* cdf;
  const float* rho;
  int64_t np;
  int nz;
  double tl_y, tl_z, ph, pw;
  STRIP_HD bool operator()(const uint32_t* c, double& pz, double& py) const {
    const double ur = u01(c[0]);
    int64_t lo = 0, hi = np;  // lower_bound
    while (lo < hi) {
      const int64_t mid = lo + ((hi - lo) >> 1);
      if (cdf[mid] < ur) lo = mid + 1; else hi = mid;
    }
    int64_t j = lo < np ? lo : np - 1;
    while (j > 0 && rho[j] <= 0.0f) --j;  // ur rounded past the end
    const int64_t iy = j / nz, iz = j - iy * nz;
    pz = tl_z + ((double)iz + u01(c[1])) * pw;
    py = tl_y - ((double)iy + u01(c[2])) * ph;
    return true;
  }
};

// Event i: attempts (i, attempt) until an emission is detected, then the
// smearing block (i, 0xFFFFFFFF, 1).  Returns kDetected, or kFailed when
// kMaxAttempts attempts all failed.  With one_emission, event i is a single
// emission (attempts only until a point is emitted, phantom.h:193-214) that
// may go undetected (kEmitted).  on_emit(pz, py) sees every emission.
enum EventStatus { kFailed = 0, kDetected = 1, kEmitted = 2 };

struct NoEmitHook {
  STRIP_HD void operator()(double, double) const {}
};

template <class Emit, class Hook = NoEmitHook>
STRIP_HD int event(const Params& p, uint64_t i, const Emit& emit, float& z_u,
                   float& z_d, float& dl, bool one_emission = false,
                   double* origin = nullptr, const Hook& on_emit = Hook()) {
  const uint32_t ilo = (uint32_t)i, ihi = (uint32_t)(i >> 32);
  double pz = 0, py = 0, t = 0;
  bool ok = false, emitted = false;
  for (uint32_t att = 0; att < kMaxAttempts && !ok; ++att) {
    uint32_t c[4] = {ilo, ihi, att, 0u};
    philox(c, p.k0, p.k1);
    if (!emit(c, pz, py)) continue;
    emitted = true;
    on_emit(pz, py);
    t = p.uniform_angle ? tan(kPi * (u01(c[3]) - 0.5))
                        : p.tmax * (2.0 * u01(c[3]) - 1.0);
    const double zu = pz + (p.R - py) * t, zd = pz - (p.R + py) * t;
    ok = fabs(zu) < p.hL && fabs(zd) < p.hL;
    if (one_emission) break;
  }
  if (origin) {
    origin[0] = pz;
    origin[1] = py;
  }
  if (!ok) return emitted && one_emission ? kEmitted : kFailed;
  uint32_t c[4] = {ilo, ihi, 0xFFFFFFFFu, 1u};
  philox(c, p.k0, p.k1);
  // Box-Muller: two normal pairs from four uniforms
  const double r0 = sqrt(-2.0 * log(u01(c[0]))), a0 = 2.0 * kPi * u01(c[1]);
  const double r1 = sqrt(-2.0 * log(u01(c[2]))), a1 = 2.0 * kPi * u01(c[3]);
  const double n0 = r0 * cos(a0), n1 = r0 * sin(a0), n2 = r1 * cos(a1);
  const double zu = pz + (p.R - py) * t;
  const double zd = pz - (p.R + py) * t;
  const double d = -2.0 * py * sqrt(t * t + 1.0);
  z_u = (float)(zu + p.sigma_z * n0);
  z_d = (float)(zd + p.sigma_z * n1);
  dl = (float)(d + p.sigma_dl * n2);
  return kDetected;
}

// Host-side set-up shared by both generators (strip_phantom.cpp).
Params make_params(const strip_geometry* g, uint64_t seed, int uniform_angle);
bool make_regions(const strip_ellipse* el, int n_el, std::vector<Region>& reg,
                  std::vector<double>& cdf);
bool make_regions(const strip_region* rg, int n_rg, std::vector<Region>& reg,
                  std::vector<double>& cdf);
bool make_image_cdf(const strip_geometry* g, const float* rho,
                    std::vector<double>& cdf);
ImageEmitter image_emitter(const strip_geometry* g, const double* cdf,
                           const float* rho);
bool valid_image_geometry(const strip_geometry* g);

}  // namespace stripgen
