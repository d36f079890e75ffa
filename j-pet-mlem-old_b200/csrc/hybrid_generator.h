// Seeded synthetic responses for the 3D hybrid path, one definition for the
// host generator (OpenMP) and the device generator (one thread per response).
// Emission points are uniform in a phantom of z-cylinders, the cylinder
// chosen by volume x activity and the point rejected when an earlier-listed
// cylinder contains it (overlaps exclusive, first on top, as the reference's
// phantoms); directions are isotropic.  Each photon of the pair is taken by
// the first detector its 2D line crosses, rings inwards out (the barrel's
// inner rings have gaps between detectors), at the projection of that
// detector's centre on the line; the response is kept when both points lie
// within |z| <= L/2.  The LOR's first detector is the larger index ("up", as
// LOR<S> orders it, src/2d/barrel/lor.h:19-21), dl = l_up - l_dn of the 3D
// path lengths, and z_up, z_dn, dl are smeared with N(0, sigma_z) and
// N(0, sigma_dl) after detection (Scanner::response_w_error,
// src/3d/hybrid/scanner.h:215-225).  Response i is a pure function of
// (seed, i): Philox-4x32-10 keyed by the seed, counter (i, attempt, block).
#pragma once

#include <math.h>
#include <stdint.h>

#include "strip_generator.h"

namespace hybridgen {

constexpr int kMaxRings = 16;
constexpr int kMaxCylinders = 32;
constexpr uint32_t kMaxAttempts = 1u << 12;  // a phantom the barrel sees fails fast

struct Ring {
  int32_t first, count;  // detector index range
  double radius;         // radius of the detectors' centres
  double angle0;         // angle of the first detector's centre
};

struct Cylinder {
  double x, y, z, r, hl, act;
};

struct Setup {
  int32_t n_rings, n_cyl;
  Ring ring[kMaxRings];
  Cylinder cyl[kMaxCylinders];
  double cum[kMaxCylinders];  // cumulative volume x activity, normalised
  double L, sigma_z, sigma_dl;
};

// First detector crossed by the 2D ray p + s d (s > 0); returns its index
// and the distance s of its centre's projection, or -1.
STRIP_HD int detect(const Setup& S, const float* poly, const float* cen, double px, double py,
                    double dx, double dy, double& s_out) {
  const double nx = -dy, ny = dx;
  for (int k = 0; k < S.n_rings; ++k) {
    const Ring& rg = S.ring[k];
    const double b = px * dx + py * dy;
    const double c = px * px + py * py - rg.radius * rg.radius;
    const double disc = b * b - c;
    const double s = -b + sqrt(disc > 0 ? disc : 0.0);
    const double hx = px + s * dx, hy = py + s * dy;
    const double rel = (atan2(hy, hx) - rg.angle0) * rg.count / (2.0 * stripgen::kPi);
    const int k0 = (int)floor(rel + 0.5);
    int best = -1;
    double best_s = 1e300;
    for (int dk = -1; dk <= 1; ++dk) {
      int m = (k0 + dk) % rg.count;
      if (m < 0) m += rg.count;
      const int det = rg.first + m;
      const float* v = poly + 8 * det;
      double lo = 1e300, hi = -1e300;
      for (int q = 0; q < 4; ++q) {
        const double sd = (v[2 * q] - px) * nx + (v[2 * q + 1] - py) * ny;
        lo = sd < lo ? sd : lo;
        hi = sd > hi ? sd : hi;
      }
      const double sc = (cen[2 * det] - px) * dx + (cen[2 * det + 1] - py) * dy;
      if (lo < 0 && hi > 0 && sc > 0 && sc < best_s) {
        best = det;
        best_s = sc;
      }
    }
    if (best >= 0) {
      s_out = best_s;
      return best;
    }
  }
  return -1;
}

struct Draw {
  uint32_t v[12];
};

STRIP_HD void draw(uint64_t seed, int64_t i, uint32_t attempt, Draw& d) {
  for (uint32_t blk = 0; blk < 3; ++blk) {
    uint32_t ctr[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), attempt, blk};
    stripgen::philox(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    for (int q = 0; q < 4; ++q) d.v[4 * blk + q] = ctr[q];
  }
}

// Response i; false when no attempt was detected (never in practice).
STRIP_HD bool generate(const Setup& S, const float* poly, const float* cen, uint64_t seed,
                       int64_t i, int16_t& first, int16_t& second, float& z_up, float& z_dn,
                       float& dl) {
  using stripgen::u01;
  for (uint32_t attempt = 0; attempt < kMaxAttempts; ++attempt) {
    Draw d;
    draw(seed, i, attempt, d);
    // cylinder by volume x activity, point uniform in it
    const double uc = u01(d.v[0]);
    int c = 0;
    while (c < S.n_cyl - 1 && uc > S.cum[c]) ++c;
    const Cylinder& cy = S.cyl[c];
    const double rad = cy.r * sqrt(u01(d.v[1])), ang = 2.0 * stripgen::kPi * u01(d.v[2]);
    const double x = cy.x + rad * cos(ang), y = cy.y + rad * sin(ang);
    const double z = cy.z + cy.hl * (2.0 * u01(d.v[3]) - 1.0);
    bool covered = false;
    for (int e = 0; e < c && !covered; ++e) {
      const Cylinder& o = S.cyl[e];
      covered = (x - o.x) * (x - o.x) + (y - o.y) * (y - o.y) <= o.r * o.r &&
                fabs(z - o.z) <= o.hl;
    }
    if (covered) continue;
    // isotropic direction
    const double phi = stripgen::kPi * u01(d.v[4]);
    const double cz = 2.0 * u01(d.v[5]) - 1.0;
    const double sz = sqrt(1.0 - cz * cz);
    const double slope = cz / sz;
    const double dx = cos(phi), dy = sin(phi);
    double s1 = 0, s2 = 0;
    const int d1 = detect(S, poly, cen, x, y, dx, dy, s1);
    if (d1 < 0) continue;
    const int d2 = detect(S, poly, cen, x, y, -dx, -dy, s2);
    if (d2 < 0 || d2 == d1) continue;
    const double z1 = z + s1 * slope, z2 = z - s2 * slope;
    if (fabs(z1) > S.L / 2 || fabs(z2) > S.L / 2) continue;
    const double l1 = s1 / sz, l2 = s2 / sz;
    const bool up1 = d1 > d2;
    // three normals (Box-Muller)
    const double r1 = sqrt(-2.0 * log(u01(d.v[6]))), t1 = 2.0 * stripgen::kPi * u01(d.v[7]);
    const double r2 = sqrt(-2.0 * log(u01(d.v[8]))), t2 = 2.0 * stripgen::kPi * u01(d.v[9]);
    const double n1 = r1 * cos(t1), n2 = r1 * sin(t1), n3 = r2 * cos(t2);
    first = (int16_t)(up1 ? d1 : d2);
    second = (int16_t)(up1 ? d2 : d1);
    z_up = (float)((up1 ? z1 : z2) + S.sigma_z * n1);
    z_dn = (float)((up1 ? z2 : z1) + S.sigma_z * n2);
    dl = (float)((up1 ? l1 - l2 : l2 - l1) + S.sigma_dl * n3);
    return true;
  }
  first = second = 0;
  z_up = z_dn = dl = 0.0f;
  return false;
}

}  // namespace hybridgen
