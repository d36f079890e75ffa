/*
 * TEST INFRASTRUCTURE ONLY -- seeded synthetic list-mode events for the
 * benchmark's CPU (reference) arm and for checking the product's generator.
 *
 * The benchmark workload is defined by a counter-based generator: event i is
 * a pure function of (seed, i).  The product library generates it on the GPU
 * or on the host; the reference arm must produce the same events without
 * loading the product library, so this file states the same definition again
 * in plain C (compiled, like the product's host generator, with
 * -ffp-contract=off and glibc's libm, so the events are bit-identical).
 *
 * Definition (the reference's phantom Monte Carlo semantics, with a uniform
 * tan(theta) over the acceptance):
 *   - Random numbers: Philox-4x32 with 10 rounds (Salmon, Moraes, Dror, Shaw,
 *     "Parallel random numbers: as easy as 1, 2, 3", SC'11), key = the 64-bit
 *     seed, counter = (i low, i high, attempt, 0); uniforms (x + 0.5) / 2^32.
 *   - Emission: ellipse chosen by area x activity (src/2d/geometry/
 *     phantom.h:120-133), point uniform in it (radius sqrt(u)), rejected when
 *     an earlier-listed ellipse contains it (phantom.h:193-204).
 *   - Direction: tan(theta) uniform in (-L/2R, L/2R); detected when both hits
 *     lie strictly inside the strips (src/2d/strip/scanner.h:196-214).
 *   - Smearing after detection (scanner.h:257-267): counter (i low, i high,
 *     0xFFFFFFFF, 1), Box-Muller normals n0, n1, n2; z_u += sigma_z n0,
 *     z_d += sigma_z n1, dl = -2 y sqrt(1 + tan^2) + sigma_dl n2.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "strip_oracle.h"

#define ORC_PI 3.14159265358979323846
#define ORC_MAX_ATTEMPTS (1u << 20)

static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (uint32_t)p1;
    c[3] = (uint32_t)p0;
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

static double unit_open(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

typedef struct {
  double z, y, a, b, cs, sn;
} orc_ellipse_t;

static int inside(const orc_ellipse_t* e, double pz, double py) {
  const double dz = pz - e->z, dy = py - e->y;
  const double u = dz * e->cs + dy * e->sn, v = -dz * e->sn + dy * e->cs;
  return (u * u) / (e->a * e->a) + (v * v) / (e->b * e->b) <= 1.0;
}

int orc_generate_events(const orc_geometry* g, const double* ellipses,
                        int n_ellipses, uint64_t seed, int64_t n, float* z_u,
                        float* z_d, float* dl) {
  if (!g || !ellipses || n_ellipses <= 0 || n < 0 || !(g->radius > 0) ||
      !(g->scintillator_length > 0))
    return -1;
  orc_ellipse_t* el = (orc_ellipse_t*)malloc(sizeof(orc_ellipse_t) * (size_t)n_ellipses);
  double* cdf = (double*)malloc(sizeof(double) * (size_t)n_ellipses);
  if (!el || !cdf) {
    free(el);
    free(cdf);
    return -1;
  }
  double total = 0;
  for (int k = 0; k < n_ellipses; ++k) {
    const double* q = ellipses + 6 * k;  /* z, y, a, b, angle (deg), activity */
    const double ang = q[4] * ORC_PI / 180.0;
    el[k].z = q[0];
    el[k].y = q[1];
    el[k].a = q[2];
    el[k].b = q[3];
    el[k].cs = cos(ang);
    el[k].sn = sin(ang);
    total += ORC_PI * q[2] * q[3] * q[5];
    cdf[k] = total;
  }
  for (int k = 0; k < n_ellipses; ++k) cdf[k] /= total;

  const double R = g->radius, half_l = g->scintillator_length / 2.0;
  const double tmax = g->scintillator_length / (2.0 * g->radius);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  int failed = 0;
#pragma omp parallel for schedule(static, 4096) reduction(| : failed)
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)((uint64_t)i >> 32);
    double pz = 0, py = 0, t = 0;
    int detected = 0;
    for (uint32_t att = 0; att < ORC_MAX_ATTEMPTS && !detected; ++att) {
      uint32_t c[4] = {lo, hi, att, 0u};
      philox4x32_10(c, k0, k1);
      const double ur = unit_open(c[0]);
      int r = 0;
      while (r < n_ellipses - 1 && ur > cdf[r]) ++r;
      const double rad = sqrt(unit_open(c[1])), phi = 2.0 * ORC_PI * unit_open(c[2]);
      const double lu = el[r].a * rad * cos(phi), lv = el[r].b * rad * sin(phi);
      pz = el[r].z + lu * el[r].cs - lv * el[r].sn;
      py = el[r].y + lu * el[r].sn + lv * el[r].cs;
      int covered = 0;
      for (int j = 0; j < r && !covered; ++j) covered = inside(&el[j], pz, py);
      if (covered) continue;
      t = tmax * (2.0 * unit_open(c[3]) - 1.0);
      const double up = pz + (R - py) * t, dn = pz - (R + py) * t;
      detected = fabs(up) < half_l && fabs(dn) < half_l;
    }
    if (!detected) {
      failed = 1;
      continue;
    }
    uint32_t c[4] = {lo, hi, 0xFFFFFFFFu, 1u};
    philox4x32_10(c, k0, k1);
    const double r0 = sqrt(-2.0 * log(unit_open(c[0]))), a0 = 2.0 * ORC_PI * unit_open(c[1]);
    const double r1 = sqrt(-2.0 * log(unit_open(c[2]))), a1 = 2.0 * ORC_PI * unit_open(c[3]);
    const double up = pz + (R - py) * t, dn = pz - (R + py) * t;
    const double d = -2.0 * py * sqrt(t * t + 1.0);
    z_u[i] = (float)(up + g->sigma_z * (r0 * cos(a0)));
    z_d[i] = (float)(dn + g->sigma_z * (r0 * sin(a0)));
    dl[i] = (float)(d + g->sigma_dl * (r1 * cos(a1)));
  }
  free(el);
  free(cdf);
  return failed ? -1 : 0;
}
