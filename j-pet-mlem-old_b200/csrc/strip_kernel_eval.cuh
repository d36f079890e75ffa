// Kernel values of the strip TOF model, factored by pixel row.
//
// For an event (y, tan, sec) and a pixel at distance (dz, dy) the reference
// evaluates (gaussian_kernel.h:51-79)
//     K = kc / sqrt(a'S a) * exp(-b'S b / 2),    S = diag(ipsz, ipsz, ipsdl)
//     a = (-(yp-R) sec^2, -(yp+R) sec^2, -2 yp sec tan),  yp = dy + y
//     b = (dz - dy tan, dz - dy tan, -2 dy sec)
// a depends on the row only, and b'S b = 2 ipsz (dz - dy tan)^2 + ipsdl b_r^2,
// so per row we keep pref = kc / sqrt(a'S a) and the constant part of the
// exponent, and per pixel K = pref * 2^(c1 * t^2 + c0) with t = dz - dy tan.
// AnalyticKernel (analytic_kernel.h:28-62) adds the o-vector: norm and b'S a
// become linear in t, so it keeps three row constants more and needs a
// reciprocal and a reciprocal square root per pixel.
#pragma once

namespace stripmlem {

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr float kLog2e = 1.4426950408889634f;

// Packed binary32 pairs: sm_100's f32x2 arithmetic issues one instruction for
// two multiplies or FMAs (each lane rounded like its scalar form).
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 unpack2(f32x2 v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// Kernel constants for given sigmas (the sigmas of the model, which may differ
// from the geometry's sigmas that fix the pixel sets).
struct KernelF {
  float ipsz, ipsdl, kc;
  float c1;      // -log2(e) * ipsz
  // Gaussian recurrence along a row of pixel pitch pw, t -> t + pw:
  //   E(t + pw) = E(t) * R(t),  R(t) = 2^(r1 t + r0),  R(t + pw) = R(t) * q
  float r1, r0;  // 2 c1 pw, c1 pw^2
  float q;       // 2^(2 c1 pw^2)
  float q3, q4;  // q^3, q^4: the pixel-pair form of the recurrence
  float lg2kc;   // log2(kc)
};

// The Gaussian along a run, two pixels per step: with R_k = R_0 q^k,
//   (E_2i+2, E_2i+3) = (E_2i, E_2i+1) * S_i,  S_i = (R_2i R_2i+1, R_2i+1 R_2i+2),
//   S_i+1 = S_i * q^4,  S_0 = (R_0^2 q, R_0^2 q^3).
struct PairRecurrence {
  f32x2 P, S, Q4;
  __device__ __forceinline__ PairRecurrence(const KernelF& k, float E0,
                                            float R0) {
    const float R2 = R0 * R0;
    P = pack2(E0, E0 * R0);
    S = pack2(R2 * k.q, R2 * k.q3);
    Q4 = pack2(k.q4, k.q4);
  }
  __device__ __forceinline__ void step() {
    P = mul2(P, S);
    S = mul2(S, Q4);
  }
};

// GaussianKernel, one row.
struct GaussRow {
  float pref, c0, dytan;
  __device__ __forceinline__ void init(const KernelF& k, float R, float y,
                                       float tan, float sec, float dy) {
    const float sec_sq = sec * sec;
    const float yp = dy + y;
    const float ap = -(yp - R) * sec_sq;
    const float aq = -(yp + R) * sec_sq;
    const float ar = -2.0f * yp * sec * tan;
    const float norm = k.ipsz * (ap * ap + aq * aq) + k.ipsdl * (ar * ar);
    const float br = -2.0f * dy * sec;
    pref = k.kc * rsqrt_approx(norm);
    c0 = -0.5f * kLog2e * k.ipsdl * (br * br);
    dytan = dy * tan;
  }
  __device__ __forceinline__ float eval(const KernelF& k, float dz) const {
    const float t = dz - dytan;
    return pref * ex2_approx(fmaf(k.c1, t * t, c0));
  }
};

// GaussianKernel row constants from three per-event ones.  With yp = dy + y,
//   a'Sa = ipsz sec^4 ((yp - R)^2 + (yp + R)^2) + ipsdl (2 yp sec tan)^2
//        = na yp^2 + nb,    na = 2 ipsz sec^4 + 4 ipsdl sec^2 tan^2,
//                           nb = 2 ipsz sec^4 R^2,
// and the row's part of the exponent, -log2(e)/2 * ipsdl (2 dy sec)^2, is
// cd dy^2 with cd = -2 log2(e) ipsdl sec^2 (the same values as GaussRow up
// to rounding, for a third of its arithmetic).
struct GaussEvent {
  float na, nb, cd;
  __device__ __forceinline__ void init(const KernelF& k, float R, float tan,
                                       float sec) {
    const float s2 = sec * sec, s4 = s2 * s2;
    na = 2.0f * k.ipsz * s4 + 4.0f * k.ipsdl * s2 * (tan * tan);
    nb = 2.0f * k.ipsz * s4 * (R * R);
    cd = -2.0f * kLog2e * k.ipsdl * s2;
  }
  // K and the recurrence ratio R at the run's first pixel, whose distance
  // from the event along z is t0 (so t = t0 - dy tan).
  __device__ __forceinline__ void row(const KernelF& k, float y, float tan,
                                      float dy, float t0, float& K0,
                                      float& R0) const {
    const float yp = dy + y;
    const float pref = k.kc * rsqrt_approx(fmaf(na, yp * yp, nb));
    const float t = fmaf(-dy, tan, t0);
    K0 = pref * ex2_approx(fmaf(k.c1 * t, t, cd * dy * dy));
    R0 = ex2_approx(fmaf(k.r1, t, k.r0));
  }
};

// GaussianKernel row with the sigma derivatives of log K.  With
// N = a'Sa = ipsz a_pq + ipsdl a_r^2 (a_pq = ap^2 + aq^2) and kc ~ 1/(sz^2 sdl):
//   sz  * dlogK/dsz  = -2 + ipsz a_pq / N + 2 ipsz t^2   = fz  + 2 ipsz t^2
//   sdl * dlogK/dsdl = -1 + ipsdl a_r^2 / N + ipsdl b_r^2 = fdl
struct GaussGradRow {
  float pref, c0, dytan, fz, fdl;
  __device__ __forceinline__ void init(const KernelF& k, float R, float y,
                                       float tan, float sec, float dy) {
    const float sec_sq = sec * sec;
    const float yp = dy + y;
    const float ap = -(yp - R) * sec_sq;
    const float aq = -(yp + R) * sec_sq;
    const float ar = -2.0f * yp * sec * tan;
    const float apq = k.ipsz * (ap * ap + aq * aq);
    const float arr = k.ipsdl * (ar * ar);
    const float norm = apq + arr;
    const float br = -2.0f * dy * sec;
    const float brr = k.ipsdl * (br * br);
    pref = k.kc * rsqrt_approx(norm);
    c0 = -0.5f * kLog2e * brr;
    dytan = dy * tan;
    fz = apq / norm - 2.0f;
    fdl = arr / norm + brr - 1.0f;
  }
};

// AnalyticKernel, one row:  with t = dz - dy tan
//   norm  = a'Sa + 2 o'Sb = n0 + n1 t
//   b'Sa  = u1 t + u0
//   b'Sb  = 2 ipsz t^2 + cr
//   K     = kc / sqrt(norm) * exp(-(b'Sb - (b'Sa)^2 / norm) / 2)
struct AnalyticRow {
  float n0, n1, u0, u1, cr, dytan;
  __device__ __forceinline__ void init(const KernelF& k, float R, float y,
                                       float tan, float sec, float dy) {
    const float sec_sq = sec * sec;
    const float yp = dy + y;
    const float ap = -(yp - R) * sec_sq;
    const float aq = -(yp + R) * sec_sq;
    const float ar = -2.0f * yp * sec * tan;
    const float orr = -yp * sec * (1.0f + 2.0f * tan * tan);
    const float br = -2.0f * dy * sec;
    const float naa = k.ipsz * (ap * ap + aq * aq) + k.ipsdl * (ar * ar);
    const float v1 = k.ipsz * tan * (ap + aq);
    const float v0 = k.ipsdl * orr * br;
    n0 = naa + 2.0f * v0;
    n1 = 2.0f * v1;
    u1 = k.ipsz * (ap + aq);
    u0 = k.ipsdl * br * ar;
    cr = k.ipsdl * (br * br);
    dytan = dy * tan;
  }
  __device__ __forceinline__ float eval(const KernelF& k, float dz) const {
    return eval_t(k, dz - dytan);
  }
  __device__ __forceinline__ float eval_t(const KernelF& k, float t) const {
    const float norm = fmaf(n1, t, n0);
    const float bia = fmaf(u1, t, u0);
    const float bib = fmaf(2.0f * k.ipsz, t * t, cr);
    const float arg = -0.5f * kLog2e * (bib - bia * bia * rcp_approx(norm));
    return k.kc * rsqrt_approx(norm) * ex2_approx(arg);
  }
};

}  // namespace stripmlem
