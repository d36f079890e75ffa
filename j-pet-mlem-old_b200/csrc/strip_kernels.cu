// sm_100a kernels of the strip list-mode TOF MLEM path.
//
//   k_event_boxes / k_bin_keys / k_bin_scatter   one-time binning of the events
//       into image tiles (events are iteration-invariant, so this is paid once)
//   k_tile      the hot kernel: one CTA per (tile, event chunk) work item.  The
//       tile's window of the image (tile + halo) is staged in shared memory
//       together with a shared-memory backprojection accumulator; a warp takes
//       one event at a time: (a) scans the event's clamped bounding box with the
//       exact binary32 ellipse test and evaluates the TOF kernel, (b) sums
//       K * rho (* s) into the per-event normalisation D_e (compensated or
//       binary64 per lane, binary64 across lanes), (c) scatters K / D_e into
//       the shared accumulator with shared-memory atomics, and finally flushes
//       the window to the global binary64 accumulator.
//   k_global    the same per-event work for events whose box does not fit a
//       window (global loads, global binary64 atomics).
//   k_update    (d) rho_j <- rho_j * acc_j * scale, acc_j <- 0.
//
// Reference behaviour: Reconstruction::bb_update (src/2d/strip/reconstruction.h:
// 220-298) and the warp kernel (src/2d/strip/cuda/reconstruction/
// warp_granularity.cuh:20-176).
#include "strip_internal.h"

namespace stripmlem {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ EventF shfl_event(const EventF& m, int src) {
  EventF e;
  e.tan = __shfl_sync(kFull, m.tan, src);
  e.y = __shfl_sync(kFull, m.y, src);
  e.z = __shfl_sync(kFull, m.z, src);
  e.sec = __shfl_sync(kFull, m.sec, src);
  e.A = __shfl_sync(kFull, m.A, src);
  e.B = __shfl_sync(kFull, m.B, src);
  e.C = __shfl_sync(kFull, m.C, src);
  e.tlx = __shfl_sync(kFull, m.tlx, src);
  e.tly = __shfl_sync(kFull, m.tly, src);
  e.brx = __shfl_sync(kFull, m.brx, src);
  e.bry = __shfl_sync(kFull, m.bry, src);
  return e;
}

// Per-lane accumulation of the normalisation sum.
template <int ACC>
struct Accum;
template <>
struct Accum<STRIP_ACCUM_FP32> {
  float s = 0.0f;
  __device__ __forceinline__ void add(float x) { s += x; }
  __device__ __forceinline__ double total() const { return (double)s; }
};
template <>
struct Accum<STRIP_ACCUM_KAHAN> {
  float s = 0.0f, c = 0.0f;
  __device__ __forceinline__ void add(float x) {
    const float yv = __fsub_rn(x, c);
    const float t = __fadd_rn(s, yv);
    c = __fsub_rn(__fsub_rn(t, s), yv);
    s = t;
  }
  __device__ __forceinline__ double total() const {
    return (double)s - (double)c;
  }
};
template <>
struct Accum<STRIP_ACCUM_FP64> {
  double s = 0.0;
  __device__ __forceinline__ void add(float x) { s += (double)x; }
  __device__ __forceinline__ double total() const { return s; }
};

template <int MODE>
struct RowEvalT;
template <>
struct RowEvalT<STRIP_MODE_CPU> {
  using T = GaussRow;
};
template <>
struct RowEvalT<STRIP_MODE_GPU> {
  using T = AnalyticRow;
};

// Shared-memory window of the image: w = rho (* s), acc = partial backprojection.
struct SmemWin {
  const float* w;
  float* acc;
  int wx0, wy0, WS;
  __device__ __forceinline__ float read(int ix, int iy) const {
    return w[(iy - wy0) * WS + (ix - wx0)];
  }
  __device__ __forceinline__ void add(int ix, int iy, float v) const {
    atomicAdd(acc + (iy - wy0) * WS + (ix - wx0), v);
  }
};

// The whole image in global memory.
template <int MODE>
struct GlobalWin {
  const float* rho;
  const float* sens;
  double* acc;
  int n_z;
  __device__ __forceinline__ float read(int ix, int iy) const {
    const int64_t gi = (int64_t)iy * n_z + ix;
    float v = __ldg(rho + gi);
    if (MODE == STRIP_MODE_GPU) v *= __ldg(sens + gi);
    return v;
  }
  __device__ __forceinline__ void add(int ix, int iy, float v) const {
    atomicAdd(acc + (int64_t)iy * n_z + ix, (double)v);
  }
};

// Row constants of 32 consecutive rows, one per lane, broadcast by shuffles.
template <int MODE>
struct RowPack {
  RowSet rs;
  typename RowEvalT<MODE>::T re;
};

template <int MODE>
__device__ __forceinline__ RowPack<MODE> shfl_row(const RowPack<MODE>& m,
                                                  int src) {
  RowPack<MODE> r;
  r.rs.dy = __shfl_sync(kFull, m.rs.dy, src);
  r.rs.Ady2 = __shfl_sync(kFull, m.rs.Ady2, src);
  r.rs.Bdy = __shfl_sync(kFull, m.rs.Bdy, src);
  r.re.pref = __shfl_sync(kFull, m.re.pref, src);
  r.re.c0 = __shfl_sync(kFull, m.re.c0, src);
  r.re.dytan = __shfl_sync(kFull, m.re.dytan, src);
  return r;
}
template <>
__device__ __forceinline__ RowPack<STRIP_MODE_GPU> shfl_row(
    const RowPack<STRIP_MODE_GPU>& m, int src) {
  RowPack<STRIP_MODE_GPU> r;
  r.rs.dy = __shfl_sync(kFull, m.rs.dy, src);
  r.rs.Ady2 = __shfl_sync(kFull, m.rs.Ady2, src);
  r.rs.Bdy = __shfl_sync(kFull, m.rs.Bdy, src);
  r.re.n0 = __shfl_sync(kFull, m.re.n0, src);
  r.re.n1 = __shfl_sync(kFull, m.re.n1, src);
  r.re.u0 = __shfl_sync(kFull, m.re.u0, src);
  r.re.u1 = __shfl_sync(kFull, m.re.u1, src);
  r.re.cr = __shfl_sync(kFull, m.re.cr, src);
  r.re.dytan = __shfl_sync(kFull, m.re.dytan, src);
  return r;
}

// Visits every in-ellipse pixel of event e: rows are taken 32 at a time (one
// row's constants per lane), then the warp sweeps each row's bbox columns
// with lanes side by side.  f(ix, iy, K) is called for in-ellipse pixels.
template <int MODE, class F>
__device__ __forceinline__ void for_each_pixel(const ScannerF& s,
                                               const KernelF& k,
                                               const EventF& e, int lane,
                                               F&& f) {
  for (int rb = e.tly; rb < e.bry; rb += 32) {
    RowPack<MODE> mine = {};
    const int my_row = rb + lane;
    if (my_row < e.bry) {
      mine.rs = row_set(s, e, my_row);
      mine.re.init(k, s.R, e.y, e.tan, e.sec, mine.rs.dy);
    }
    const int nr = min(32, e.bry - rb);
    for (int j = 0; j < nr; ++j) {
      const RowPack<MODE> r = shfl_row<MODE>(mine, j);
      const int iy = rb + j;
      for (int iz = e.tlx + lane; iz < e.brx; iz += 32) {
        const float dz = col_dz(s, e, iz);
        if (in_ellipse(r.rs, e.C, dz)) f(iz, iy, r.re.eval(k, dz));
      }
    }
  }
}

template <int OP, int MODE, int ACC, class Win>
__device__ __forceinline__ void process_event(const LaunchArgs& a,
                                              const EventF& e, const Win& win,
                                              int lane, int64_t pos) {
  if (OP == OP_MLEM || OP == OP_FORWARD) {
    Accum<ACC> acc;
    for_each_pixel<MODE>(a.s, a.k, e, lane, [&](int ix, int iy, float kv) {
      acc.add(kv * win.read(ix, iy));
    });
    const double D = warp_sum(acc.total());
    if (OP == OP_FORWARD) {
      if (lane == 0) a.y_out[a.perm[pos]] = D;
      return;
    }
    // reconstruction.h:290 -- an all-zero denominator contributes nothing
    if (!(D > 0.0)) return;
    const float inv = (float)(1.0 / D);
    for_each_pixel<MODE>(a.s, a.k, e, lane, [&](int ix, int iy, float kv) {
      win.add(ix, iy, kv * inv);
    });
  } else if (OP == OP_ADJOINT) {
    const float w = (float)a.w_in[a.perm[pos]];
    if (w == 0.0f) return;
    for_each_pixel<MODE>(a.s, a.k, e, lane, [&](int ix, int iy, float kv) {
      win.add(ix, iy, kv * w);
    });
  }
}

template <int OP, int MODE, int ACC>
__global__ void __launch_bounds__(kThreads) k_tile(LaunchArgs a) {
  extern __shared__ float smem[];
  const WorkItem it = a.items[blockIdx.x];
  int wx0, wy0, wx1, wy1;
  tile_window(a.t, a.s.n_z, a.s.n_y, it.tile, wx0, wy0, wx1, wy1);
  const int wxn = wx1 - wx0, wyn = wy1 - wy0, WS = a.t.WS;
  float* s_w = smem;
  float* s_acc = smem + a.t.WYmax * WS;
  constexpr bool kReads = (OP == OP_MLEM || OP == OP_FORWARD);
  constexpr bool kWrites = (OP == OP_MLEM || OP == OP_ADJOINT);
  for (int q = threadIdx.x; q < wxn * wyn; q += blockDim.x) {
    const int r = q / wxn, c = q - r * wxn;
    const int64_t gi = (int64_t)(wy0 + r) * a.s.n_z + wx0 + c;
    if (kReads) {
      float v = a.rho[gi];
      if (MODE == STRIP_MODE_GPU) v *= a.sens[gi];
      s_w[r * WS + c] = v;
    }
    if (kWrites) s_acc[r * WS + c] = 0.0f;
  }
  __syncthreads();
  const SmemWin win{s_w, s_acc, wx0, wy0, WS};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int64_t end = it.begin + it.count;
  for (int64_t base = it.begin + (int64_t)warp * 32; base < end;
       base += (int64_t)nw * 32) {
    const int64_t ei = base + lane;
    EventF mine = {};
    if (ei < end) event_setup(a.s, a.zu[ei], a.zd[ei], a.dl[ei], mine);
    const int nh = (int)min((int64_t)32, end - base);
    for (int j = 0; j < nh; ++j) {
      const EventF e = shfl_event(mine, j);
      process_event<OP, MODE, ACC>(a, e, win, lane, base + j);
    }
  }
  if (kWrites) {
    __syncthreads();
    for (int q = threadIdx.x; q < wxn * wyn; q += blockDim.x) {
      const int r = q / wxn, c = q - r * wxn;
      const float v = s_acc[r * WS + c];
      if (v != 0.0f)
        atomicAdd(a.acc + (int64_t)(wy0 + r) * a.s.n_z + wx0 + c, (double)v);
    }
  }
}

template <int OP, int MODE, int ACC>
__global__ void __launch_bounds__(kThreads) k_global(LaunchArgs a) {
  const GlobalWin<MODE> win{a.rho, a.sens, a.acc, a.s.n_z};
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwt = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t end = a.g_begin + a.g_count;
  for (int64_t base = a.g_begin + wid * 32; base < end; base += nwt * 32) {
    const int64_t ei = base + lane;
    EventF mine = {};
    if (ei < end) event_setup(a.s, a.zu[ei], a.zd[ei], a.dl[ei], mine);
    const int nh = (int)min((int64_t)32, end - base);
    for (int j = 0; j < nh; ++j) {
      const EventF e = shfl_event(mine, j);
      process_event<OP, MODE, ACC>(a, e, win, lane, base + j);
    }
  }
}

__global__ void k_event_boxes(ScannerF s, const float* zu, const float* zd,
                              const float* dl, int64_t n, int4* boxes,
                              int* max_wh, unsigned long long* n_empty) {
  int lw = 0, lh = 0;
  unsigned empty = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    EventF e;
    event_setup(s, zu[i], zd[i], dl[i], e);
    const int w = e.brx - e.tlx, h = e.bry - e.tly;
    boxes[i] = make_int4(e.tlx, e.tly, e.brx, e.bry);
    if (w <= 0 || h <= 0) {
      ++empty;
    } else {
      lw = max(lw, w);
      lh = max(lh, h);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lw = max(lw, __shfl_xor_sync(kFull, lw, o));
    lh = max(lh, __shfl_xor_sync(kFull, lh, o));
    empty += __shfl_xor_sync(kFull, empty, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(max_wh, lw);
    atomicMax(max_wh + 1, lh);
    if (empty) atomicAdd(n_empty, (unsigned long long)empty);
  }
}

// key = subset * (n_tiles + 1) + tile, tile == n_tiles for the global path,
// -1 for an empty box.
__global__ void k_bin_keys(Tiling t, int n_z, int n_y, const int4* boxes,
                           const int64_t* orig, int64_t n, int n_subsets,
                           int* keys, unsigned long long* hist) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwt = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = wid * 32; base < n; base += nwt * 32) {
    const int64_t i = base + lane;
    int key = -1;
    if (i < n) {
      const int4 b = boxes[i];
      if (b.z > b.x && b.w > b.y) {
        const int mx = (b.x + b.z) >> 1, my = (b.y + b.w) >> 1;
        int tile = (my / t.TY) * t.ntx + (mx / t.TX);
        int wx0, wy0, wx1, wy1;
        tile_window(t, n_z, n_y, tile, wx0, wy0, wx1, wy1);
        if (b.x < wx0 || b.z > wx1 || b.y < wy0 || b.w > wy1) tile = t.n_tiles;
        const int64_t e = orig ? orig[i] : i;
        key = (int)(e % n_subsets) * (t.n_tiles + 1) + tile;
      }
      keys[i] = key;
    }
    const unsigned peers = __match_any_sync(kFull, key);
    if (key >= 0 && lane == __ffs(peers) - 1)
      atomicAdd(hist + key, (unsigned long long)__popc(peers));
  }
}

__global__ void k_bin_scatter(const int* keys, int64_t n, const float* zu,
                              const float* zd, const float* dl,
                              const int64_t* orig, unsigned long long* cursor,
                              float* ozu, float* ozd, float* odl,
                              int64_t* operm) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwt = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = wid * 32; base < n; base += nwt * 32) {
    const int64_t i = base + lane;
    const int key = i < n ? keys[i] : -1;
    const unsigned peers = __match_any_sync(kFull, key);
    const int leader = __ffs(peers) - 1;
    unsigned long long p0 = 0;
    if (key >= 0 && lane == leader)
      p0 = atomicAdd(cursor + key, (unsigned long long)__popc(peers));
    p0 = __shfl_sync(kFull, p0, leader);
    if (key >= 0) {
      const int64_t p = (int64_t)p0 + __popc(peers & ((1u << lane) - 1u));
      ozu[p] = zu[i];
      ozd[p] = zd[i];
      odl[p] = dl[i];
      operm[p] = orig ? orig[i] : i;
    }
  }
}

__global__ void k_update(float* rho, double* acc, int64_t n, double scale) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    rho[j] = (float)((double)rho[j] * acc[j] * scale);
    acc[j] = 0.0;
  }
}

// Scanner::sensitivity / pixel_sensitivity (scanner.h:147-185), binary32.
__device__ float sens_point(const ScannerF& s, float px, float py) {
  const float L_plus = s.half_L + px, L_minus = s.half_L - px;
  float R_plus = s.R + py, R_minus = s.R - py;
  if (R_plus <= 0.0f) R_plus = 1.0f;
  if (R_minus <= 0.0f) R_minus = 1.0f;
  const float a = L_minus / R_minus, b = L_plus / R_plus;
  const float c = -L_plus / R_minus, d = -L_minus / R_plus;
  return 0.318309886183790672f * (atanf(fminf(a, b)) - atanf(fmaxf(c, d)));
}

__global__ void k_sensitivity(ScannerF s, int five_point, float* out) {
  const int64_t n = (int64_t)s.n_y * s.n_z;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int py = (int)(j / s.n_z), px = (int)(j - (int64_t)py * s.n_z);
    const float cz = s.tl_z_half_w + (float)px * s.pw;
    const float cy = s.tl_y_half_h - (float)py * s.ph;
    float v;
    if (five_point) {
      const float hx = s.pw / 2.0f, hy = s.ph / 2.0f;
      v = sens_point(s, cz, cy) / 3.0f + sens_point(s, cz + hx, cy + hy) / 6.0f +
          sens_point(s, cz - hx, cy - hy) / 6.0f +
          sens_point(s, cz - hx, cy + hy) / 6.0f +
          sens_point(s, cz + hx, cy - hy) / 6.0f;
    } else {
      v = sens_point(s, cz, cy);
    }
    out[j] = v;
  }
}

// Pixel-set parity: one warp per event, the same enumeration as k_tile.
__global__ void k_debug_sets(ScannerF s, const float* zu, const float* zd,
                             const float* dl, int64_t n, int32_t* n_bb,
                             int32_t* n_in, uint64_t* digest) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwt = ((int64_t)gridDim.x * blockDim.x) >> 5;
  KernelF k{s.ipsz, s.ipsdl, s.kc, -kLog2e * s.ipsz};
  for (int64_t i = wid; i < n; i += nwt) {
    EventF e;
    event_setup(s, zu[i], zd[i], dl[i], e);
    unsigned cnt = 0;
    unsigned long long h = 0;
    for_each_pixel<STRIP_MODE_CPU>(s, k, e, lane, [&](int ix, int iy, float) {
      ++cnt;
      h += mix64((uint64_t)((int64_t)iy * s.n_z + ix) + 1u);
    });
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cnt += __shfl_xor_sync(kFull, cnt, o);
      h += __shfl_xor_sync(kFull, h, o);
    }
    if (lane == 0) {
      const int w = e.brx - e.tlx, hh = e.bry - e.tly;
      if (n_bb) n_bb[i] = (w > 0 && hh > 0) ? w * hh : 0;
      if (n_in) n_in[i] = (int32_t)cnt;
      if (digest) digest[i] = h;
    }
  }
}

// Work totals over binned events (same enumeration as k_tile).
__global__ void k_count_work(ScannerF s, const float* zu, const float* zd,
                             const float* dl, int64_t n,
                             unsigned long long* out) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwt = ((int64_t)gridDim.x * blockDim.x) >> 5;
  KernelF k{s.ipsz, s.ipsdl, s.kc, -kLog2e * s.ipsz};
  unsigned long long bb = 0, in = 0, ne = 0;
  for (int64_t i = wid; i < n; i += nwt) {
    EventF e;
    event_setup(s, zu[i], zd[i], dl[i], e);
    unsigned cnt = 0;
    for_each_pixel<STRIP_MODE_CPU>(s, k, e, lane,
                                   [&](int, int, float) { ++cnt; });
    const int w = e.brx - e.tlx, h = e.bry - e.tly;
    if (lane == 0 && w > 0 && h > 0) bb += (unsigned long long)w * h;
    in += cnt;
    const unsigned tot = __reduce_add_sync(kFull, cnt);
    if (lane == 0 && tot > 0) ++ne;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) in += __shfl_xor_sync(kFull, in, o);
  if (lane == 0) {
    atomicAdd(out, bb);
    atomicAdd(out + 1, in);
    atomicAdd(out + 2, ne);
  }
}

__global__ void k_scale_copy(const double* acc, const float* sens, double* out,
                             int64_t n) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    out[j] = sens ? acc[j] * (double)sens[j] : acc[j];
}

// Binary32 FMA throughput probe: 8 independent register-resident FMA chains
// per thread; 2 * 8 * 16 * iters flops per thread.
__global__ void __launch_bounds__(512) k_fma_peak(float* out, int iters, float a,
                                                  float b) {
  float x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = (float)(threadIdx.x + j) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = fmaf(x[j], a, b);
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

int grid_for(int64_t n, int per_block = kThreads, int cap = 148 * 16) {
  int64_t g = (n + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

template <int OP, int MODE, int ACC>
cudaError_t launch_tile_t(const LaunchArgs& a, cudaStream_t st) {
  auto fn = k_tile<OP, MODE, ACC>;
  cudaError_t err = cudaFuncSetAttribute(
      fn, cudaFuncAttributeMaxDynamicSharedMemorySize, a.t.smem_bytes);
  if (err != cudaSuccess) return err;
  fn<<<a.n_items, kThreads, a.t.smem_bytes, st>>>(a);
  return cudaGetLastError();
}

template <int OP, int MODE, int ACC>
cudaError_t launch_global_t(const LaunchArgs& a, cudaStream_t st) {
  const int grid = grid_for(a.g_count, 8 * 32);
  k_global<OP, MODE, ACC><<<grid, kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

#define STRIP_DISPATCH(FN, op, mode, accum, a, st)                         \
  do {                                                                     \
    if ((mode) == STRIP_MODE_CPU) {                                        \
      if ((accum) == STRIP_ACCUM_FP32)                                     \
        return FN<op, STRIP_MODE_CPU, STRIP_ACCUM_FP32>(a, st);            \
      if ((accum) == STRIP_ACCUM_FP64)                                     \
        return FN<op, STRIP_MODE_CPU, STRIP_ACCUM_FP64>(a, st);            \
      return FN<op, STRIP_MODE_CPU, STRIP_ACCUM_KAHAN>(a, st);             \
    }                                                                      \
    if ((accum) == STRIP_ACCUM_FP32)                                       \
      return FN<op, STRIP_MODE_GPU, STRIP_ACCUM_FP32>(a, st);              \
    if ((accum) == STRIP_ACCUM_FP64)                                       \
      return FN<op, STRIP_MODE_GPU, STRIP_ACCUM_FP64>(a, st);              \
    return FN<op, STRIP_MODE_GPU, STRIP_ACCUM_KAHAN>(a, st);               \
  } while (0)

cudaError_t launch_tile(int op, int mode, int accum, const LaunchArgs& a,
                        cudaStream_t st) {
  if (a.n_items <= 0) return cudaSuccess;
  switch (op) {
    case OP_MLEM:
      STRIP_DISPATCH(launch_tile_t, OP_MLEM, mode, accum, a, st);
    case OP_FORWARD:
      STRIP_DISPATCH(launch_tile_t, OP_FORWARD, mode, accum, a, st);
    case OP_ADJOINT:
      STRIP_DISPATCH(launch_tile_t, OP_ADJOINT, mode, accum, a, st);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_global(int op, int mode, int accum, const LaunchArgs& a,
                          cudaStream_t st) {
  if (a.g_count <= 0) return cudaSuccess;
  switch (op) {
    case OP_MLEM:
      STRIP_DISPATCH(launch_global_t, OP_MLEM, mode, accum, a, st);
    case OP_FORWARD:
      STRIP_DISPATCH(launch_global_t, OP_FORWARD, mode, accum, a, st);
    case OP_ADJOINT:
      STRIP_DISPATCH(launch_global_t, OP_ADJOINT, mode, accum, a, st);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_event_boxes(const ScannerF& s, const float* zu,
                               const float* zd, const float* dl, int64_t n,
                               int4* boxes, int* max_wh,
                               unsigned long long* n_empty, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_event_boxes<<<grid_for(n), kThreads, 0, st>>>(s, zu, zd, dl, n, boxes,
                                                  max_wh, n_empty);
  return cudaGetLastError();
}

cudaError_t launch_bin_keys(const Tiling& t, int n_z, int n_y,
                            const int4* boxes, const int64_t* orig, int64_t n,
                            int n_subsets, int* keys, unsigned long long* hist,
                            cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_bin_keys<<<grid_for(n), kThreads, 0, st>>>(t, n_z, n_y, boxes, orig, n,
                                               n_subsets, keys, hist);
  return cudaGetLastError();
}

cudaError_t launch_bin_scatter(const int* keys, int64_t n, const float* zu,
                               const float* zd, const float* dl,
                               const int64_t* orig, unsigned long long* cursor,
                               float* ozu, float* ozd, float* odl,
                               int64_t* operm, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_bin_scatter<<<grid_for(n), kThreads, 0, st>>>(keys, n, zu, zd, dl, orig,
                                                  cursor, ozu, ozd, odl, operm);
  return cudaGetLastError();
}

cudaError_t launch_update(float* rho, double* acc, int64_t n_pix, double scale,
                          cudaStream_t st) {
  k_update<<<grid_for(n_pix), kThreads, 0, st>>>(rho, acc, n_pix, scale);
  return cudaGetLastError();
}

cudaError_t launch_sensitivity(const ScannerF& s, int five_point, float* out,
                               cudaStream_t st) {
  const int64_t n = (int64_t)s.n_y * s.n_z;
  k_sensitivity<<<grid_for(n), kThreads, 0, st>>>(s, five_point, out);
  return cudaGetLastError();
}

cudaError_t launch_debug_sets(const ScannerF& s, const float* zu,
                              const float* zd, const float* dl, int64_t n,
                              int32_t* n_bb, int32_t* n_in, uint64_t* digest,
                              cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_debug_sets<<<grid_for(n * 32), kThreads, 0, st>>>(s, zu, zd, dl, n, n_bb,
                                                      n_in, digest);
  return cudaGetLastError();
}

cudaError_t launch_scale_copy(const double* acc, const float* sens,
                              double* out, int64_t n_pix, cudaStream_t st) {
  k_scale_copy<<<grid_for(n_pix), kThreads, 0, st>>>(acc, sens, out, n_pix);
  return cudaGetLastError();
}

cudaError_t launch_count_work(const ScannerF& s, const float* zu,
                              const float* zd, const float* dl, int64_t n,
                              unsigned long long* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_count_work<<<grid_for(n * 32), kThreads, 0, st>>>(s, zu, zd, dl, n, out);
  return cudaGetLastError();
}

cudaError_t launch_fma_peak(int n_sm, int iters, float* out, double* flops,
                            cudaStream_t st) {
  const int blocks = n_sm * 4, threads = 512;
  k_fma_peak<<<blocks, threads, 0, st>>>(out, iters, 0.99999f, 1e-5f);
  *flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  return cudaGetLastError();
}

}  // namespace stripmlem
