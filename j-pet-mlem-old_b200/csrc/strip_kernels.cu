// sm_100a kernels of the strip list-mode TOF MLEM path.
//
//   k_event_boxes / k_bin_keys / k_bin_scatter   one-time binning of the events
//       into image tiles (events are iteration-invariant, so this is paid once)
//   k_tile      the hot kernel: one CTA per (tile, event chunk) work item.  The
//       tile's window of the image (tile + halo) is staged in shared memory
//       next to a shared-memory backprojection accumulator.  A warp takes one
//       event at a time:
//         (a) event setup and the exact per-row pixel runs of its 3-sigma
//             ellipse (strip_rows.cuh), the TOF kernel's row constants;
//         (b) D_e = sum K * rho (* s): lane per row, the Gaussian advanced
//             along the row's run by the recurrence E <- E * R, R <- R * q
//             (two multiplies per pixel), per-row binary32 partials combined
//             across rows in binary32, Kahan or binary64, and across lanes in
//             binary64;
//         (c) the same walk scatters K / D_e with shared-memory atomics;
//       and the window is finally flushed into the global binary64
//       accumulator.
//   k_global    the same per-event work for events whose box does not fit a
//       window (global loads, global binary64 atomics).
//   k_update    (d) rho_j <- rho_j * acc_j * scale, acc_j <- 0.
//
// Reference behaviour: Reconstruction::bb_update (src/2d/strip/reconstruction.h:
// 220-298) and the warp kernel (src/2d/strip/cuda/reconstruction/
// warp_granularity.cuh:20-176).
#include <algorithm>

#include "strip_internal.h"
#include "strip_rows.cuh"

namespace stripmlem {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
// Threads of a tile CTA whose windows leave room for two CTAs per SM.
#ifndef STRIP_TILE_THREADS
#define STRIP_TILE_THREADS 512
#endif
constexpr int kTileThreads = STRIP_TILE_THREADS;
// Tile kernels whose shared-memory windows leave room for one CTA per SM
// run 1024-thread CTAs (32 warps, 64 registers each), so the SM keeps as
// many resident warps as with two 512-thread CTAs.
constexpr int kWideThreads = 1024;
// Column-major tile windows where they fit (tile_column_stride).
#ifndef STRIP_COLUMN_MAJOR
#define STRIP_COLUMN_MAJOR 1
#endif
constexpr int kMaxWarps = kWideThreads / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// A set-up event as a warp holds it until its turn: tan, y, z, sec and the
// clamped box (columns and rows lie in [0, 32767]) in two words.  The
// ellipse's A, B, C follow from tan and sec (and the scanner) by the same
// rounded binary32 operations as in event_setup, so they are formed again
// when the event is taken (fewer registers held through the walks).
struct EventPack {
  float tan, y, z, sec;
  unsigned x, yb;  // tlx | brx << 16, tly | bry << 16
};
__device__ __forceinline__ EventPack pack_event(const EventF& e) {
  return EventPack{e.tan, e.y, e.z, e.sec, (unsigned)e.tlx | ((unsigned)e.brx << 16),
                   (unsigned)e.tly | ((unsigned)e.bry << 16)};
}
__device__ __forceinline__ EventF shfl_event(const ScannerF& s, const EventPack& m, int src) {
  EventF e;
  e.tan = __shfl_sync(kFull, m.tan, src);
  e.y = __shfl_sync(kFull, m.y, src);
  e.z = __shfl_sync(kFull, m.z, src);
  e.sec = __shfl_sync(kFull, m.sec, src);
  const unsigned x = __shfl_sync(kFull, m.x, src), yb = __shfl_sync(kFull, m.yb, src);
  e.tlx = (int)(x & 0xFFFFu);
  e.brx = (int)(x >> 16);
  e.tly = (int)(yb & 0xFFFFu);
  e.bry = (int)(yb >> 16);
  // gaussian_kernel.h:120-122, as event_setup
  const float tt = __fmul_rn(e.tan, e.tan);
  e.A = __fadd_rn(__fmul_rn(__fmul_rn(__fmul_rn(4.0f, e.sec), e.sec), s.ipsdl),
                  __fmul_rn(__fmul_rn(2.0f, tt), s.ipsz));
  e.B = __fmul_rn(__fmul_rn(-4.0f, e.tan), s.ipsz);
  e.C = __fmul_rn(2.0f, s.ipsz);
  return e;
}

// Accumulation of the per-row partial sums of D_e within a lane.
template <int ACC>
struct RowSum;
template <>
struct RowSum<STRIP_ACCUM_FP32> {
  float s = 0.0f;
  __device__ __forceinline__ void add(float x) { s += x; }
  __device__ __forceinline__ double total() const { return (double)s; }
};
template <>
struct RowSum<STRIP_ACCUM_KAHAN> {
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
struct RowSum<STRIP_ACCUM_FP64> {
  double s = 0.0;
  __device__ __forceinline__ void add(float x) { s += (double)x; }
  __device__ __forceinline__ double total() const { return s; }
};

// Binary32 -> integer by a power-of-two addend: for 0 <= x * s < 2^23 the
// bits of x * s + 2^23 (one FFMA, round to nearest) minus those of 2^23 are
// round(x * s); for |x * s| < 2^22 the same with 1.5 * 2^23 gives the
// two's-complement round(x * s).
constexpr float kMagic = 8388608.0f;
constexpr unsigned kMagicBits = 0x4B000000u;
constexpr float kMagicSigned = 12582912.0f;
constexpr unsigned kMagicSignedBits = 0x4B400000u;
__device__ __forceinline__ unsigned to_fixed(float x, float s) {
  return __float_as_uint(fmaf(x, s, kMagic)) - kMagicBits;
}

// Shared-memory access by 32-bit shared-space byte address: the walks below
// advance one address register per step and let the loads and atomics use
// immediate offsets.
__device__ __forceinline__ float lds32(uint32_t addr) {
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}
__device__ __forceinline__ void red_shared_add(uint32_t addr, unsigned v) {
  asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// Row of rank i among an event's H box rows, ranked middle-out: the centre
// row first, then alternately below and above.
__device__ __forceinline__ int ranked_row(int H, int i) {
  const int mid = (H - 1) >> 1;
  return mid + ((i & 1) ? ((i + 1) >> 1) : -(i >> 1));
}

// How a shared-memory window accumulates the backprojection:
//   kAccF32     binary32 atomics (a load and a compare-and-swap per add here)
//   kAccU32     unsigned fixed point, the 2^23 addend (rho-weighted MLEM)
//   kAccU32Cvt  unsigned fixed point, cvt.rni (scales above 2^22)
//   kAccS32     signed fixed point, the 1.5 * 2^23 addend (adjoint)
//   kAccU32Unw  unsigned fixed point of K / D (cvt.rni), rho applied at the
//               flush (MLEM from an item's second pass on)
// The fixed-point kinds use native 32-bit integer shared atomics; the scale
// `fixed_unit` is a power of two chosen per work item so that no sum wraps.
enum AccKind { kAccF32 = 0, kAccU32 = 1, kAccU32Cvt = 2, kAccS32 = 3, kAccU32Unw = 4 };

// Per-CTA state of the work item in flight: the unweighted window's
// fixed-point budget (units of 2^8), the item's sum of 1 / D_e, and the
// events the unweighted window had no room for (bit i: event begin + i).
constexpr unsigned kBudgetUnits = (unsigned)(kFixedBudget / 256.0f);
__shared__ unsigned s_fx_budget;
__shared__ float s_item_rsum;
__shared__ unsigned s_fb_bits[kMaxItemEvents / 32];
__shared__ int s_fb_n;

// A tile's window in shared memory: row-major with row stride WS (CS = 0), or
// column-major with column stride CS words (a multiple of 32).  Column-major,
// a lane walking its row stays in one bank, that of its row (its word
// addresses differ by multiples of 32), so the lanes of a row block -- rows
// of distinct banks, whatever their runs' first columns -- do not conflict;
// row-major, a lane's bank follows its run's first column, and the lanes of
// one instruction collide about twice as often (a bank-conflict simulation
// over the benchmark's events: 2.39 wavefronts per walk instruction
// row-major, 1.80 column-major).
template <int KIND, int CS = 0>
struct SmemWin {
  const float* w;
  float* acc;
  int wx0, wy0, WS;
  float fixed_unit;
  uint32_t w_sh, acc_sh;  // shared-space addresses of w and acc
  static constexpr bool kShared = true;
  // words between neighbouring pixels of a row, and their byte distance
  static constexpr int kStep = CS ? CS : 1;
  static constexpr uint32_t kPixB = 4u * kStep;
  __device__ __forceinline__ uint32_t w_addr(int p) const { return w_sh + 4u * (uint32_t)p; }
  __device__ __forceinline__ uint32_t acc_addr(int p) const { return acc_sh + 4u * (uint32_t)p; }
  __device__ __forceinline__ float unit() const {
    return KIND == kAccF32 ? 1.0f : fixed_unit;
  }
  __device__ __forceinline__ int ptr(int iy, int col) const {
    return CS ? (col - wx0) * CS + (iy - wy0) : (iy - wy0) * WS + (col - wx0);
  }
  // A lane's run of row iy kept in one register: window offset << 16 | len
  // (windows hold < 2^16 words, runs < 2^16).
  __device__ __forceinline__ unsigned pack_run(int iy, int lo, int len) const {
    return len > 0 ? ((unsigned)ptr(iy, lo) << 16) | (unsigned)len : 0u;
  }
  __device__ __forceinline__ int run_ptr(unsigned v, const EventF&, int,
                                         int) const {
    return (int)(v >> 16);
  }
  __device__ __forceinline__ float read(int p, int j) const { return w[p + j * kStep]; }
  // acc_j += v (v already scaled by unit())
  __device__ __forceinline__ void add(int p, int j, float v) const {
    if constexpr (KIND == kAccS32)
      atomicAdd(reinterpret_cast<int*>(acc) + p + j * kStep,
                (int)(__float_as_uint(v + kMagicSigned) - kMagicSignedBits));
    else
      atomicAdd(acc + p + j * kStep, v);
  }
  // acc_j += K_j w_j / D_e for K_j = E * pref and sc = pref / D_e * unit()
  __device__ __forceinline__ void add_weighted(int p, int j, float E,
                                               float sc) const {
    const unsigned v = KIND == kAccU32Cvt ? __float2uint_rn(E * w[p + j * kStep] * sc)
                                          : to_fixed(E * w[p + j * kStep], sc);
    atomicAdd(reinterpret_cast<unsigned*>(acc) + p + j * kStep, v);
  }
  // signed fixed point: the adjoint's pair walk adds two pixels a step
  __host__ __device__ static constexpr bool pair_add() { return KIND == kAccS32; }
  __host__ __device__ static constexpr bool unweighted() { return KIND == kAccU32Unw; }
  __host__ __device__ static constexpr bool fine() { return KIND == kAccU32Cvt; }
  // the rho-weighted MLEM scatter takes two pixels a step
  __host__ __device__ static constexpr bool pair_scatter() {
    return KIND == kAccU32 || KIND == kAccU32Cvt;
  }
};

// The whole image in global memory.
template <int MODE>
struct GlobalWin {
  const float* rho;
  const float* sens;
  double* acc;
  int n_z;
  __device__ __forceinline__ int64_t ptr(int iy, int col) const {
    return (int64_t)iy * n_z + col;
  }
  // lo << 16 | len; the row is recomputed from the lane's rank
  __device__ __forceinline__ unsigned pack_run(int, int lo, int len) const {
    return len > 0 ? ((unsigned)lo << 16) | (unsigned)len : 0u;
  }
  __device__ __forceinline__ int64_t run_ptr(unsigned v, const EventF& e,
                                             int H, int rank) const {
    return ptr(e.tly + ranked_row(H, rank), (int)(v >> 16));
  }
  __device__ __forceinline__ float read(int64_t p, int j) const {
    float v = __ldg(rho + p + j);
    if (MODE == STRIP_MODE_GPU) v *= __ldg(sens + p + j);
    return v;
  }
  __device__ __forceinline__ void add(int64_t p, int j, float v) const {
    atomicAdd(acc + p + j, (double)v);
  }
  __device__ __forceinline__ float unit() const { return 1.0f; }
  static constexpr bool kShared = false;
  __device__ __forceinline__ uint32_t w_addr(int64_t) const { return 0; }
  __device__ __forceinline__ uint32_t acc_addr(int64_t) const { return 0; }
  __host__ __device__ static constexpr bool pair_scatter() { return false; }
  __host__ __device__ static constexpr bool pair_add() { return false; }
  __host__ __device__ static constexpr bool unweighted() { return false; }
  __device__ __forceinline__ void add_weighted(int64_t p, int j, float E,
                                               float sc) const {
    atomicAdd(acc + p + j, (double)(E * read(p, j) * sc));
  }
};

// Walks the lane's share of the flattened pixel list of rows
// [row0, row0 + nrows).  For each run piece, f(r, col, cnt) is called with
// the row index within the block, the first column and the pixel count.
template <class F>
__device__ __forceinline__ void walk_share(const RowTables& T, int nrows,
                                           int n, int lane, F&& f) {
  int f0, f1;
  int r = lane_share(T, nrows, n, lane, f0, f1);
  int pos = f0;
  while (pos < f1) {
    const int rs = T.start[r], re = T.start[r + 1];
    if (re > pos) {
      const int cnt = min(re, f1) - pos;
      f(r, T.lo[r] + (pos - rs), cnt);
      pos += cnt;
    }
    ++r;
  }
}

// ---------------------------------------------------------------------------
// Lane-per-row event processing.  An event is worked on by a group of LPE
// lanes: a whole warp, a half-warp or a quarter-warp.  The box rows
// of an event are ranked middle-out (the centre row first, then alternately
// below and above), so a block of LPE consecutive ranks holds rows of
// similar run length; lane l of the group owns, in block k, the row of rank
// LPE k + l.  A lane keeps its rows' run (lo, len) and recurrence state
// (K0, R0) in registers across both passes: pass 1 walks its runs with
// K <- K*R, R <- R*q (no per-pixel exponential, no per-pixel bookkeeping),
// pass 2 walks them again from the stored state.  Events with more than
// LPE * row_blocks rows are processed in super-blocks and rebuilt for pass 2.
//
// The GaussianKernel's MLEM gives each event a half-warp: 16-row blocks
// follow an ellipse's run lengths (longest in the middle rows, shortest at
// the tips) more closely than 32-row blocks, so fewer lanes idle in the
// set-up and in the walks (each block walks as long as its longest run), and
// two events share the per-event shuffles and reductions.  The forward and
// adjoint, which keep no rows between passes, go further: a quarter-warp per
// event, 8-row blocks, four events per warp.  The AnalyticKernel (six row
// constants a block) and the sigma gradient keep one event per warp.
// ---------------------------------------------------------------------------
#ifndef STRIP_LPE
#define STRIP_LPE 16
#endif
#ifndef STRIP_PROJ_LPE
#define STRIP_PROJ_LPE 8
#endif
template <int OP, int MODE>
__host__ __device__ constexpr int lanes_per_event() {
  return MODE != STRIP_MODE_CPU || OP == OP_GRAD ? 32
         : OP == OP_MLEM                        ? STRIP_LPE
         : STRIP_LPE == 32                      ? 32
                                                : STRIP_PROJ_LPE;
}
// Row blocks a lane keeps in registers (a super-block is LPE * blocks rows).
// MLEM keeps its rows for both passes: with half-warps 5 blocks hold the at
// most 76 box rows of sigma_dl = 25 mm on 1 mm pixels in one super-block.
// The persistent batch kernel, whose members' constants take registers of
// their own, keeps 4 (64 rows).  The forward and adjoint walk each row once,
// so smaller super-blocks cost them only the loop, and free registers.
#ifndef STRIP_MLEM_BLOCKS
#define STRIP_MLEM_BLOCKS 5
#endif
#ifndef STRIP_BATCH_BLOCKS
#define STRIP_BATCH_BLOCKS 4
#endif
#ifndef STRIP_PROJ_BLOCKS
#define STRIP_PROJ_BLOCKS 3
#endif
#ifndef STRIP_PROJ_BLOCKS8
#define STRIP_PROJ_BLOCKS8 3
#endif
#ifndef STRIP_WHOLE_BLOCKS
#define STRIP_WHOLE_BLOCKS 3
#endif
template <int OP, int LPE, bool BATCH = false>
__host__ __device__ constexpr int row_blocks() {
  return LPE == 32        ? (OP == OP_MLEM ? STRIP_WHOLE_BLOCKS : 3)
         : LPE == 8       ? STRIP_PROJ_BLOCKS8
         : OP != OP_MLEM  ? STRIP_PROJ_BLOCKS
         : BATCH          ? STRIP_BATCH_BLOCKS
                          : STRIP_MLEM_BLOCKS;
}
// Whether a launch whose tallest event box has max_rows rows gives its events
// fewer than 32 lanes (lanes_per_event): MLEM only when one super-block
// holds every event, since past it pass 2 rebuilds the rows of the further
// super-blocks (a whole warp's 96-row super-block suits taller boxes, e.g.
// the up to 126 rows of sigma_dl = 42 mm on 1 mm pixels, better: measured
// on the 64-instance batch); the forward and adjoint walk each row once and
// always do.
#ifndef STRIP_BATCH_HALF
#define STRIP_BATCH_HALF 1
#endif
__host__ __device__ constexpr bool half_warp_events(int op, int max_rows, bool batch = false) {
  return batch ? STRIP_BATCH_HALF && max_rows <= 16 * STRIP_BATCH_BLOCKS
               : op != OP_MLEM || max_rows <= 16 * STRIP_MLEM_BLOCKS;
}

// Sum over the lanes of one event's group (every lane of the warp calls it).
template <int LPE>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = LPE / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Walk GaussianKernel runs two pixels per step with packed f32x2 arithmetic.
#ifndef STRIP_PAIRS
#define STRIP_PAIRS 1
#endif
constexpr bool kPairs = STRIP_PAIRS != 0;

template <int MODE, int NB>
struct LaneRows;

// Run of block b: run[b] = the window's packed run (len == 0: no run).
__device__ __forceinline__ int run_len(unsigned v) { return (int)(v & 0xFFFFu); }

// GaussianKernel: K along the run from K0 = K(t0) and the ratio R0
template <int NB>
struct LaneRows<STRIP_MODE_CPU, NB> {
  unsigned run[NB];
  float K0[NB], R0[NB];
};
// AnalyticKernel: direct evaluation per pixel from the row constants
template <int NB>
struct LaneRows<STRIP_MODE_GPU, NB> {
  unsigned run[NB];
  float t0[NB], n0[NB], n1[NB], u0[NB], u1[NB], cr[NB];
};

// Builds the lane's rows of ranks rank0 + LPE * b + sub (b < NB) of an event
// of H rows (H = 0: no rows).
template <int MODE, bool CLOSED_ONLY, int LPE, int NB, class Win>
__device__ __forceinline__ void build_lane_rows_t(const ScannerF& s,
                                                const KernelF& k,
                                                const EventF& e,
                                                const EventRows& er,
                                                const GaussEvent& ge, int H,
                                                int rank0, int sub,
                                                const Win& win,
                                                LaneRows<MODE, NB>& L) {
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    L.run[b] = 0u;
    if constexpr (MODE == STRIP_MODE_CPU) {  // rows without a run walk nothing
      L.K0[b] = 0.0f;
      L.R0[b] = 0.0f;
    }
    const int i = rank0 + LPE * b + sub;
    if (i < H) {
      const int iy = e.tly + ranked_row(H, i);
      const RowSet rs = row_set(s, e, iy);
      int lo;
      const int len = row_run<CLOSED_ONLY>(s, e, er, rs, lo);
      L.run[b] = win.pack_run(iy, lo, len);
      if (len > 0) {
        const float t0 = (fmaf((float)lo, s.pw, s.tl_z_half_w) - e.z);
        if constexpr (MODE == STRIP_MODE_CPU) {
          ge.row(k, e.y, e.tan, rs.dy, t0, L.K0[b], L.R0[b]);
        } else {
          AnalyticRow g;
          g.init(k, s.R, e.y, e.tan, e.sec, rs.dy);
          L.t0[b] = t0 - g.dytan;
          L.n0[b] = g.n0;
          L.n1[b] = g.n1;
          L.u0[b] = g.u0;
          L.u1[b] = g.u1;
          L.cr[b] = g.cr;
        }
      }
    }
  }
}

// The same, with the row runs' general search compiled out when the
// geometry lets the closed form settle every row (uniform per launch).
template <int MODE, int LPE, int NB, class Win>
__device__ __forceinline__ void build_lane_rows(const ScannerF& s,
                                                const KernelF& k,
                                                const EventF& e,
                                                const EventRows& er,
                                                const GaussEvent& ge, int H,
                                                int rank0, int sub,
                                                const Win& win,
                                                LaneRows<MODE, NB>& L) {
  if (s.min_closed_hw == 0.0f)
    build_lane_rows_t<MODE, true, LPE>(s, k, e, er, ge, H, rank0, sub, win, L);
  else
    build_lane_rows_t<MODE, false, LPE>(s, k, e, er, ge, H, rank0, sub, win, L);
}

// Pass 1 over the lane's rows: sum over runs of K_j * w_j.  nb (the blocks
// to walk) is the same in every lane of the warp.
template <int MODE, int ACC, int LPE, int NB, class Win>
__device__ __forceinline__ void pass1_rows(const ScannerF& s, const KernelF& k,
                                           const EventF& e, int H, int rank0,
                                           int sub, const LaneRows<MODE, NB>& L,
                                           int nb, const Win& win,
                                           RowSum<ACC>& acc) {
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int n = run_len(L.run[b]);
    // every lane enters (a lane without a run walks n = 0 pixels): the warp
    // stays converged instead of branching around empty rows
    if (b < nb) {
      const auto p = win.run_ptr(L.run[b], e, H, rank0 + LPE * b + sub);
      float a = 0.0f;
      if constexpr (MODE == STRIP_MODE_CPU && kPairs && Win::kShared) {
        // two pixels per step: a count-down loop over pairs, one shared
        // address register, float2 arithmetic
        const float K0 = L.K0[b], R0 = L.R0[b], R2 = R0 * R0;
        float2 P = make_float2(K0, K0 * R0);
        float2 S = make_float2(R2 * k.q, R2 * k.q3);
        const float2 Q4 = make_float2(k.q4, k.q4);
        float2 A = make_float2(0.0f, 0.0f);
        uint32_t ad = win.w_addr(p);
#pragma unroll 2
        for (int c = n >> 1; c > 0; --c, ad += 2 * Win::kPixB) {
          A = __ffma2_rn(P, make_float2(lds32(ad), lds32(ad + Win::kPixB)), A);
          P = __fmul2_rn(P, S);
          S = __fmul2_rn(S, Q4);
        }
        a = A.x + A.y;
        if (n & 1) a = fmaf(P.x, lds32(ad), a);
      } else if constexpr (MODE == STRIP_MODE_CPU && kPairs) {
        PairRecurrence g(k, L.K0[b], L.R0[b]);
        f32x2 A = pack2(0.0f, 0.0f);
#pragma unroll 2
        for (int j = 0; j + 1 < n; j += 2) {
          A = fma2(g.P, pack2(win.read(p, j), win.read(p, j + 1)), A);
          g.step();
        }
        const float2 a2 = unpack2(A);
        a = a2.x + a2.y;
        if (n & 1) a = fmaf(unpack2(g.P).x, win.read(p, n - 1), a);
      } else if constexpr (MODE == STRIP_MODE_CPU) {
        float K = L.K0[b], R = L.R0[b];
#pragma unroll 4
        for (int j = 0; j < n; ++j) {
          a = fmaf(K, win.read(p, j), a);
          K *= R;
          R *= k.q;
        }
      } else {
        AnalyticRow g;
        g.n0 = L.n0[b];
        g.n1 = L.n1[b];
        g.u0 = L.u0[b];
        g.u1 = L.u1[b];
        g.cr = L.cr[b];
#pragma unroll 2
        for (int j = 0; j < n; ++j)
          a = fmaf(g.eval_t(k, fmaf((float)j, s.pw, L.t0[b])), win.read(p, j), a);
      }
      acc.add(a);
    }
  }
}

// Pass 2 over the lane's rows: acc_j += K_j * scale, or, WEIGHTED (MLEM with
// the reference CPU semantics), acc_j += K_j * w_j * scale.  A lane whose
// event does not scatter (go false) walks no pixels.
template <int MODE, bool WEIGHTED, int LPE, int NB, class Win>
__device__ __forceinline__ void pass2_rows(const ScannerF& s, const KernelF& k,
                                           const EventF& e, int H, int rank0,
                                           int sub, const LaneRows<MODE, NB>& L,
                                           int nb, const Win& win,
                                           float scale, bool go) {
  // the event's factor in the window's units (clamped: a denominator so
  // small that 1 / D overflows still scatters finite values)
  const float sc = WEIGHTED ? fminf(scale * win.unit(), 3.0e38f)
                            : scale * win.unit();
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int n = go ? run_len(L.run[b]) : 0;
    // every lane enters (a lane without a run walks n = 0 pixels): the warp
    // stays converged instead of branching around empty rows
    if (b < nb) {
      const auto p = win.run_ptr(L.run[b], e, H, rank0 + LPE * b + sub);
      if constexpr (MODE == STRIP_MODE_CPU && WEIGHTED && Win::unweighted()) {
        // K / D in fixed point: no image reads, one conversion per pixel
        const float K0 = L.K0[b] * sc, R0 = L.R0[b], R2 = R0 * R0;
        float2 P = make_float2(K0, K0 * R0);
        float2 S = make_float2(R2 * k.q, R2 * k.q3);
        const float2 Q4 = make_float2(k.q4, k.q4);
        uint32_t aa = win.acc_addr(p);
#pragma unroll 2
        for (int c = n >> 1; c > 0; --c, aa += 2 * Win::kPixB) {
          red_shared_add(aa, __float2uint_rn(P.x));
          red_shared_add(aa + Win::kPixB, __float2uint_rn(P.y));
          P = __fmul2_rn(P, S);
          S = __fmul2_rn(S, Q4);
        }
        if (n & 1) red_shared_add(aa, __float2uint_rn(P.x));
      } else if constexpr (MODE == STRIP_MODE_CPU && WEIGHTED && kPairs &&
                    Win::pair_scatter()) {
        // pass 1's walk with K scaled by sc = unit / D from the start, so
        // u = K w / D in fixed point is one FFMA per pixel (the 2^23 addend)
        // and native shared integer reductions
        const float K0 = L.K0[b] * sc, R0 = L.R0[b], R2 = R0 * R0;
        float2 P = make_float2(K0, K0 * R0);
        float2 S = make_float2(R2 * k.q, R2 * k.q3);
        const float2 Q4 = make_float2(k.q4, k.q4);
        uint32_t ad = win.w_addr(p), aa = win.acc_addr(p);
#pragma unroll 2
        for (int c = n >> 1; c > 0; --c, ad += 2 * Win::kPixB, aa += 2 * Win::kPixB) {
          const float2 w2 = make_float2(lds32(ad), lds32(ad + Win::kPixB));
          unsigned v0, v1;
          if constexpr (Win::fine()) {
            const float2 x = __fmul2_rn(P, w2);
            v0 = __float2uint_rn(x.x);
            v1 = __float2uint_rn(x.y);
          } else {
            const float2 x = __ffma2_rn(P, w2, make_float2(kMagic, kMagic));
            v0 = __float_as_uint(x.x) - kMagicBits;
            v1 = __float_as_uint(x.y) - kMagicBits;
          }
          red_shared_add(aa, v0);
          red_shared_add(aa + Win::kPixB, v1);
          P = __fmul2_rn(P, S);
          S = __fmul2_rn(S, Q4);
        }
        if (n & 1) {
          const float w = lds32(ad);
          red_shared_add(aa, Win::fine() ? __float2uint_rn(P.x * w) : to_fixed(P.x, w));
        }
      } else if constexpr (MODE == STRIP_MODE_CPU && WEIGHTED) {
        float K = L.K0[b], R = L.R0[b];
#pragma unroll 4
        for (int j = 0; j < n; ++j) {
          win.add_weighted(p, j, K, sc);
          K *= R;
          R *= k.q;
        }
      } else if constexpr (MODE == STRIP_MODE_CPU && kPairs && Win::pair_add()) {
        // the adjoint's signed fixed point: K_j w_e with w_e and the unit
        // folded into the run's first value, two pixels a step; rounding by
        // the 1.5 * 2^23 addend (|addend| < 2^22: round to nearest even, as
        // cvt.rni) keeps the conversions off the MUFU/conversion pipe
        const float K0 = L.K0[b] * sc, R0 = L.R0[b], R2 = R0 * R0;
        float2 P = make_float2(K0, K0 * R0);
        float2 S = make_float2(R2 * k.q, R2 * k.q3);
        const float2 Q4 = make_float2(k.q4, k.q4);
        uint32_t aa = win.acc_addr(p);
#pragma unroll 2
        for (int c = n >> 1; c > 0; --c, aa += 2 * Win::kPixB) {
          const float2 x = __fadd2_rn(P, make_float2(kMagicSigned, kMagicSigned));
          red_shared_add(aa, __float_as_uint(x.x) - kMagicSignedBits);
          red_shared_add(aa + Win::kPixB, __float_as_uint(x.y) - kMagicSignedBits);
          P = __fmul2_rn(P, S);
          S = __fmul2_rn(S, Q4);
        }
        if (n & 1) red_shared_add(aa, (unsigned)__float2int_rn(P.x));
      } else if constexpr (MODE == STRIP_MODE_CPU) {
        float K = L.K0[b], R = L.R0[b];
#pragma unroll 4
        for (int j = 0; j < n; ++j) {
          win.add(p, j, K * sc);
          K *= R;
          R *= k.q;
        }
      } else {
        AnalyticRow g;
        g.n0 = L.n0[b];
        g.n1 = L.n1[b];
        g.u0 = L.u0[b];
        g.u1 = L.u1[b];
        g.cr = L.cr[b];
#pragma unroll 2
        for (int j = 0; j < n; ++j)
          win.add(p, j, g.eval_t(k, fmaf((float)j, s.pw, L.t0[b])) * sc);
      }
    }
  }
}

// OP_GRAD, GaussianKernel: adds w_e * d/d(sz, sdl) sum_j K_j w_j to
// grad_out[0..1].  Lane per row (plain order); per row the run is walked with
// the same recurrence as pass 1 while s0 = sum E w and s2 = sum E w t^2 are
// gathered, so the row's share is pref * (fz s0 + 2 ipsz s2) / sz and
// pref * fdl * s0 / sdl.
// Per-event data besides the event itself, loaded by the lane that sets the
// event up (so the dependent global loads overlap instead of stalling the
// warp at every event): OP_FORWARD the caller's index of the event,
// OP_ADJOINT its weight (binned order), OP_GRAD its weight (caller order).
struct EventAux {
  int64_t out = 0;
  double w = 0.0;
  float wf = 0.0f;
};

template <int OP>
__device__ __forceinline__ EventAux load_aux(const LaunchArgs& a, int64_t pos) {
  EventAux x;
  if constexpr (OP == OP_FORWARD) x.out = a.perm[pos];
  if constexpr (OP == OP_ADJOINT) x.wf = a.wf_in[pos];
  if constexpr (OP == OP_GRAD) x.w = a.w_in[a.perm[pos]];
  return x;
}

template <int OP>
__device__ __forceinline__ EventAux shfl_aux(const EventAux& m, int src) {
  EventAux x;
  if constexpr (OP == OP_FORWARD) x.out = __shfl_sync(kFull, m.out, src);
  if constexpr (OP == OP_ADJOINT) x.wf = __shfl_sync(kFull, m.wf, src);
  if constexpr (OP == OP_GRAD) x.w = __shfl_sync(kFull, m.w, src);
  return x;
}

template <class Win>
__device__ __forceinline__ void grad_event(const LaunchArgs& a,
                                           const EventF& e,
                                           const EventRows& er, int H,
                                           const Win& win, int lane,
                                           double w) {
  if (w == 0.0) return;
  double gz = 0.0, gdl = 0.0;
  for (int i = lane; i < H; i += 32) {
    const int iy = e.tly + i;
    const RowSet rs = row_set(a.s, e, iy);
    int lo;
    const int len = row_run(a.s, e, er, rs, lo);
    if (len <= 0) continue;
    GaussGradRow g;
    g.init(a.k, a.s.R, e.y, e.tan, e.sec, rs.dy);
    const float t0 = fmaf((float)lo, a.s.pw, a.s.tl_z_half_w) - e.z - g.dytan;
    float E = ex2_approx(fmaf(a.k.c1 * t0, t0, g.c0));
    float R = ex2_approx(fmaf(a.k.r1, t0, a.k.r0));
    const auto p = win.ptr(iy, lo);
    float s0 = 0.0f, s2 = 0.0f;
    for (int j = 0; j < len; ++j) {
      const float ew = E * win.read(p, j);
      const float t = fmaf((float)j, a.s.pw, t0);
      s0 += ew;
      s2 = fmaf(ew * t, t, s2);
      E *= R;
      R *= a.k.q;
    }
    gz += (double)(g.pref * fmaf(g.fz, s0, 2.0f * a.k.ipsz * s2));
    gdl += (double)(g.pref * g.fdl * s0);
  }
  gz = warp_sum(gz);
  gdl = warp_sum(gdl);
  if (lane == 0) {
    atomicAdd(a.grad_out, w * gz / a.sz);
    atomicAdd(a.grad_out + 1, w * gdl / a.sdl);
  }
}

// The event of lane src of the warp's set-up lanes (`mine`), or, when `has`
// is false, an event without box rows.
__device__ __forceinline__ EventF fetch_event(const ScannerF& s, const EventPack& mine,
                                              int src, bool has) {
  EventF e = shfl_event(s, mine, src);
  if (!has) e.bry = e.tly;
  return e;
}

// One event on a group of LPE lanes (every lane of the warp calls this; with
// LPE < 32 each group of the warp brings its own event, and an empty event
// has no box rows): the event of set-up lane src (has: there is one).  Returns, in
// the event's lanes, 1 / D_e for an MLEM event with a positive denominator
// (the work item's statistic), 0 otherwise; -1 / D_e for an event the
// unweighted window had no room for (not scattered: the caller runs it again
// in a weighted window).  The event's set-up values are not kept through
// pass 2: the rare events whose rows need a second super-block fetch the
// event again (fewer live registers in the walks).
template <int OP, int MODE, int ACC, int LPE, int NB, class Win>
__device__ __forceinline__ float process_event(const LaunchArgs& a,
                                               const EventPack& mine, int src, bool has,
                                               const Win& win,
                                               int lane, const EventAux& aux) {
  static_assert(LPE == 32 || LPE == 16 || LPE == 8, "a warp, a half or a quarter per event");
  static_assert(OP != OP_GRAD || LPE == 32, "the sigma gradient takes a warp");
  const EventF e = fetch_event(a.s, mine, src, has);
  const int sub = lane & (LPE - 1);
  const int H = (e.bry > e.tly && e.brx > e.tlx) ? e.bry - e.tly : 0;
  int Hw = H;  // the warp's largest, for loop bounds the whole warp shares
#pragma unroll
  for (int o = LPE; o < 32; o <<= 1) Hw = max(Hw, __shfl_xor_sync(kFull, Hw, o));
  if (Hw == 0) return 0.0f;
  const EventRows er = event_rows(a.s, e);
  if constexpr (OP == OP_GRAD) {
    grad_event(a, e, er, H, win, lane, aux.w);
    return 0.0f;
  }
  GaussEvent ge{};
  if constexpr (MODE == STRIP_MODE_CPU) ge.init(a.k, a.s.R, e.tan, e.sec);
  constexpr int kSuper = LPE * NB;
  LaneRows<MODE, NB> L;
  float scale;
  bool go;  // this lane's event scatters
  if (OP == OP_MLEM || OP == OP_FORWARD) {
    RowSum<ACC> acc;
    // super-blocks of rows last to first, so that the registers end holding
    // the first (the middle rows, the longest runs): pass 2 rebuilds only
    // the others
    for (int r0 = ((Hw - 1) / kSuper) * kSuper; r0 >= 0; r0 -= kSuper) {
      build_lane_rows<MODE, LPE>(a.s, a.k, e, er, ge, H, r0, sub, win, L);
      pass1_rows<MODE, ACC, LPE>(a.s, a.k, e, H, r0, sub, L,
                                 min(NB, (Hw - r0 + LPE - 1) / LPE), win, acc);
    }
    const double D = group_sum<LPE>(acc.total());
    if (OP == OP_FORWARD) {
      if (sub == 0 && H > 0) a.y_out[aux.out] = D;
      return 0.0f;
    }
    // reconstruction.h:290 -- an all-zero denominator contributes nothing
    go = H > 0 && D > 0.0;
    scale = go ? rcp_approx((float)D) : 0.0f;  // within an ulp of 1 / D; 0 or inf at the range ends
  } else {
    scale = aux.wf;  // OP_ADJOINT
    go = H > 0 && scale != 0.0f;
  }
  float ret = go ? scale : 0.0f;
  if constexpr (Win::unweighted()) {
    // reserve the event's largest addend, kbound * unit / D (rounded up, in
    // units of 2^8), from the item's fixed-point budget
    const float need = a.kbound * scale * win.unit();
    int ok = 0;
    if (sub == 0 && go && need < kFixedBudget) {
      const unsigned nu = (unsigned)(need * (1.0f / 256.0f)) + 1u;
      const unsigned old = atomicAdd(&s_fx_budget, nu);
      ok = old + nu <= kBudgetUnits;
      if (!ok) atomicSub(&s_fx_budget, nu);
    }
    ok = __shfl_sync(kFull, ok, lane & ~(LPE - 1));
    if (go && !ok) {
      ret = -scale;
      go = false;
    }
  }
  if (!__any_sync(kFull, go)) return OP == OP_MLEM ? ret : 0.0f;
  constexpr bool kWeighted = OP == OP_MLEM && MODE == STRIP_MODE_CPU;
  if (OP == OP_MLEM) {  // the registers hold the first super-block
    pass2_rows<MODE, kWeighted, LPE>(a.s, a.k, e, H, 0, sub, L,
                                     min(NB, (Hw + LPE - 1) / LPE), win, scale, go);
    if (Hw <= kSuper) return ret;
  }
  const EventF e2 = OP == OP_MLEM ? fetch_event(a.s, mine, src, has) : e;
  const EventRows er2 = OP == OP_MLEM ? event_rows(a.s, e2) : er;
  GaussEvent ge2 = ge;
  if constexpr (OP == OP_MLEM && MODE == STRIP_MODE_CPU) ge2.init(a.k, a.s.R, e2.tan, e2.sec);
  for (int r0 = OP == OP_MLEM ? kSuper : 0; r0 < Hw; r0 += kSuper) {
    build_lane_rows<MODE, LPE>(a.s, a.k, e2, er2, ge2, H, r0, sub, win, L);
    pass2_rows<MODE, kWeighted, LPE>(a.s, a.k, e2, H, r0, sub, L,
                                     min(NB, (Hw - r0 + LPE - 1) / LPE), win, scale, go);
  }
  return OP == OP_MLEM ? ret : 0.0f;
}

__device__ __forceinline__ RowTables warp_tables(char* base, int cap, int warp) {
  return row_tables_at(base + (size_t)warp * row_table_bytes(cap), cap);
}

// Fixed-point scale of an adjoint work item: every addend is K_j w_e with
// K_j <= a.kbound (the GaussianKernel's bound, E <= 1 and a'Sa >= 2 R^2 ipsz)
// and |w_e| <= W, the item's largest weight, so with B = kbound * W the
// scale 2^s keeps each addend below 2^22 and the item's sum below 2^31.
__device__ int adjoint_shift(const LaunchArgs& a, const WorkItem& it, int lane) {
  __shared__ float s_wmax[kMaxWarps];
  __shared__ int s_shift;
  float m = 0.0f;
  for (int64_t i = it.begin + threadIdx.x; i < it.begin + it.count;
       i += blockDim.x)
    m = fmaxf(m, fabsf(a.wf_in[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(kFull, m, o));
  if (lane == 0) s_wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float W = 0.0f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) W = fmaxf(W, s_wmax[i]);
    const float B = a.kbound * W * 1.0001f;
    const float n = (float)it.count + (float)(it.count >> 7) + 1.0f;
    const float lim = fminf(4194304.0f, 2147483648.0f / n);
    int sh = 0;
    if (B > 0.0f && B < 3.0e38f)
      sh = (int)floorf(log2f(lim / B)) - 1;
    s_shift = max(-120, min(120, sh));
  }
  __syncthreads();
  return s_shift;
}

// The events of a work item: warps pull groups of a.grab (1..32) events from
// a shared counter until the item is done (lanes < a.grab set the group's
// events up in parallel).  With `only`, just the events whose bit is set:
// the rerun, in a weighted window, of the events an unweighted window had no
// room for (their 1 / D_e is counted already).
template <int OP, int MODE, int ACC, int LPE, int NB, class Win>
__device__ __forceinline__ void run_item(const LaunchArgs& a, const WorkItem& it,
                                         const Win& win, int lane,
                                         int* next_group,
                                         const unsigned* only = nullptr) {
  constexpr int kPerWarp = 32 / LPE;  // events the warp works on at once
  const int half = lane / LPE;        // this lane's event of the kPerWarp
  const int64_t end = it.begin + it.count;
  const int grab = a.grab;
  float rsum = 0.0f;  // the sum of 1 / D_e of this lane's events
  for (;;) {
    int g = 0;
    if (lane == 0) g = atomicAdd(next_group, 1);
    g = __shfl_sync(kFull, g, 0);
    const int64_t base = it.begin + (int64_t)g * grab;
    if (base >= end) break;
    const int64_t ei = base + lane;
    EventPack mine = {};
    EventAux aux;
    if (lane < grab && ei < end) {
      const int off = (int)(ei - it.begin);
      if (!only || ((only[off >> 5] >> (off & 31)) & 1u)) {
        aux = load_aux<OP>(a, ei);
        EventF ev;
        event_setup(a.s, a.zu[ei], a.zd[ei], a.dl[ei], ev);
        mine = pack_event(ev);
      }
    }
    const int nh = (int)min((int64_t)grab, end - base);
    for (int j0 = 0; j0 < nh; j0 += kPerWarp) {
      const int j = j0 + half;
      const bool has = j < nh;  // no event for this half: no rows
      const float r = process_event<OP, MODE, ACC, LPE, NB>(
          a, mine, has ? j : j0, has, win, lane, shfl_aux<OP>(aux, has ? j : j0));
      if (r < 0.0f) {  // not scattered: no room in the unweighted window
        if ((lane & (LPE - 1)) == 0) {
          const int off = (int)(base + j - it.begin);
          atomicOr(&s_fb_bits[off >> 5], 1u << (off & 31));
          atomicAdd(&s_fb_n, 1);
        }
        rsum -= r;
      } else {
        rsum += r;
      }
    }
  }
  if (OP == OP_MLEM && (lane & (LPE - 1)) == 0 && !only && rsum != 0.0f)
    atomicAdd(&s_item_rsum, rsum);
}

// Sum of v over the CTA, returned to every thread (two barriers).
__device__ __forceinline__ float block_sum(float v) {
  __shared__ float s_part[kMaxWarps];
  __shared__ float s_total;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
    s_total = t;
  }
  __syncthreads();
  return s_total;
}

// One work item on the whole CTA: stage the window, run the events, flush.
// `index` is the item's index among the launch's items (its statistic in
// a.item_hist).  The CTA may run further items afterwards (the batched
// kernel): the caller synchronises before the shared memory is reused.
template <int OP, int MODE, int ACC, int LPE, int NB, int CS>
__device__ __forceinline__ void tile_item(const LaunchArgs& a,
                                          const WorkItem it, int index,
                                          char* smem_raw, int* s_next_group) {
  int wx0, wy0, wx1, wy1;
  tile_window(a.t, a.s.n_z, a.s.n_y, it.tile, wx0, wy0, wx1, wy1);
  const int wxn = wx1 - wx0, wyn = wy1 - wy0, WS = a.t.WS;
  float* s_w = reinterpret_cast<float*>(smem_raw);
  // the adjoint reads no image: its accumulator is the only window
  float* s_acc = OP == OP_ADJOINT ? s_w : s_w + (CS ? a.t.WXmax * CS : a.t.WYmax * WS);
  constexpr bool kReads = (OP != OP_ADJOINT);
  constexpr bool kWrites = (OP == OP_MLEM || OP == OP_ADJOINT);
  constexpr bool kFixedMlem = (OP == OP_MLEM && MODE == STRIP_MODE_CPU);
  if (threadIdx.x == 0) {
    *s_next_group = 0;
    s_fx_budget = 0u;
    s_item_rsum = 0.0f;
    s_fb_n = 0;
  }
  if (kFixedMlem)
    for (int q = threadIdx.x; q < kMaxItemEvents / 32; q += blockDim.x) s_fb_bits[q] = 0u;
  const int lane = threadIdx.x & 31;
  float wsum = 0.0f;
  // window word of (row r, column c): row-major or column-major (CS)
  auto widx = [WS](int r, int c) { return CS ? c * CS + r : r * WS + c; };
  for (int q = threadIdx.x; q < wxn * wyn; q += blockDim.x) {
    const int r = q / wxn, c = q - r * wxn;
    const int64_t gi = (int64_t)(wy0 + r) * a.s.n_z + wx0 + c;
    if (kReads) {
      float v = a.rho[gi];
      if (MODE == STRIP_MODE_GPU) v *= a.sens[gi];
      s_w[widx(r, c)] = v;
      wsum += v;
    }
    if (kWrites) s_acc[widx(r, c)] = 0.0f;
  }
  __syncthreads();
  const uint32_t w_sh = (uint32_t)__cvta_generic_to_shared(s_w);
  const uint32_t acc_sh = (uint32_t)__cvta_generic_to_shared(s_acc);
  // Adds the window accumulator (fixed point at scale 2^fshift, times the
  // image value for an unweighted window, which is zeroed on the way) into
  // the global binary64 accumulator.
  auto flush = [&](int fshift, bool unweighted) {
    unsigned* s_acc_u = reinterpret_cast<unsigned*>(s_acc);
    const int* s_acc_i = reinterpret_cast<const int*>(s_acc);
    for (int q = threadIdx.x; q < wxn * wyn; q += blockDim.x) {
      const int r = q / wxn, c = q - r * wxn;
      double v;
      const int wi = widx(r, c);
      if constexpr (kFixedMlem) {
        v = ldexp((double)s_acc_u[wi], -fshift);
        if (unweighted) {
          v *= (double)s_w[wi];
          s_acc_u[wi] = 0u;
        }
      } else if constexpr (OP == OP_ADJOINT && MODE == STRIP_MODE_CPU) {
        v = ldexp((double)s_acc_i[wi], -fshift);
      } else {
        v = (double)s_acc[wi];
      }
      if (v != 0.0)
        atomicAdd(a.acc + (int64_t)(wy0 + r) * a.s.n_z + wx0 + c, v);
    }
  };
  // A weighted MLEM window over `count` events of the item (those of `only`,
  // or all); returns its scale's exponent.
  auto run_weighted = [&](int count, const unsigned* only) {
    const int fs = fixed_shift(count);
    run_item<OP, MODE, ACC, LPE, NB>(
        a, it, SmemWin<kAccU32Cvt, CS>{s_w, s_acc, wx0, wy0, WS, exp2f((float)fs), w_sh, acc_sh},
        lane, s_next_group, only);
    return fs;
  };
  if constexpr (kFixedMlem) {
    // the unweighted window once the item has a statistic, else weighted
    const float wmean = block_sum(wsum) / (float)(wxn * wyn);
    const float hist = a.item_hist ? a.item_hist[index] : 0.0f;
    const float B = hist / wmean;  // this pass's sum of 1 / D_e, estimated
    const float lim = 1073741824.0f / (a.kbound * B);  // 2^30 / (kbound B)
    int fshift = 0;
    bool unweighted = false;
    if (hist > 0.0f && wmean > 0.0f && B > 0.0f && B < 3.0e38f && lim > 0.0f &&
        lim < 3.0e38f) {
      fshift = (int)floorf(log2f(lim));
      unweighted = fshift >= -120 && fshift <= 120;
    }
    if (unweighted) {
      run_item<OP, MODE, ACC, LPE, NB>(
          a, it,
          SmemWin<kAccU32Unw, CS>{s_w, s_acc, wx0, wy0, WS, exp2f((float)fshift), w_sh, acc_sh},
          lane, s_next_group);
      __syncthreads();
      flush(fshift, true);
      const int n_fb = s_fb_n;
      if (n_fb > 0) {  // the events that found no room, in a weighted window
        __syncthreads();  // the flush has zeroed the window accumulator
        if (threadIdx.x == 0) {
          *s_next_group = 0;
          if (a.n_fallback) atomicAdd(a.n_fallback, (unsigned long long)n_fb);
        }
        __syncthreads();
        const int fs = run_weighted(n_fb, s_fb_bits);
        __syncthreads();
        flush(fs, false);
      }
    } else {
      const int fs = run_weighted(it.count, nullptr);
      __syncthreads();
      flush(fs, false);
    }
    if (threadIdx.x == 0 && a.item_hist) a.item_hist[index] = s_item_rsum * wmean;
  } else if constexpr (OP == OP_ADJOINT && MODE == STRIP_MODE_CPU) {
    const int fshift = adjoint_shift(a, it, lane);
    run_item<OP, MODE, ACC, LPE, NB>(
        a, it,
        SmemWin<kAccS32, CS>{s_w, s_acc, wx0, wy0, WS, exp2f((float)fshift), w_sh, acc_sh},
        lane, s_next_group);
    __syncthreads();
    flush(fshift, false);
  } else {
    run_item<OP, MODE, ACC, LPE, NB>(a, it,
                            SmemWin<kAccF32, CS>{s_w, s_acc, wx0, wy0, WS, 1.0f, w_sh, acc_sh},
                            lane, s_next_group);
    if (kWrites) {
      __syncthreads();
      flush(0, false);
    }
  }
}

// CTAs per SM a tile kernel is compiled for: MLEM keeps two windows (image
// and accumulator) and up to 64 registers a thread (2 x 16 warps per SM);
// the GaussianKernel forward and adjoint keep one window each; at 2 x 16
// warps (64 registers, no spills) they ran 5 % / 1 % faster than at
// 3 x 16 warps (40 registers, with spills) once they took a quarter-warp per
// event.
#ifndef STRIP_FWD_CTAS
#define STRIP_FWD_CTAS 2
#endif
#ifndef STRIP_ADJ_CTAS
#define STRIP_ADJ_CTAS 2
#endif
template <int OP, int MODE>
constexpr int tile_ctas_per_sm() {
  return MODE != STRIP_MODE_CPU ? 2
         : OP == OP_FORWARD    ? STRIP_FWD_CTAS
         : OP == OP_ADJOINT    ? STRIP_ADJ_CTAS
                               : 2;
}
template <int OP>
constexpr int tile_windows() { return OP == OP_MLEM ? 2 : 1; }

template <int OP, int MODE, int ACC, int THREADS, int LPE, int CS>
__global__ void __launch_bounds__(THREADS, THREADS == kWideThreads
                                               ? 1
                                               : tile_ctas_per_sm<OP, MODE>())
    k_tile(const __grid_constant__ LaunchArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ int s_next_group;
  tile_item<OP, MODE, ACC, LPE, row_blocks<OP, LPE>(), CS>(a, a.items[blockIdx.x], blockIdx.x,
                                                           smem_raw, &s_next_group);
}

// Persistent tile kernel over the work items of several reconstructions: a
// CTA takes item after item from a global counter; item i belongs to member
// items[i].member, whose arguments live in the kernel's parameter space.
template <int MODE, int ACC, int THREADS, int LPE, int CS>
__global__ void __launch_bounds__(THREADS, THREADS == kWideThreads ? 1 : 2)
    k_tile_batch(const __grid_constant__ BatchArgs b, const BatchItem* items,
                 int n_items, int* counter) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ int s_next_group;
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int i = s_item;
    if (i >= n_items) break;
    const BatchItem bi = items[i];
    tile_item<OP_MLEM, MODE, ACC, LPE, row_blocks<OP_MLEM, LPE, true>(), CS>(b.member[bi.member],
                                  WorkItem{bi.tile, bi.count, bi.begin},
                                  bi.index, smem_raw, &s_next_group);
    __syncthreads();  // before the next item's window overwrites this one
  }
}

// rho_j <- acc_j * scale (or rho_j * acc_j * scale), acc_j <- 0 for every
// member: blockIdx.y selects the member.
__global__ void k_update_batch(const __grid_constant__ BatchUpdateArgs u) {
  const int m = blockIdx.y;
  if (m >= u.n) return;
  float* rho = u.rho[m];
  double* acc = u.acc[m];
  const int64_t n = u.n_pix[m];
  const int weighted = u.weighted;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    rho[j] = weighted ? (float)(acc[j] * u.scale)
                      : (float)((double)rho[j] * acc[j] * u.scale);
    acc[j] = 0.0;
  }
}

template <int OP, int MODE, int ACC>
__global__ void __launch_bounds__(kThreads) k_global(LaunchArgs a) {
  constexpr int LPE = lanes_per_event<OP, MODE>();
  constexpr int kPerWarp = 32 / LPE;
  const GlobalWin<MODE> win{a.rho, a.sens, a.acc, a.s.n_z};
  const int lane = threadIdx.x & 31;
  const int half = lane / LPE;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwt = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t end = a.g_begin + a.g_count;
  for (int64_t base = a.g_begin + wid * 32; base < end; base += nwt * 32) {
    const int64_t ei = base + lane;
    EventPack mine = {};
    EventAux aux;
    if (ei < end) {
      aux = load_aux<OP>(a, ei);
      EventF ev;
      event_setup(a.s, a.zu[ei], a.zd[ei], a.dl[ei], ev);
      mine = pack_event(ev);
    }
    const int nh = (int)min((int64_t)32, end - base);
    for (int j0 = 0; j0 < nh; j0 += kPerWarp) {
      const int j = j0 + half;
      const bool has = j < nh;
      process_event<OP, MODE, ACC, LPE, row_blocks<OP, LPE>()>(
          a, mine, has ? j : j0, has, win, lane, shfl_aux<OP>(aux, has ? j : j0));
    }
  }
}

__global__ void k_split_triples(const float* __restrict__ aos, int64_t n,
                                float* __restrict__ zu, float* __restrict__ zd,
                                float* __restrict__ dl) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    zu[i] = aos[3 * i];
    zd[i] = aos[3 * i + 1];
    dl[i] = aos[3 * i + 2];
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
// Keys and their histogram; with n_local > 0 (the number of keys) the CTA
// counts in shared memory first and adds its counts once per key.
__global__ void k_bin_keys(Tiling t, int n_z, int n_y, const int4* boxes,
                           const int64_t* orig, int64_t n, int n_subsets,
                           int* keys, unsigned long long* hist, int n_local) {
  extern __shared__ unsigned s_hist[];
  for (int k = threadIdx.x; k < n_local; k += blockDim.x) s_hist[k] = 0u;
  if (n_local > 0) __syncthreads();
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
    if (key >= 0 && lane == __ffs(peers) - 1) {
      if (n_local > 0)
        atomicAdd(s_hist + key, (unsigned)__popc(peers));
      else
        atomicAdd(hist + key, (unsigned long long)__popc(peers));
    }
  }
  if (n_local > 0) {
    __syncthreads();
    for (int k = threadIdx.x; k < n_local; k += blockDim.x)
      if (s_hist[k]) atomicAdd(hist + k, (unsigned long long)s_hist[k]);
  }
}

// Scatters the events into their bins.  With n_local > 0 (the number of
// keys) each CTA takes a contiguous chunk, counts its keys in shared memory,
// reserves its slots with one global atomic per key, and places events from
// shared-memory offsets; otherwise one warp-aggregated global atomic per key
// and warp.
__global__ void k_bin_scatter(const int* keys, int64_t n, const float* zu,
                              const float* zd, const float* dl,
                              const int64_t* orig, unsigned long long* cursor,
                              float* ozu, float* ozd, float* odl,
                              int64_t* operm, int n_local) {
  const int lane = threadIdx.x & 31;
  auto place = [&](int64_t i, int64_t p) {
    ozu[p] = zu[i];
    ozd[p] = zd[i];
    odl[p] = dl[i];
    operm[p] = orig ? orig[i] : i;
  };
  if (n_local > 0) {
    extern __shared__ unsigned long long s_base[];  // n_local bases, then counts
    unsigned* s_cnt = reinterpret_cast<unsigned*>(s_base + n_local);
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t c0 = (int64_t)blockIdx.x * chunk;
    const int64_t c1 = min(n, c0 + chunk);
    for (int k = threadIdx.x; k < n_local; k += blockDim.x) s_cnt[k] = 0u;
    __syncthreads();
    for (int64_t base = c0 + (threadIdx.x & ~31); base < c1; base += blockDim.x) {
      const int64_t i = base + lane;
      const int key = i < c1 ? keys[i] : -1;
      const unsigned peers = __match_any_sync(kFull, key);
      if (key >= 0 && lane == __ffs(peers) - 1) atomicAdd(s_cnt + key, (unsigned)__popc(peers));
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n_local; k += blockDim.x) {
      s_base[k] = s_cnt[k] ? atomicAdd(cursor + k, (unsigned long long)s_cnt[k]) : 0ull;
      s_cnt[k] = 0u;
    }
    __syncthreads();
    for (int64_t base = c0 + (threadIdx.x & ~31); base < c1; base += blockDim.x) {
      const int64_t i = base + lane;
      const int key = i < c1 ? keys[i] : -1;
      const unsigned peers = __match_any_sync(kFull, key);
      const int leader = __ffs(peers) - 1;
      unsigned o = 0;
      if (key >= 0 && lane == leader) o = atomicAdd(s_cnt + key, (unsigned)__popc(peers));
      o = __shfl_sync(kFull, o, leader);
      if (key >= 0)
        place(i, (int64_t)s_base[key] + o + __popc(peers & ((1u << lane) - 1u)));
    }
    return;
  }
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
    if (key >= 0) place(i, (int64_t)p0 + __popc(peers & ((1u << lane) - 1u)));
  }
}

// Orders the events of each work item for the column-major windows' banks.
// A lane's bank there is its row's, (row - wy0) mod 32, and the rows of a
// row block, ranked middle-out from the event's middle row m, cover a fixed
// set of residues around m: for 16-row blocks half of Z_32 whose other half
// is the same set around m + 16, for 8-row blocks a quarter whose shifts by
// 8, 16 and 24 tile Z_32.  So the item is laid out in quads of events whose
// middle rows are v, v + 16, v + 8 and v + 24 mod 32 (the half-warp pairs of
// MLEM take (v, v + 16) and (v + 8, v + 24), the quarter-warps of the
// forward and adjoint all four), then pairs (v, v + 16) of the events left,
// then the rest.  One CTA per item; the order within a middle-row class is
// that of the atomics.  The results change only by the order of the binary32
// sums.
__global__ void k_item_order(ScannerF s, Tiling t, const WorkItem* __restrict__ items,
                             const float* __restrict__ zu, const float* __restrict__ zd,
                             const float* __restrict__ dl, const int64_t* __restrict__ perm,
                             float* ozu, float* ozd, float* odl, int64_t* operm) {
  __shared__ int s_n[32], s_cnt[32];
  __shared__ int s_q[32], s_qbase[32], s_p[32], s_pbase[32], s_sbase[32];
  const WorkItem it = items[blockIdx.x];
  int wx0, wy0, wx1, wy1;
  tile_window(t, s.n_z, s.n_y, it.tile, wx0, wy0, wx1, wy1);
  if (threadIdx.x < 32) {
    s_n[threadIdx.x] = 0;
    s_cnt[threadIdx.x] = 0;
  }
  __syncthreads();
  auto cls = [&](int64_t i) {
    EventF e;
    event_setup(s, zu[i], zd[i], dl[i], e);
    return (e.tly + ((e.bry - e.tly - 1) >> 1) - wy0) & 31;
  };
  // class counts and, below, ranks: one shared atomic per class and warp
  // (lanes of a class found by __match_any_sync)
  const int lane = threadIdx.x & 31;
  const int n_round = (it.count + blockDim.x - 1) / blockDim.x * blockDim.x;
  for (int k = threadIdx.x; k < n_round; k += blockDim.x) {
    const int v = k < it.count ? cls(it.begin + k) : -1;
    const unsigned peers = __match_any_sync(kFull, v);
    if (v >= 0 && lane == __ffs(peers) - 1) atomicAdd(&s_n[v], __popc(peers));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int left[32];
    for (int v = 0; v < 32; ++v) left[v] = s_n[v];
    int pos = 0;
    for (int v = 0; v < 8; ++v) {  // quads: v, v + 16, v + 8, v + 24
      const int c[4] = {v, v + 16, v + 8, v + 24};
      const int q = min(min(left[c[0]], left[c[1]]), min(left[c[2]], left[c[3]]));
      for (int j = 0; j < 4; ++j) {
        s_q[c[j]] = q;
        s_qbase[c[j]] = pos + j;
        left[c[j]] -= q;
      }
      pos += 4 * q;
    }
    for (int v = 0; v < 16; ++v) {  // pairs: v, v + 16
      const int p = min(left[v], left[v + 16]);
      s_p[v] = s_p[v + 16] = p;
      s_pbase[v] = pos;
      s_pbase[v + 16] = pos + 1;
      left[v] -= p;
      left[v + 16] -= p;
      pos += 2 * p;
    }
    for (int v = 0; v < 32; ++v) {  // the rest
      s_sbase[v] = pos;
      pos += left[v];
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n_round; k += blockDim.x) {
    const int64_t i = it.begin + k;
    const int v = k < it.count ? cls(i) : -1;
    const unsigned peers = __match_any_sync(kFull, v);
    const int leader = __ffs(peers) - 1;
    int r0 = 0;
    if (v >= 0 && lane == leader) r0 = atomicAdd(&s_cnt[v], __popc(peers));
    r0 = __shfl_sync(kFull, r0, leader);
    if (v < 0) continue;
    const int r = r0 + __popc(peers & ((1u << lane) - 1u));
    const int q = s_q[v], p = s_p[v];
    const int at = r < q ? s_qbase[v] + 4 * r
                         : r < q + p ? s_pbase[v] + 2 * (r - q) : s_sbase[v] + (r - q - p);
    const int64_t o = it.begin + at;
    ozu[o] = zu[i];
    ozd[o] = zd[i];
    odl[o] = dl[i];
    operm[o] = perm[i];
  }
}

__global__ void k_gather_weights(const int64_t* perm, const double* w,
                                 int64_t n, float* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)w[perm[i]];
}

__global__ void k_update_out(const float* rho_in, float* rho_out,
                             const double* acc, int64_t n, int weighted) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    rho_out[j] = weighted ? (float)acc[j] : (float)((double)rho_in[j] * acc[j]);
}

__global__ void k_update(float* rho, double* acc, int64_t n, double scale,
                         int weighted) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    rho[j] = weighted ? (float)(acc[j] * scale)
                      : (float)((double)rho[j] * acc[j] * scale);
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

// Pixel-set parity and work counts: one warp per event, the same row-run
// enumeration (build_rows / walk_share) as the reconstruction kernels.
template <bool DEBUG>
__global__ void __launch_bounds__(kThreads) k_sets(
    ScannerF s, const float* zu, const float* zd, const float* dl, int64_t n,
    int cap, int32_t* n_bb, int32_t* n_in, uint64_t* digest,
    unsigned long long* totals) {
  extern __shared__ __align__(16) char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const RowTables T = warp_tables(smem_raw, cap, warp);
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwt = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const KernelF k{};
  unsigned long long tb = 0, ti = 0, tn = 0;
  for (int64_t i = wid; i < n; i += nwt) {
    EventF e;
    event_setup(s, zu[i], zd[i], dl[i], e);
    const int H = e.bry - e.tly, W = e.brx - e.tlx;
    unsigned cnt = 0;
    unsigned long long h = 0;
    if (H > 0 && W > 0) {
      const EventRows er = event_rows(s, e);
      for (int r0 = 0; r0 < H; r0 += cap) {
        const int nr = min(cap, H - r0);
        if (r0 > 0) __syncwarp();
        const int m = s.min_closed_hw == 0.0f
                          ? build_rows<0, true>(s, k, e, er, e.tly + r0, nr, T, lane)
                          : build_rows<0, false>(s, k, e, er, e.tly + r0, nr, T, lane);
        cnt += m;
        if (DEBUG) {
          walk_share(T, nr, m, lane, [&](int r, int col, int c) {
            const int64_t idx = (int64_t)(e.tly + r0 + r) * s.n_z + col;
            for (int j = 0; j < c; ++j) h += mix64((uint64_t)(idx + j) + 1u);
          });
        }
      }
      __syncwarp();
    }
    if (DEBUG) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(kFull, h, o);
      if (lane == 0) {
        if (n_bb) n_bb[i] = (H > 0 && W > 0) ? W * H : 0;
        if (n_in) n_in[i] = (int32_t)cnt;
        if (digest) digest[i] = h;
      }
    } else if (lane == 0 && H > 0 && W > 0) {
      tb += (unsigned long long)W * H;
      ti += cnt;
      tn += cnt > 0;
    }
  }
  if (!DEBUG && lane == 0) {
    atomicAdd(totals, tb);
    atomicAdd(totals + 1, ti);
    atomicAdd(totals + 2, tn);
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

constexpr int kSetsCap = 64;

template <int OP, int MODE, int ACC, int LPE>
cudaError_t launch_tile_lpe(const LaunchArgs& a, cudaStream_t st) {
  const int smem = a.t.smem_bytes / 2 * tile_windows<OP>();
  const bool wide = smem > kNarrowSmemBytes;  // one CTA per SM: 1024 threads
  auto fn = a.t.cs == kColumnStride
                ? (wide ? k_tile<OP, MODE, ACC, kWideThreads, LPE, kColumnStride>
                        : k_tile<OP, MODE, ACC, kTileThreads, LPE, kColumnStride>)
                : (wide ? k_tile<OP, MODE, ACC, kWideThreads, LPE, 0>
                        : k_tile<OP, MODE, ACC, kTileThreads, LPE, 0>);
  cudaError_t err = cudaFuncSetAttribute(
      fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (err != cudaSuccess) return err;
  fn<<<a.n_items, wide ? kWideThreads : kTileThreads, smem, st>>>(a);
  return cudaGetLastError();
}

template <int OP, int MODE, int ACC>
cudaError_t launch_tile_t(const LaunchArgs& a, cudaStream_t st) {
  constexpr int kLanes = lanes_per_event<OP, MODE>();
  if constexpr (kLanes < 32) {
    if (half_warp_events(OP, a.t.max_rows)) return launch_tile_lpe<OP, MODE, ACC, kLanes>(a, st);
  }
  return launch_tile_lpe<OP, MODE, ACC, 32>(a, st);
}

template <int OP, int MODE, int ACC>
cudaError_t launch_global_t(const LaunchArgs& a, cudaStream_t st) {
  const int grid = grid_for(a.g_count, kWarps * 32);
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

// Two windows (the image and the accumulator) of WYmax rows of stride WS.
int tile_smem_bytes(int WYmax, int WS) { return 2 * WYmax * WS * 4; }

// The column stride of a tiling's windows: kColumnStride (column-major) when
// the windows are at most that many rows high and their column-major form
// fits `budget` bytes, else 0 (row-major).
int tile_column_stride(int WXmax, int WYmax, int budget) {
  if (!STRIP_COLUMN_MAJOR) return 0;
  return WYmax <= kColumnStride && 2 * WXmax * kColumnStride * 4 <= budget ? kColumnStride : 0;
}

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
    case OP_GRAD:  // GaussianKernel only
      if (mode != STRIP_MODE_CPU) return cudaErrorInvalidValue;
      return launch_tile_t<OP_GRAD, STRIP_MODE_CPU, STRIP_ACCUM_FP32>(a, st);
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
    case OP_GRAD:  // GaussianKernel only
      if (mode != STRIP_MODE_CPU) return cudaErrorInvalidValue;
      return launch_global_t<OP_GRAD, STRIP_MODE_CPU, STRIP_ACCUM_FP32>(a, st);
    default:
      return cudaErrorInvalidValue;
  }
}

template <int THREADS, int CS, class F>
cudaError_t with_tile_batch_t(int mode, int accum, bool half, F&& pick) {
  if (mode == STRIP_MODE_CPU) {
    constexpr int H = lanes_per_event<OP_MLEM, STRIP_MODE_CPU>();
    if (half) {
      if (accum == STRIP_ACCUM_FP32)
        return pick(k_tile_batch<STRIP_MODE_CPU, STRIP_ACCUM_FP32, THREADS, H, CS>);
      if (accum == STRIP_ACCUM_FP64)
        return pick(k_tile_batch<STRIP_MODE_CPU, STRIP_ACCUM_FP64, THREADS, H, CS>);
      return pick(k_tile_batch<STRIP_MODE_CPU, STRIP_ACCUM_KAHAN, THREADS, H, CS>);
    }
    if (accum == STRIP_ACCUM_FP32)
      return pick(k_tile_batch<STRIP_MODE_CPU, STRIP_ACCUM_FP32, THREADS, 32, CS>);
    if (accum == STRIP_ACCUM_FP64)
      return pick(k_tile_batch<STRIP_MODE_CPU, STRIP_ACCUM_FP64, THREADS, 32, CS>);
    return pick(k_tile_batch<STRIP_MODE_CPU, STRIP_ACCUM_KAHAN, THREADS, 32, CS>);
  }
  if (accum == STRIP_ACCUM_FP32)
    return pick(k_tile_batch<STRIP_MODE_GPU, STRIP_ACCUM_FP32, THREADS, 32, CS>);
  if (accum == STRIP_ACCUM_FP64)
    return pick(k_tile_batch<STRIP_MODE_GPU, STRIP_ACCUM_FP64, THREADS, 32, CS>);
  return pick(k_tile_batch<STRIP_MODE_GPU, STRIP_ACCUM_KAHAN, THREADS, 32, CS>);
}

// The persistent batch kernel of a class: windows that fit two CTAs per SM
// run 512-thread CTAs, wider ones 1024-thread CTAs, one per SM; half-warp
// events where every member's tallest box allows them; row-major or
// column-major windows (cs).
template <class F>
cudaError_t with_tile_batch(int mode, int accum, int smem_bytes, int max_rows, int cs,
                            F&& pick) {
  const bool half = half_warp_events(OP_MLEM, max_rows, true);
  const bool wide = smem_bytes > kNarrowSmemBytes;
  if (cs == kColumnStride)
    return wide ? with_tile_batch_t<kWideThreads, kColumnStride>(mode, accum, half, pick)
                : with_tile_batch_t<kTileThreads, kColumnStride>(mode, accum, half, pick);
  return wide ? with_tile_batch_t<kWideThreads, 0>(mode, accum, half, pick)
              : with_tile_batch_t<kTileThreads, 0>(mode, accum, half, pick);
}

cudaError_t tile_batch_reserve_smem(int mode, int accum, int smem_bytes, int max_rows, int cs) {
  return with_tile_batch(mode, accum, smem_bytes, max_rows, cs, [&](auto fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem_bytes);
  });
}

cudaError_t launch_tile_batch(int mode, int accum, const BatchArgs& b,
                              const BatchItem* items, int n_items, int* counter,
                              int smem_bytes, int max_rows, int cs, int sm_count,
                              cudaStream_t st) {
  if (n_items <= 0) return cudaSuccess;
  const bool wide = smem_bytes > kNarrowSmemBytes;
  auto pick = [&](auto fn) -> cudaError_t {
    const int grid = std::min(n_items, sm_count * (wide ? 1 : 2));
    fn<<<grid, wide ? kWideThreads : kTileThreads, smem_bytes, st>>>(b, items, n_items, counter);
    return cudaGetLastError();
  };
  return with_tile_batch(mode, accum, smem_bytes, max_rows, cs, pick);
}


cudaError_t launch_update_batch(const BatchUpdateArgs& u, int64_t max_pix,
                                cudaStream_t st) {
  if (u.n <= 0) return cudaSuccess;
  const int gx = (int)std::min<int64_t>(std::max<int64_t>((max_pix + kThreads - 1) / kThreads, 1), 64);
  k_update_batch<<<dim3(gx, u.n), kThreads, 0, st>>>(u);
  return cudaGetLastError();
}

cudaError_t launch_split_triples(const float* aos, int64_t n, float* zu, float* zd,
                                 float* dl, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_split_triples<<<grid_for(n), kThreads, 0, st>>>(aos, n, zu, zd, dl);
  return cudaGetLastError();
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
  // per-CTA counts in shared memory up to 12288 keys (48 KB)
  const int64_t n_keys = (int64_t)n_subsets * (t.n_tiles + 1);
  const int n_local = n_keys <= 12288 ? (int)n_keys : 0;
  k_bin_keys<<<grid_for(n), kThreads, n_local * sizeof(unsigned), st>>>(
      t, n_z, n_y, boxes, orig, n, n_subsets, keys, hist, n_local);
  return cudaGetLastError();
}

cudaError_t launch_bin_scatter(const int* keys, int64_t n, const float* zu,
                               const float* zd, const float* dl,
                               const int64_t* orig, unsigned long long* cursor,
                               float* ozu, float* ozd, float* odl,
                               int64_t* operm, int64_t n_keys, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  // per-CTA reservations in shared memory up to 4096 keys (48 KB)
  const int n_local = n_keys <= 4096 ? (int)n_keys : 0;
  k_bin_scatter<<<grid_for(n), kThreads, n_local * 12, st>>>(
      keys, n, zu, zd, dl, orig, cursor, ozu, ozd, odl, operm, n_local);
  return cudaGetLastError();
}

cudaError_t launch_update(float* rho, double* acc, int64_t n_pix, double scale,
                          int weighted, cudaStream_t st) {
  k_update<<<grid_for(n_pix), kThreads, 0, st>>>(rho, acc, n_pix, scale,
                                                 weighted);
  return cudaGetLastError();
}

cudaError_t launch_item_order(const ScannerF& s, const Tiling& t, const WorkItem* items,
                              int n_items, const float* zu, const float* zd, const float* dl,
                              const int64_t* perm, float* ozu, float* ozd, float* odl,
                              int64_t* operm, cudaStream_t st) {
  if (n_items <= 0) return cudaSuccess;
  k_item_order<<<n_items, 256, 0, st>>>(s, t, items, zu, zd, dl, perm, ozu, ozd, odl, operm);
  return cudaGetLastError();
}

cudaError_t launch_gather_weights(const int64_t* perm, const double* w,
                                  int64_t n, float* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_gather_weights<<<grid_for(n), kThreads, 0, st>>>(perm, w, n, out);
  return cudaGetLastError();
}

cudaError_t launch_update_out(const float* rho_in, float* rho_out,
                              const double* acc, int64_t n_pix, int weighted,
                              cudaStream_t st) {
  k_update_out<<<grid_for(n_pix), kThreads, 0, st>>>(rho_in, rho_out, acc, n_pix,
                                                     weighted);
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
  const int smem = kWarps * row_table_bytes(kSetsCap);
  k_sets<true><<<grid_for(n * 32), kThreads, smem, st>>>(
      s, zu, zd, dl, n, kSetsCap, n_bb, n_in, digest, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_count_work(const ScannerF& s, const float* zu,
                              const float* zd, const float* dl, int64_t n,
                              unsigned long long* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int smem = kWarps * row_table_bytes(kSetsCap);
  k_sets<false><<<grid_for(n * 32), kThreads, smem, st>>>(
      s, zu, zd, dl, n, kSetsCap, nullptr, nullptr, nullptr, out);
  return cudaGetLastError();
}

cudaError_t launch_scale_copy(const double* acc, const float* sens,
                              double* out, int64_t n_pix, cudaStream_t st) {
  k_scale_copy<<<grid_for(n_pix), kThreads, 0, st>>>(acc, sens, out, n_pix);
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
