// Internal interfaces between the C-ABI layer (strip_capi.cu) and the
// kernels (strip_kernels.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "stripmlem.h"
#include "strip_device.cuh"
#include "strip_kernel_eval.cuh"

namespace stripmlem {

// A unit of work of the tile kernel: `count` events starting at sorted
// position `begin`, all of whose boxes lie inside the window of `tile`.
struct WorkItem {
  int32_t tile;
  int32_t count;
  int64_t begin;
};

// MLEM backprojection with the reference CPU semantics accumulates, per event
// and pixel, u = K_j rho_j / D_e -- what reconstruction.h:276-295 scatters --
// and u lies in [0, 1] because D_e = sum_k K_k rho_k.  The tile kernel's
// shared-memory window therefore accumulates u in unsigned 32-bit fixed point
// (native integer shared atomics instead of a compare-and-swap loop per
// binary32 add).  A work item of `count` events uses the scale 2^s with the
// largest s <= kMaxFixedShift for which (count + count/128 + 1) * 2^s <=
// 2^32, so no pixel sum can wrap: s = 19 for the largest items
// (kMaxItemEvents), 22 for 1016 events, 30 for the smallest.
//
// From the second pass over an item on, the window instead accumulates
// K_j / D_e ("unweighted"): rho_j multiplies the pixel's sum once, when the
// window is flushed, so the scatter walk reads no image values.  K_j / D_e
// has no a-priori bound, so the scale comes from the item's previous pass:
// with B the item's sum of 1 / D_e (kept as B times the window's mean image
// value, so a rescaled image rescales it) the scale is the largest 2^s <=
// 2^30 / (kbound B).  Before its scatter each event reserves its largest
// addend, kbound 2^s / D_e, from a per-item budget of 2^32 - 2^24 (rounding
// included), so no pixel sum can wrap.  An event that does not fit is not
// scattered; once the unweighted window is flushed, those events run again
// in a weighted window of their own.
constexpr int kMaxFixedShift = 30;
// Dynamic shared memory of a tile window that still runs two CTAs per SM.
constexpr int kNarrowSmemBytes = 111 * 1024;
constexpr float kFixedBudget = 4278190080.0f;  // 2^32 - 2^24
constexpr int kMaxItemEvents = 8000;

__host__ __device__ inline int fixed_shift(int count) {
  const unsigned m = (unsigned)count + ((unsigned)count >> 7) + 1u;
  int lg = 0;  // ceil(log2(m))
  while ((1u << lg) < m && lg < 31) ++lg;
  const int s = 32 - lg;
  return s < kMaxFixedShift ? s : kMaxFixedShift;
}

// Image tiling.  Tile (bx, by) owns pixels [bx*TX, (bx+1)*TX) x [by*TY, ...);
// its shared-memory window adds a halo of (HX, HY) pixels on each side,
// clamped to the image.  WXmax/WYmax bound every window, WS is the padded
// shared-memory row stride.
struct Tiling {
  int TX, TY, HX, HY, ntx, nty, n_tiles;
  int WXmax, WYmax, WS;
  int smem_bytes;  // the two shared-memory windows
  int max_rows;    // the most box rows of any event (the kernels' lane layout)
  int cs;          // window column stride: kColumnStride (column-major) or 0
};
// Column stride of column-major tile windows (words; a multiple of 32).
constexpr int kColumnStride = 128;

__host__ __device__ inline void tile_window(const Tiling& t, int n_z, int n_y,
                                            int tile, int& wx0, int& wy0,
                                            int& wx1, int& wy1) {
  const int bx = tile % t.ntx, by = tile / t.ntx;
  wx0 = bx * t.TX - t.HX;
  wx0 = wx0 < 0 ? 0 : wx0;
  wy0 = by * t.TY - t.HY;
  wy0 = wy0 < 0 ? 0 : wy0;
  wx1 = (bx + 1) * t.TX + t.HX;
  wx1 = wx1 > n_z ? n_z : wx1;
  wy1 = (by + 1) * t.TY + t.HY;
  wy1 = wy1 > n_y ? n_y : wy1;
}

// What a tile / global-path launch computes.
enum Op {
  OP_MLEM = 0,     // D_e, then acc_j += K_ej / D_e
  OP_FORWARD = 1,  // y_e = D_e
  OP_ADJOINT = 2,  // acc_j += K_ej * w_e
  OP_GRAD = 3      // d/dsigma of sum_e w_e D_e
};

// Event triples (z_u, z_d, dl) x n -> three arrays.
cudaError_t launch_split_triples(const float* aos, int64_t n, float* zu, float* zd,
                                 float* dl, cudaStream_t st);

struct LaunchArgs {
  ScannerF s;
  KernelF k;          // kernel constants (model sigmas)
  Tiling t;
  const float* zu;    // events, binned order
  const float* zd;
  const float* dl;
  const int64_t* perm;   // binned position -> caller's event index
  const float* rho;      // image
  const float* sens;     // pixel sensitivity (gpu mode) or null
  double* acc;           // backprojection accumulator (binary64)
  const WorkItem* items;
  int n_items;
  int64_t g_begin;       // global-path event range [g_begin, g_begin+g_count)
  int64_t g_count;
  double* y_out;         // OP_FORWARD: per event (caller order)
  const double* w_in;    // OP_GRAD: per event weights in the caller's order
  const float* wf_in;    // OP_ADJOINT: per event weights in binned order
  double* grad_out;      // OP_GRAD: 2 doubles (atomic)
  double sz, sdl;        // OP_GRAD: model sigmas
  float kbound;          // bound of the GaussianKernel values (OP_ADJOINT,
                         // OP_MLEM with the reference CPU semantics)
  int grab;              // events a warp takes per counter step (1..32)
  int* status;           // device status word (0 = ok)
  // OP_MLEM, GaussianKernel: per work item (indexed like `items`), the
  // item's sum of 1 / D_e times its window's mean image value from the last
  // pass over the item (0: none yet), which sizes the unweighted fixed-point
  // window of the next pass; may be null
  float* item_hist;
  unsigned long long* n_fallback;  // events rerun in a weighted window, or null
};

// Several reconstructions in one persistent launch (strip_batch.cu): the
// members' arguments travel in the kernel parameter space (up to 32 KB).
constexpr int kMaxBatch = 64;
struct BatchArgs {
  LaunchArgs member[kMaxBatch];
};
static_assert(sizeof(BatchArgs) <= 32000, "batch arguments exceed the parameter space");
struct BatchItem {
  int32_t member;
  int32_t tile;
  int32_t count;
  int32_t pad;    // host-side: the item's shared-memory class
  int64_t begin;
  int32_t index;  // the item's index among its member's work items
  int32_t pad2;
};
struct BatchUpdateArgs {
  int n;
  int weighted;
  double scale;
  float* rho[kMaxBatch];
  double* acc[kMaxBatch];
  int64_t n_pix[kMaxBatch];
};

// ---- host helpers (strip_capi.cu) ------------------------------------------
// Scanner<float, short> + GaussianKernel<float> constants of a geometry, and
// the kernel constants of given model sigmas (pixel pitch pw).
ScannerF make_scanner(const strip_geometry& g);
KernelF make_kernel(double sigma_z, double sigma_dl, float pw);

// ---- launchers (strip_kernels.cu) ----------------------------------------
int tile_smem_bytes(int WYmax, int WS);
int tile_column_stride(int WXmax, int WYmax, int budget);
cudaError_t launch_event_boxes(const ScannerF& s, const float* zu,
                               const float* zd, const float* dl, int64_t n,
                               int4* boxes, int* max_wh, unsigned long long* n_empty,
                               cudaStream_t st);
cudaError_t launch_bin_keys(const Tiling& t, int n_z, int n_y, const int4* boxes,
                            const int64_t* orig, int64_t n, int n_subsets,
                            int* keys, unsigned long long* hist,
                            cudaStream_t st);
cudaError_t launch_bin_scatter(const int* keys, int64_t n, const float* zu,
                               const float* zd, const float* dl,
                               const int64_t* orig,
                               unsigned long long* cursor, float* ozu,
                               float* ozd, float* odl, int64_t* operm,
                               int64_t n_keys, cudaStream_t st);
cudaError_t launch_tile(int op, int mode, int accum, const LaunchArgs& a,
                        cudaStream_t st);
// The events of each work item (binned arrays zu.. perm) reordered into
// ozu.. operm for the column-major windows' banks (k_item_order).
cudaError_t launch_item_order(const ScannerF& s, const Tiling& t, const WorkItem* items,
                              int n_items, const float* zu, const float* zd, const float* dl,
                              const int64_t* perm, float* ozu, float* ozd, float* odl,
                              int64_t* operm, cudaStream_t st);
cudaError_t launch_global(int op, int mode, int accum, const LaunchArgs& a,
                          cudaStream_t st);
// rho_j <- rho_j * acc_j * scale, or acc_j * scale when the accumulator holds
// rho-weighted contributions (weighted: STRIP_MODE_CPU MLEM); acc_j <- 0.
cudaError_t launch_update(float* rho, double* acc, int64_t n_pix, double scale,
                          int weighted, cudaStream_t st);
// rho_out_j = rho_in_j * acc_j, or acc_j when weighted (acc is left as is)
cudaError_t launch_update_out(const float* rho_in, float* rho_out,
                              const double* acc, int64_t n_pix, int weighted,
                              cudaStream_t st);
// Whether MLEM in `mode` accumulates rho-weighted contributions.
inline int mlem_weighted(int mode) { return mode == STRIP_MODE_CPU; }
// out_i = w[perm_i]: caller-order weights into binned order (binary32, the
// precision the adjoint scales its kernel values with)
cudaError_t launch_gather_weights(const int64_t* perm, const double* w,
                                  int64_t n, float* out, cudaStream_t st);
// Sets the batched tile kernel's dynamic shared-memory limit (before a
// launch is captured into a graph).
// max_rows: the most box rows of any event of the launch's members; cs:
// their windows' column stride (0: row-major).
cudaError_t tile_batch_reserve_smem(int mode, int accum, int smem_bytes, int max_rows, int cs);
cudaError_t launch_tile_batch(int mode, int accum, const BatchArgs& b,
                              const BatchItem* items, int n_items, int* counter,
                              int smem_bytes, int max_rows, int cs, int sm_count,
                              cudaStream_t st);
cudaError_t launch_update_batch(const BatchUpdateArgs& u, int64_t max_pix,
                                cudaStream_t st);
cudaError_t launch_sensitivity(const ScannerF& s, int five_point, float* out,
                               cudaStream_t st);
cudaError_t launch_debug_sets(const ScannerF& s, const float* zu,
                              const float* zd, const float* dl, int64_t n,
                              int32_t* n_bb, int32_t* n_in, uint64_t* digest,
                              cudaStream_t st);
cudaError_t launch_scale_copy(const double* acc, const float* sens,
                              double* out, int64_t n_pix, cudaStream_t st);
cudaError_t launch_count_work(const ScannerF& s, const float* zu,
                              const float* zd, const float* dl, int64_t n,
                              unsigned long long* out, cudaStream_t st);
cudaError_t launch_fma_peak(int n_sm, int iters, float* out, double* flops,
                            cudaStream_t st);

}  // namespace stripmlem
