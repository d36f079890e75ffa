// C ABI of the strip MLEM library (include/stripmlem.h): contexts, event
// binning, the iteration driver and the projection entry points.  The host
// side owns no arithmetic that decides pixel sets; it only narrows the
// scanner parameters to binary32 exactly as Scanner<float, short> does
// (src/2d/strip/scanner.h:39-67) -- this translation unit is compiled with
// -ffp-contract=off so those few host operations round as the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "stripmlem.h"
#include "strip_internal.h"
#include "strip_ctx.h"

using namespace stripmlem;

namespace {

int fail(strip_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

#define CK(call)                                                         \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess)                                               \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? STRIP_E_NOMEM   \
                                                       : STRIP_E_CUDA,   \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                  __FILE__, __LINE__);                                   \
  } while (0)

}  // namespace

namespace stripmlem {

static int16_t narrow16(int32_t v) { return (int16_t)(uint16_t)(uint32_t)v; }

// Scanner<float, short>(R, L, n_y, n_z, p_h, p_w, s_z, s_dl, c_y, c_z) and
// GaussianKernel<float>(s_z, s_dl): scanner.h:50-67, gaussian_kernel.h:27-33.
ScannerF make_scanner(const strip_geometry& g) {
  ScannerF s;
  s.R = (float)g.radius;
  s.L = (float)g.scintillator_length;
  s.n_y = narrow16(g.n_y_pixels);
  s.n_z = narrow16(g.n_z_pixels);
  s.ph = (float)g.pixel_height;
  s.pw = (float)g.pixel_width;
  s.sz = (float)g.sigma_z;
  s.sdl = (float)g.sigma_dl;
  s.cy = (float)g.center_y;
  s.cz = (float)g.center_z;
  const float size_y = (float)s.n_y * s.ph;
  const float size_z = (float)s.n_z * s.pw;
  s.tl_y = s.cy + size_y / 2.0f;
  s.tl_z = s.cz - size_z / 2.0f;
  s.tl_y_half_h = s.tl_y - s.ph / 2.0f;
  s.tl_z_half_w = s.tl_z + s.pw / 2.0f;
  s.half_L = s.L / 2.0f;
  s.ipsz = 1.0f / (s.sz * s.sz);
  s.ipsdl = 1.0f / (s.sdl * s.sdl);
  s.kc = (float)((1.0 / (2.0 * M_PI * M_PI)) *
                 (double)sqrtf((s.ipsz * s.ipsz) * s.ipsdl));
  s.inv_pw = 1.0f / s.pw;
  s.inv2z = 0.5f / s.ipsz;
  // A column half a pixel or more beyond a run end has q - 9 >=
  // C pw^2 (1/4 + hw) (C = 2 ipsz, hw the run's half width in pixels); the
  // two-test run ends need that margin far above the rounding of q (a few
  // 1e-5): 2e-3 here, which every row meets when sigma_z <= ~22 pixels.
  const double cpw2 = 2.0 * (double)s.ipsz * (double)s.pw * (double)s.pw;
  s.min_closed_hw = (float)std::max(0.0, 2e-3 / cpw2 - 0.25);
  return s;
}

KernelF make_kernel(double sigma_z, double sigma_dl, float pw) {
  KernelF k;
  const float sz = (float)sigma_z, sdl = (float)sigma_dl;
  k.ipsz = 1.0f / (sz * sz);
  k.ipsdl = 1.0f / (sdl * sdl);
  k.kc = (float)((1.0 / (2.0 * M_PI * M_PI)) *
                 (double)sqrtf((k.ipsz * k.ipsz) * k.ipsdl));
  k.c1 = -kLog2e * k.ipsz;
  k.r1 = 2.0f * k.c1 * pw;
  k.r0 = k.c1 * pw * pw;
  k.q = (float)exp2(2.0 * (double)k.c1 * (double)pw * (double)pw);
  k.q3 = (float)exp2(6.0 * (double)k.c1 * (double)pw * (double)pw);
  k.q4 = (float)exp2(8.0 * (double)k.c1 * (double)pw * (double)pw);
  k.lg2kc = (float)log2((double)k.kc);
  return k;
}

}  // namespace stripmlem

// Each work item's events ordered for the column-major windows' banks
// (k_item_order; a build-time switch for comparisons).
#ifndef STRIP_ITEM_ORDER
#define STRIP_ITEM_ORDER 1
#endif
// With the item size chosen per binning, the last STRIP_TAIL_WAVES waves of
// a subset's work items (by events, one wave = two CTAs per SM, each with a
// full item) are cut into STRIP_TAIL_PIECES pieces each, so the launch's last
// CTAs finish close together without the per-item cost of small items
// everywhere (0: off).
#ifndef STRIP_TAIL_PIECES
#define STRIP_TAIL_PIECES 4
#endif
#ifndef STRIP_TAIL_WAVES
#define STRIP_TAIL_WAVES 1
#endif

namespace {

template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

int set_device(strip_ctx* ctx) {
  CK(cudaSetDevice(ctx->device));
  return STRIP_OK;
}

// Chooses the tile size and halos for the largest event box, within the
// shared memory of 2 CTAs per SM; when even 16 x 16 tiles leave the halos too
// large for that, within the shared memory of one CTA per SM (half the
// resident warps, but every event stays on the shared-memory path) before
// the halos shrink and the largest boxes fall to the global-memory path.
Tiling choose_tiling(const strip_ctx* ctx, int max_w, int max_h) {
  const int n_z = ctx->s.n_z, n_y = ctx->s.n_y;
  const int wide_budget = ctx->smem_optin - 2048;  // static shared memory
  // two CTAs per SM: 2 x (dynamic + ~1.1 KB static + 1 KB reserved) within
  // the SM's 228 KB
  int budget = std::min(ctx->smem_optin, kNarrowSmemBytes);
  Tiling t{};
  int TX = ctx->tile_pref, TY = ctx->tile_pref;
  int HX = max_w / 2 + 2, HY = max_h / 2 + 2;
  for (;;) {
    const int WX = std::min(n_z, TX + 2 * HX), WY = std::min(n_y, TY + 2 * HY);
    // Row stride = 2 (mod 32): the 32 lanes of a warp walk runs on 32
    // different rows, so a lane's bank is (row * WS + column) mod 32; of all
    // residues, 2 (and 30) spread the middle-out-ranked rows of realistic
    // ellipses over the banks best (fewest shared-memory wavefronts in a
    // simulation over events of the 800 x 400 geometry).
    const int WS = WX + ((2 - WX % 32) + 32) % 32;
    const int bytes = tile_smem_bytes(WY, WS);
    if (bytes <= budget || (HX <= 8 && HY <= 8)) {
      t.TX = TX;
      t.TY = TY;
      t.HX = HX;
      t.HY = HY;
      t.WXmax = WX;
      t.WYmax = WY;
      t.WS = WS;
      t.smem_bytes = bytes;
      break;
    }
    if (TX > 16 || TY > 16) {
      TX = TY = 16;
      continue;
    }
    if (budget < wide_budget) {
      budget = wide_budget;
      TX = TY = ctx->tile_pref;
      continue;
    }
    if (HX >= HY) HX = HX * 3 / 4; else HY = HY * 3 / 4;
  }
  // column-major windows where they fit the same budget (fewer shared-memory
  // bank conflicts in the walks)
  t.cs = tile_column_stride(t.WXmax, t.WYmax, budget);
  if (t.cs) t.smem_bytes = 2 * t.WXmax * t.cs * 4;
  t.ntx = (n_z + t.TX - 1) / t.TX;
  t.nty = (n_y + t.TY - 1) / t.TY;
  t.n_tiles = t.ntx * t.nty;
  return t;
}

// Sorts events (device arrays; `orig` maps them to the caller's indices or is
// null for identity) into (subset, tile) bins and builds the work items.
// On success the context owns the new binned arrays.
int bin_events(strip_ctx* ctx, const float* zu, const float* zd,
               const float* dl, const int64_t* orig, int64_t n,
               int n_subsets) {
  cudaStream_t st = ctx->stream;
  cudaEventRecord(ctx->ev0, st);
  int4* boxes = nullptr;
  int* keys = nullptr;
  int* d_wh = nullptr;
  unsigned long long* d_empty = nullptr;
  unsigned long long* d_hist = nullptr;
  float *ozu = nullptr, *ozd = nullptr, *odl = nullptr;
  int64_t* operm = nullptr;
  auto cleanup = [&]() {
    ev_free(ctx, boxes);
    ev_free(ctx, keys);
    dfree(d_wh);
    dfree(d_empty);
    dfree(d_hist);
    ev_free(ctx, ozu);
    ev_free(ctx, ozd);
    ev_free(ctx, odl);
    ev_free(ctx, operm);
  };
  int rc = STRIP_OK;
#define CKB(call)                                                        \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      rc = fail(ctx, e_ == cudaErrorMemoryAllocation ? STRIP_E_NOMEM     \
                                                     : STRIP_E_CUDA,     \
                "%s: %s", #call, cudaGetErrorString(e_));                \
      cleanup();                                                         \
      return rc;                                                         \
    }                                                                    \
  } while (0)
  const size_t nn = (size_t)std::max<int64_t>(n, 1);
  CKB(ev_alloc(ctx, &boxes, nn * sizeof(int4)));
  CKB(ev_alloc(ctx, &keys, nn * sizeof(int)));
  CKB(cudaMalloc(&d_wh, 2 * sizeof(int)));
  CKB(cudaMalloc(&d_empty, sizeof(unsigned long long)));
  CKB(cudaMemsetAsync(d_wh, 0, 2 * sizeof(int), st));
  CKB(cudaMemsetAsync(d_empty, 0, sizeof(unsigned long long), st));
  CKB(launch_event_boxes(ctx->s, zu, zd, dl, n, boxes, d_wh, d_empty, st));
  int wh[2] = {0, 0};
  unsigned long long n_empty = 0;
  CKB(cudaMemcpyAsync(wh, d_wh, sizeof wh, cudaMemcpyDeviceToHost, st));
  CKB(cudaMemcpyAsync(&n_empty, d_empty, sizeof n_empty,
                      cudaMemcpyDeviceToHost, st));
  CKB(cudaStreamSynchronize(st));

  Tiling t = choose_tiling(ctx, wh[0], wh[1]);
  t.max_rows = wh[1];
  const int n_keys = n_subsets * (t.n_tiles + 1);
  CKB(cudaMalloc(&d_hist, (size_t)n_keys * sizeof(unsigned long long)));
  CKB(cudaMemsetAsync(d_hist, 0, (size_t)n_keys * sizeof(unsigned long long),
                      st));
  CKB(launch_bin_keys(t, ctx->s.n_z, ctx->s.n_y, boxes, orig, n, n_subsets,
                      keys, d_hist, st));
  std::vector<unsigned long long> hist(n_keys), offs(n_keys);
  CKB(cudaMemcpyAsync(hist.data(), d_hist, n_keys * sizeof(unsigned long long),
                      cudaMemcpyDeviceToHost, st));
  CKB(cudaStreamSynchronize(st));
  unsigned long long total = 0;
  for (int k = 0; k < n_keys; ++k) {
    offs[k] = total;
    total += hist[k];
  }
  const size_t nb = (size_t)std::max<unsigned long long>(total, 1);
  CKB(ev_alloc(ctx, &ozu, nb * sizeof(float)));
  CKB(ev_alloc(ctx, &ozd, nb * sizeof(float)));
  CKB(ev_alloc(ctx, &odl, nb * sizeof(float)));
  CKB(ev_alloc(ctx, &operm, nb * sizeof(int64_t)));
  CKB(cudaMemcpyAsync(d_hist, offs.data(), n_keys * sizeof(unsigned long long),
                      cudaMemcpyHostToDevice, st));
  CKB(launch_bin_scatter(keys, n, zu, zd, dl, orig, d_hist, ozu, ozd, odl,
                         operm, n_keys, st));

  // Work items: chunks of each (subset, tile) bin, sized for >= ~8 waves and
  // at most kMaxItemEvents events (the fixed-point window accumulator's
  // bound).  Chunk k of every tile precedes chunk k + 1 of any tile, so the
  // CTAs resident at one time work on different tiles and their window
  // flushes rarely hit the same pixels together.
  std::vector<WorkItem> items;
  std::vector<int> ib(n_subsets), ic(n_subsets);
  std::vector<int64_t> gb(n_subsets), gc(n_subsets);
  const int64_t per_sub = (int64_t)(total / (unsigned long long)n_subsets) + 1;
  const int64_t target = (int64_t)ctx->sm_count * 2 * 8;
  const int64_t chunk =
      ctx->item_events > 0
          ? std::min<int64_t>(kMaxItemEvents, ctx->item_events)
          : std::min<int64_t>(kMaxItemEvents,
                              std::max<int64_t>(2048, per_sub / target + 1));
  for (int sb = 0; sb < n_subsets; ++sb) {
    ib[sb] = (int)items.size();
    for (int64_t round = 0;; ++round) {
      bool any = false;
      for (int tile = 0; tile < t.n_tiles; ++tile) {
        const int key = sb * (t.n_tiles + 1) + tile;
        const int64_t c = (int64_t)hist[key] - round * chunk;
        if (c <= 0) continue;
        const int64_t m = std::min(c, chunk);
        items.push_back(WorkItem{tile, (int32_t)m, (int64_t)offs[key] + round * chunk});
        any = true;
      }
      if (!any) break;
    }
    if (STRIP_TAIL_PIECES > 1 && ctx->item_events <= 0 && ctx->tail_split) {
      // the subset's last items, back to about one wave's worth of events
      // (an item size set by hand is kept as set)
      const int64_t tail = (int64_t)STRIP_TAIL_WAVES * ctx->sm_count * 2 * chunk;
      size_t k = items.size();
      int64_t acc = 0;
      while (k > (size_t)ib[sb] && acc + items[k - 1].count <= tail) acc += items[--k].count;
      if (k < items.size()) {
        // piece p of every item before piece p + 1 of any: the CTAs resident
        // at one time still work on different tiles
        std::vector<WorkItem> cut;
        for (int pc = 0; pc < STRIP_TAIL_PIECES; ++pc)
          for (size_t i = k; i < items.size(); ++i) {
            const WorkItem w = items[i];
            const int64_t piece = (w.count + STRIP_TAIL_PIECES - 1) / STRIP_TAIL_PIECES;
            const int64_t o = pc * piece;
            if (o < w.count)
              cut.push_back(WorkItem{w.tile, (int32_t)std::min<int64_t>(piece, w.count - o),
                                     w.begin + o});
          }
        items.resize(k);
        items.insert(items.end(), cut.begin(), cut.end());
      }
    }
    ic[sb] = (int)items.size() - ib[sb];
    const int gkey = sb * (t.n_tiles + 1) + t.n_tiles;
    gb[sb] = (int64_t)offs[gkey];
    gc[sb] = (int64_t)hist[gkey];
  }
  WorkItem* d_items = nullptr;
  CKB(cudaMalloc(&d_items, std::max<size_t>(items.size(), 1) * sizeof(WorkItem)));
  float* d_ihist = nullptr;
  {
    const size_t hb = std::max<size_t>(items.size(), 1) * sizeof(float);
    cudaError_t e = cudaMalloc(&d_ihist, hb);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_ihist, 0, hb, st);
    if (e != cudaSuccess) {
      cudaFree(d_items);
      cudaFree(d_ihist);
      CKB(e);
    }
  }
  if (!items.empty()) {
    cudaError_t e = cudaMemcpyAsync(d_items, items.data(),
                                    items.size() * sizeof(WorkItem),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      cudaFree(d_items);
      cudaFree(d_ihist);
      CKB(e);
    }
  }
  // column-major windows: each item's events in quads of middle-row classes
  // (k_item_order); the binned arrays are replaced by the ordered ones
  if (t.cs != 0 && !items.empty() && STRIP_ITEM_ORDER) {
    // the boxes and keys are done with: the pool hands their memory to the
    // ordered arrays
    ev_free(ctx, boxes);
    ev_free(ctx, keys);
    float *qzu = nullptr, *qzd = nullptr, *qdl = nullptr;
    int64_t* qperm = nullptr;
    cudaError_t e = ev_alloc(ctx, &qzu, nb * sizeof(float));
    if (e == cudaSuccess) e = ev_alloc(ctx, &qzd, nb * sizeof(float));
    if (e == cudaSuccess) e = ev_alloc(ctx, &qdl, nb * sizeof(float));
    if (e == cudaSuccess) e = ev_alloc(ctx, &qperm, nb * sizeof(int64_t));
    if (e == cudaSuccess)
      e = launch_item_order(ctx->s, t, d_items, (int)items.size(), ozu, ozd, odl, operm, qzu,
                            qzd, qdl, qperm, st);
    if (e != cudaSuccess) {
      ev_free(ctx, qzu);
      ev_free(ctx, qzd);
      ev_free(ctx, qdl);
      ev_free(ctx, qperm);
      cudaStreamSynchronize(st);
      cudaFree(d_items);
      cudaFree(d_ihist);
      CKB(e);
    }
    std::swap(ozu, qzu);
    std::swap(ozd, qzd);
    std::swap(odl, qdl);
    std::swap(operm, qperm);
    ev_free(ctx, qzu);
    ev_free(ctx, qzd);
    ev_free(ctx, qdl);
    ev_free(ctx, qperm);
  }
  cudaEventRecord(ctx->ev1, st);
  {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      cudaFree(d_items);
      cudaFree(d_ihist);
      CKB(e);
    }
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);

  // commit
  ev_free(ctx, ctx->d_zu);
  ev_free(ctx, ctx->d_zd);
  ev_free(ctx, ctx->d_dl);
  ev_free(ctx, ctx->d_perm);
  dfree(ctx->d_items);
  dfree(ctx->d_item_hist);
  ctx->d_item_hist = d_ihist;
  ctx->d_zu = ozu;
  ctx->d_zd = ozd;
  ctx->d_dl = odl;
  ctx->d_perm = operm;
  ozu = ozd = odl = nullptr;
  operm = nullptr;
  ctx->d_items = d_items;
  ctx->items.swap(items);
  ctx->sub_item_begin.swap(ib);
  ctx->sub_item_count.swap(ic);
  ctx->sub_g_begin.swap(gb);
  ctx->sub_g_count.swap(gc);
  ctx->n_binned = (int64_t)total;
  ev_free(ctx, ctx->d_wbin);  // sized for the previous binning
  ctx->n_subsets = n_subsets;
  ctx->t = t;
  ctx->max_w = wh[0];
  ctx->max_h = wh[1];
  int64_t n_ovf = 0;
  for (int sb = 0; sb < n_subsets; ++sb) n_ovf += ctx->sub_g_count[sb];
  strip_stats& S = ctx->stats;
  S.n_events = ctx->n_events;
  S.n_empty = (int64_t)n_empty;
  S.n_overflow = n_ovf;
  S.n_tiles_z = t.ntx;
  S.n_tiles_y = t.nty;
  S.tile_z = t.TX;
  S.tile_y = t.TY;
  S.halo_z = t.HX;
  S.halo_y = t.HY;
  S.n_work_items = (int32_t)ctx->items.size();
  S.max_item_events = 0;
  for (const WorkItem& w : ctx->items)
    S.max_item_events = std::max(S.max_item_events, w.count);
  S.n_subsets = n_subsets;
  S.max_box_w = wh[0];
  S.max_box_h = wh[1];
  S.smem_bytes = t.smem_bytes;
  S.last_setup_ms = ms;
  cleanup();
  return STRIP_OK;
#undef CKB
}

int ensure_sens5(strip_ctx* ctx) {
  if (ctx->d_sens5) return STRIP_OK;
  CK(cudaMalloc(&ctx->d_sens5, ctx->n_pix * sizeof(float)));
  CK(launch_sensitivity(ctx->s, 1, ctx->d_sens5, ctx->stream));
  return STRIP_OK;
}

int check_ready(strip_ctx* ctx) {
  if (!ctx) return STRIP_E_INVALID;
  if (ctx->n_subsets <= 0)
    return fail(ctx, STRIP_E_STATE, "no events: call strip_set_events first");
  return STRIP_OK;
}

LaunchArgs base_args(strip_ctx* ctx) {
  LaunchArgs a{};
  a.s = ctx->s;
  a.k = make_kernel(ctx->g.sigma_z, ctx->g.sigma_dl, ctx->s.pw);
  a.t = ctx->t;
  a.zu = ctx->d_zu;
  a.zd = ctx->d_zd;
  a.dl = ctx->d_dl;
  a.perm = ctx->d_perm;
  a.rho = ctx->d_rho;
  a.acc = ctx->d_acc;
  a.status = ctx->d_status;
  a.grab = ctx->grab;
  // GaussianKernel values are at most kc / sqrt(2 R^2 ipsz): E <= 1 and
  // a'Sa >= ipsz (ap^2 + aq^2) >= 2 R^2 ipsz sec^4
  a.kbound = (float)((double)a.k.kc /
                     ((double)ctx->s.R * std::sqrt(2.0 * (double)a.k.ipsz)) * 1.02);
  a.n_fallback = ctx->d_fallback;
  return a;
}

// The work items and global-path range of OSEM subset sb, with the items'
// unweighted-window statistics (MLEM).
void set_subset(strip_ctx* ctx, LaunchArgs& a, int sb) {
  a.items = ctx->d_items + ctx->sub_item_begin[sb];
  a.item_hist = ctx->d_item_hist ? ctx->d_item_hist + ctx->sub_item_begin[sb] : nullptr;
  a.n_items = ctx->sub_item_count[sb];
  a.g_begin = ctx->sub_g_begin[sb];
  a.g_count = ctx->sub_g_count[sb];
}

// Re-bins the resident events for n_subsets OSEM subsets when the current
// binning differs: the binned arrays become the input, perm keeps the
// caller's indices.
int ensure_binning(strip_ctx* ctx, int n_subsets) {
  if (n_subsets == ctx->n_subsets) return STRIP_OK;
  float* zu = ctx->d_zu;
  float* zd = ctx->d_zd;
  float* dl = ctx->d_dl;
  int64_t* pm = ctx->d_perm;
  ctx->d_zu = ctx->d_zd = ctx->d_dl = nullptr;
  ctx->d_perm = nullptr;
  const int rc = bin_events(ctx, zu, zd, dl, pm, ctx->n_binned, n_subsets);
  if (rc != STRIP_OK) {
    ctx->d_zu = zu;
    ctx->d_zd = zd;
    ctx->d_dl = dl;
    ctx->d_perm = pm;
    return rc;
  }
  ev_free(ctx, zu);
  ev_free(ctx, zd);
  ev_free(ctx, dl);
  ev_free(ctx, pm);
  return STRIP_OK;
}

// Runs op over every subset's work items and global-path events.
int run_all(strip_ctx* ctx, int op, int mode, LaunchArgs a) {
  for (int sb = 0; sb < ctx->n_subsets; ++sb) {
    a.items = ctx->d_items + ctx->sub_item_begin[sb];
    a.n_items = ctx->sub_item_count[sb];
    a.g_begin = ctx->sub_g_begin[sb];
    a.g_count = ctx->sub_g_count[sb];
    CK(launch_tile(op, mode, ctx->accum, a, ctx->stream));
    CK(launch_global(op, mode, ctx->accum, a, ctx->stream));
  }
  return STRIP_OK;
}

}  // namespace

extern "C" {

int strip_ctx_create(const strip_geometry* g, int device, strip_ctx** out) {
  if (!g || !out) return STRIP_E_INVALID;
  *out = nullptr;
  if (g->n_y_pixels <= 0 || g->n_z_pixels <= 0 || g->n_y_pixels > 32767 ||
      g->n_z_pixels > 32767 || !(g->pixel_height > 0) ||
      !(g->pixel_width > 0) || !(g->sigma_z > 0) || !(g->sigma_dl > 0) ||
      !(g->radius > 0))
    return STRIP_E_INVALID;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev <= 0) {
    cudaGetLastError();
    return STRIP_E_NODEVICE;
  }
  if (device < 0 || device >= n_dev) return STRIP_E_INVALID;
  strip_ctx* ctx = new (std::nothrow) strip_ctx();
  if (!ctx) return STRIP_E_NOMEM;
  ctx->device = device;
  ctx->g = *g;
  ctx->s = make_scanner(*g);
  ctx->n_pix = (int64_t)ctx->s.n_y * ctx->s.n_z;
  int rc = STRIP_OK;
  do {
    if (cudaSetDevice(device) != cudaSuccess) { rc = STRIP_E_CUDA; break; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { rc = STRIP_E_CUDA; break; }
    snprintf(ctx->devname, sizeof ctx->devname, "%s", prop.name);
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_optin = (int)prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { rc = STRIP_E_CUDA; break; }
    {
      // the event buffers' pool keeps its memory between binnings (no
      // release to the device until the context is destroyed)
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.handleTypes = cudaMemHandleTypeNone;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = device;
      if (cudaMemPoolCreate(&ctx->pool, &props) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
      } else {
        cudaGetLastError();
        ctx->pool = nullptr;  // plain allocations
      }
    }
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) { rc = STRIP_E_CUDA; break; }
    if (cudaMalloc(&ctx->d_rho, ctx->n_pix * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&ctx->d_acc_own, ctx->n_pix * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&ctx->d_status, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->d_fallback, sizeof(unsigned long long)) != cudaSuccess) {
      rc = STRIP_E_NOMEM;
      break;
    }
    ctx->d_acc = ctx->d_acc_own;
    std::vector<float> ones((size_t)ctx->n_pix, 1.0f);  // reconstruction.h:59
    if (cudaMemcpy(ctx->d_rho, ones.data(), ctx->n_pix * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(ctx->d_acc, 0, ctx->n_pix * sizeof(double)) != cudaSuccess ||
        cudaMemset(ctx->d_status, 0, sizeof(int)) != cudaSuccess ||
        cudaMemset(ctx->d_fallback, 0, sizeof(unsigned long long)) != cudaSuccess) {
      rc = STRIP_E_CUDA;
      break;
    }
  } while (0);
  if (rc != STRIP_OK) {
    cudaGetLastError();
    strip_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return STRIP_OK;
}

int strip_ctx_destroy(strip_ctx* ctx) {
  if (!ctx) return STRIP_E_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  dfree(ctx->d_rho);
  dfree(ctx->d_acc_own);
  dfree(ctx->d_sens5);
  ev_free(ctx, ctx->d_wbin);
  ev_free(ctx, ctx->d_zu);
  ev_free(ctx, ctx->d_zd);
  ev_free(ctx, ctx->d_dl);
  ev_free(ctx, ctx->d_perm);
  dfree(ctx->d_items);
  dfree(ctx->d_item_hist);
  dfree(ctx->d_fallback);
  dfree(ctx->d_status);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (cudaEvent_t ev : ctx->tile_marks) cudaEventDestroy(ev);
  release_staging(ctx);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);  // the pool's frees above
    cudaStreamDestroy(ctx->stream);
  }
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  delete ctx;
  return STRIP_OK;
}

int strip_last_error(const strip_ctx* ctx, char* buf, size_t size) {
  if (!ctx || !buf || size == 0) return STRIP_E_INVALID;
  snprintf(buf, size, "%s", ctx->err.c_str());
  return STRIP_OK;
}

int strip_device_name(const strip_ctx* ctx, char* buf, size_t size) {
  if (!ctx || !buf || size == 0) return STRIP_E_INVALID;
  snprintf(buf, size, "%s", ctx->devname);
  return STRIP_OK;
}

int strip_set_accumulation(strip_ctx* ctx, int accum) {
  if (!ctx) return STRIP_E_INVALID;
  if (accum < STRIP_ACCUM_FP32 || accum > STRIP_ACCUM_FP64)
    return fail(ctx, STRIP_E_INVALID, "unknown accumulation %d", accum);
  ctx->accum = accum;
  return STRIP_OK;
}

int strip_get_stats(const strip_ctx* ctx, strip_stats* out) {
  if (!ctx || !out) return STRIP_E_INVALID;
  *out = ctx->stats;
  return STRIP_OK;
}

int strip_set_events_device(strip_ctx* ctx, const float* zu, const float* zd,
                            const float* dl, int64_t n, int n_subsets) {
  if (!ctx) return STRIP_E_INVALID;
  if (n < 0 || (n > 0 && (!zu || !zd || !dl)) || n_subsets < 1 ||
      n_subsets > 4096)
    return fail(ctx, STRIP_E_INVALID, "invalid events (n=%lld, subsets=%d)",
                (long long)n, n_subsets);
  if (int rc = set_device(ctx)) return rc;
  ctx->n_events = n;
  return bin_events(ctx, zu, zd, dl, nullptr, n, n_subsets);
}

int strip_set_events(strip_ctx* ctx, const float* zu, const float* zd,
                     const float* dl, int64_t n, int n_subsets) {
  if (!ctx) return STRIP_E_INVALID;
  if (n < 0 || (n > 0 && (!zu || !zd || !dl)) || n_subsets < 1 ||
      n_subsets > 4096)
    return fail(ctx, STRIP_E_INVALID, "invalid events (n=%lld, subsets=%d)",
                (long long)n, n_subsets);
  if (int rc = set_device(ctx)) return rc;
  float* d = nullptr;
  const size_t bytes = (size_t)std::max<int64_t>(n, 1) * sizeof(float);
  CK(ev_alloc(ctx, &d, 3 * bytes));
  float* dzu = d;
  float* dzd = d + std::max<int64_t>(n, 1);
  float* ddl = d + 2 * std::max<int64_t>(n, 1);
  if (n > 0) {
    const auto t0 = std::chrono::steady_clock::now();
    if (int rc = upload_soa(ctx, zu, zd, dl, n, dzu, dzd, ddl)) {
      ev_free(ctx, d);
      return rc;
    }
    ctx->stats.last_upload_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  ctx->n_events = n;
  int rc = bin_events(ctx, dzu, dzd, ddl, nullptr, n, n_subsets);
  ev_free(ctx, d);
  return rc;
}

int strip_set_responses(strip_ctx* ctx, const float* t, int64_t n,
                        int n_subsets) {
  if (!ctx) return STRIP_E_INVALID;
  if (n < 0 || (n > 0 && !t) || n_subsets < 1 || n_subsets > 4096)
    return fail(ctx, STRIP_E_INVALID, "invalid responses");
  if (int rc = set_device(ctx)) return rc;
  // the triples go to the device as they are; a kernel splits them
  // (AoS -> SoA, gpu_events_soa.h:18-22)
  return upload_responses(ctx, t, n, n_subsets);
}

int strip_set_image(strip_ctx* ctx, const float* rho) {
  if (!ctx || !rho) return STRIP_E_INVALID;
  for (int64_t j = 0; j < ctx->n_pix; ++j)
    if (!(rho[j] >= 0.0f) || !std::isfinite(rho[j]))
      return fail(ctx, STRIP_E_INVALID,
                  "strip_set_image: pixel %lld is negative or not finite",
                  (long long)j);
  if (int rc = set_device(ctx)) return rc;
  CK(cudaMemcpyAsync(ctx->d_rho, rho, ctx->n_pix * sizeof(float),
                     cudaMemcpyHostToDevice, ctx->stream));
  // a new image: the next pass over each item starts from a weighted window
  if (ctx->d_item_hist && !ctx->items.empty())
    CK(cudaMemsetAsync(ctx->d_item_hist, 0, ctx->items.size() * sizeof(float),
                       ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_get_image(strip_ctx* ctx, float* rho) {
  if (!ctx || !rho) return STRIP_E_INVALID;
  if (int rc = set_device(ctx)) return rc;
  CK(cudaMemcpyAsync(rho, ctx->d_rho, ctx->n_pix * sizeof(float),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_get_sensitivity(strip_ctx* ctx, int five_point, float* out) {
  if (!ctx || !out) return STRIP_E_INVALID;
  if (int rc = set_device(ctx)) return rc;
  float* d = nullptr;
  CK(cudaMalloc(&d, ctx->n_pix * sizeof(float)));
  cudaError_t e = launch_sensitivity(ctx->s, five_point ? 1 : 0, d, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, d, ctx->n_pix * sizeof(float),
                        cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  CK(e);
  return STRIP_OK;
}

int strip_iterate(strip_ctx* ctx, int n_iter, int mode, int n_subsets,
                  int first, strip_progress_cb progress, void* user) {
  if (int rc = check_ready(ctx)) return rc;
  if (n_iter < 0 || (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU) ||
      n_subsets < 1 || n_subsets > 4096)
    return fail(ctx, STRIP_E_INVALID, "invalid iterate arguments");
  if (int rc = set_device(ctx)) return rc;
  if (int rc = ensure_binning(ctx, n_subsets)) return rc;
  if (mode == STRIP_MODE_GPU)
    if (int rc = ensure_sens5(ctx)) return rc;
  LaunchArgs a = base_args(ctx);
  a.sens = (mode == STRIP_MODE_GPU) ? ctx->d_sens5 : nullptr;
  int launches = 0;
  // one event pair per tile launch, for the tile kernel's device time
  const size_t n_marks = (size_t)n_iter * ctx->n_subsets;
  while (ctx->tile_marks.size() < 2 * n_marks) {
    cudaEvent_t ev;
    CK(cudaEventCreate(&ev));
    ctx->tile_marks.push_back(ev);
  }
  size_t mark = 0;
  CK(cudaMemsetAsync(ctx->d_fallback, 0, sizeof(unsigned long long), ctx->stream));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  for (int it = 0; it < n_iter; ++it) {
    if (progress) {
      CK(cudaStreamSynchronize(ctx->stream));
      progress(first + it, 0, user);
    }
    for (int sb = 0; sb < ctx->n_subsets; ++sb) {
      set_subset(ctx, a, sb);
      CK(cudaEventRecord(ctx->tile_marks[2 * mark], ctx->stream));
      CK(launch_tile(OP_MLEM, mode, ctx->accum, a, ctx->stream));
      CK(cudaEventRecord(ctx->tile_marks[2 * mark + 1], ctx->stream));
      ++mark;
      CK(launch_global(OP_MLEM, mode, ctx->accum, a, ctx->stream));
      CK(launch_update(ctx->d_rho, ctx->d_acc, ctx->n_pix,
                       (double)ctx->n_subsets, mlem_weighted(mode), ctx->stream));
      launches += (a.n_items > 0) + (a.g_count > 0) + 1;
    }
    if (progress) {
      CK(cudaStreamSynchronize(ctx->stream));
      if (progress(first + it, 1, user)) {
        ++it;
        break;
      }
    }
  }
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  unsigned long long n_fb = 0;
  CK(cudaMemcpyAsync(&n_fb, ctx->d_fallback, sizeof(n_fb), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->stats.n_fallback = (int64_t)n_fb;
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  double tile_ms = 0;
  for (size_t m = 0; m < mark; ++m) {
    float t = 0;
    if (cudaEventElapsedTime(&t, ctx->tile_marks[2 * m],
                             ctx->tile_marks[2 * m + 1]) == cudaSuccess)
      tile_ms += t;
  }
  ctx->stats.last_iterate_ms = ms;
  ctx->stats.last_tile_ms = tile_ms;
  ctx->stats.kernel_launches = launches;
  return STRIP_OK;
}

int strip_set_accumulator(strip_ctx* ctx, double* d_acc) {
  if (!ctx) return STRIP_E_INVALID;
  if (int rc = set_device(ctx)) return rc;
  if (d_acc) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, d_acc) != cudaSuccess ||
        at.type != cudaMemoryTypeDevice || at.device != ctx->device) {
      cudaGetLastError();
      return fail(ctx, STRIP_E_INVALID,
                  "strip_set_accumulator: not device memory of this context's device");
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->d_acc = d_acc ? d_acc : ctx->d_acc_own;
  CK(cudaMemsetAsync(ctx->d_acc, 0, ctx->n_pix * sizeof(double), ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_accumulate(strip_ctx* ctx, int mode, int n_subsets, int subset) {
  if (int rc = check_ready(ctx)) return rc;
  if ((mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU) || n_subsets < 1 ||
      n_subsets > 4096 || subset < 0 || subset >= n_subsets)
    return fail(ctx, STRIP_E_INVALID, "invalid accumulate arguments");
  if (int rc = set_device(ctx)) return rc;
  if (int rc = ensure_binning(ctx, n_subsets)) return rc;
  if (mode == STRIP_MODE_GPU)
    if (int rc = ensure_sens5(ctx)) return rc;
  LaunchArgs a = base_args(ctx);
  a.sens = (mode == STRIP_MODE_GPU) ? ctx->d_sens5 : nullptr;
  set_subset(ctx, a, subset);
  CK(cudaMemsetAsync(ctx->d_fallback, 0, sizeof(unsigned long long), ctx->stream));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  CK(launch_tile(OP_MLEM, mode, ctx->accum, a, ctx->stream));
  CK(launch_global(OP_MLEM, mode, ctx->accum, a, ctx->stream));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->stats.last_iterate_ms = ms;
  ctx->stats.last_tile_ms = ms;
  ctx->stats.kernel_launches = (a.n_items > 0) + (a.g_count > 0);
  ctx->acc_mode = mode;
  return STRIP_OK;
}

int strip_update(strip_ctx* ctx, double scale) {
  if (!ctx) return STRIP_E_INVALID;
  if (!(scale > 0) || !std::isfinite(scale))
    return fail(ctx, STRIP_E_INVALID, "invalid update scale");
  if (int rc = set_device(ctx)) return rc;
  CK(launch_update(ctx->d_rho, ctx->d_acc, ctx->n_pix, scale,
                   mlem_weighted(ctx->acc_mode), ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

}  // extern "C"

namespace {

bool valid_sigmas(double sz, double sdl) {
  return sz > 0 && sdl > 0 && std::isfinite(sz) && std::isfinite(sdl);
}

// The device-buffer cores of the projections: enqueue on the context stream,
// no synchronisation.
int forward_dev(strip_ctx* ctx, const float* d_rho, double sz, double sdl,
                int mode, double* d_y) {
  if (mode == STRIP_MODE_GPU)
    if (int rc = ensure_sens5(ctx)) return rc;
  CK(cudaMemsetAsync(d_y, 0, ctx->n_events * sizeof(double), ctx->stream));
  LaunchArgs a = base_args(ctx);
  a.k = make_kernel(sz, sdl, ctx->s.pw);
  a.rho = d_rho;
  a.sens = (mode == STRIP_MODE_GPU) ? ctx->d_sens5 : nullptr;
  a.y_out = d_y;
  return run_all(ctx, OP_FORWARD, mode, a);
}

int adjoint_dev(strip_ctx* ctx, const double* d_w, double sz, double sdl,
                int mode, double* d_g) {
  if (mode == STRIP_MODE_GPU)
    if (int rc = ensure_sens5(ctx)) return rc;
  CK(cudaMemsetAsync(d_g, 0, ctx->n_pix * sizeof(double), ctx->stream));
  // the weights in binned order (read contiguously by the kernels)
  if (!ctx->d_wbin && ctx->n_binned > 0)
    CK(ev_alloc(ctx, &ctx->d_wbin, ctx->n_binned * sizeof(float)));
  CK(launch_gather_weights(ctx->d_perm, d_w, ctx->n_binned, ctx->d_wbin,
                           ctx->stream));
  LaunchArgs a = base_args(ctx);
  a.k = make_kernel(sz, sdl, ctx->s.pw);
  a.acc = d_g;
  a.wf_in = ctx->d_wbin;
  // GaussianKernel values are at most kc / sqrt(2 R^2 ipsz): E <= 1 and
  // a'Sa >= ipsz (ap^2 + aq^2) >= 2 R^2 ipsz sec^4
  a.kbound = (float)((double)a.k.kc /
                     ((double)ctx->s.R * std::sqrt(2.0 * (double)a.k.ipsz)) * 1.02);
  if (int rc = run_all(ctx, OP_ADJOINT, mode, a)) return rc;
  if (mode == STRIP_MODE_GPU)
    CK(launch_scale_copy(d_g, ctx->d_sens5, d_g, ctx->n_pix, ctx->stream));
  return STRIP_OK;
}

int grad_dev(strip_ctx* ctx, const float* d_rho, const double* d_w, double sz,
             double sdl, double* d_out2) {
  CK(cudaMemsetAsync(d_out2, 0, 2 * sizeof(double), ctx->stream));
  LaunchArgs a = base_args(ctx);
  a.k = make_kernel(sz, sdl, ctx->s.pw);
  a.rho = d_rho;
  a.w_in = d_w;
  a.grad_out = d_out2;
  a.sz = sz;
  a.sdl = sdl;
  return run_all(ctx, OP_GRAD, STRIP_MODE_CPU, a);
}

// Device scratch of a host-buffer call, freed on every path.
struct Scratch {
  std::vector<void*> p;
  ~Scratch() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  cudaError_t get(T** out, int64_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<int64_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) p.push_back(q);
    *out = static_cast<T*>(q);
    return e;
  }
};

}  // namespace

extern "C" {

int strip_forward_device(strip_ctx* ctx, const float* d_rho, double sigma_z,
                         double sigma_dl, int mode, double* d_y) {
  if (int rc = check_ready(ctx)) return rc;
  if (!d_rho || !d_y || !valid_sigmas(sigma_z, sigma_dl) ||
      (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU))
    return fail(ctx, STRIP_E_INVALID, "invalid forward arguments");
  if (int rc = set_device(ctx)) return rc;
  if (int rc = forward_dev(ctx, d_rho, sigma_z, sigma_dl, mode, d_y)) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_adjoint_device(strip_ctx* ctx, const double* d_w, double sigma_z,
                         double sigma_dl, int mode, double* d_g) {
  if (int rc = check_ready(ctx)) return rc;
  if (!d_w || !d_g || !valid_sigmas(sigma_z, sigma_dl) ||
      (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU))
    return fail(ctx, STRIP_E_INVALID, "invalid adjoint arguments");
  if (int rc = set_device(ctx)) return rc;
  if (int rc = adjoint_dev(ctx, d_w, sigma_z, sigma_dl, mode, d_g)) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_grad_sigma_device(strip_ctx* ctx, const float* d_rho,
                            const double* d_w, double sigma_z,
                            double sigma_dl, double* d_grad) {
  if (int rc = check_ready(ctx)) return rc;
  if (!d_rho || !d_w || !d_grad || !valid_sigmas(sigma_z, sigma_dl))
    return fail(ctx, STRIP_E_INVALID, "invalid grad_sigma arguments");
  if (int rc = set_device(ctx)) return rc;
  if (int rc = grad_dev(ctx, d_rho, d_w, sigma_z, sigma_dl, d_grad)) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_forward(strip_ctx* ctx, const float* rho, double sigma_z,
                  double sigma_dl, int mode, double* y) {
  if (int rc = check_ready(ctx)) return rc;
  if (!rho || !y || !valid_sigmas(sigma_z, sigma_dl) ||
      (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU))
    return fail(ctx, STRIP_E_INVALID, "invalid forward arguments");
  if (int rc = set_device(ctx)) return rc;
  Scratch sc;
  float* d_img;
  double* d_y;
  CK(sc.get(&d_img, ctx->n_pix));
  CK(sc.get(&d_y, ctx->n_events));
  CK(cudaMemcpyAsync(d_img, rho, ctx->n_pix * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  if (int rc = forward_dev(ctx, d_img, sigma_z, sigma_dl, mode, d_y)) return rc;
  CK(cudaMemcpyAsync(y, d_y, ctx->n_events * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_adjoint(strip_ctx* ctx, const double* w, double sigma_z,
                  double sigma_dl, int mode, double* g) {
  if (int rc = check_ready(ctx)) return rc;
  if (!w || !g || !valid_sigmas(sigma_z, sigma_dl) ||
      (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU))
    return fail(ctx, STRIP_E_INVALID, "invalid adjoint arguments");
  if (int rc = set_device(ctx)) return rc;
  Scratch sc;
  double* d_w;
  double* d_g;
  CK(sc.get(&d_w, ctx->n_events));
  CK(sc.get(&d_g, ctx->n_pix));
  CK(cudaMemcpyAsync(d_w, w, ctx->n_events * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (int rc = adjoint_dev(ctx, d_w, sigma_z, sigma_dl, mode, d_g)) return rc;
  CK(cudaMemcpyAsync(g, d_g, ctx->n_pix * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_grad_sigma(strip_ctx* ctx, const float* rho, const double* w,
                     double sigma_z, double sigma_dl, double* d_sigma_z,
                     double* d_sigma_dl) {
  if (int rc = check_ready(ctx)) return rc;
  if (!rho || !w || !d_sigma_z || !d_sigma_dl || !valid_sigmas(sigma_z, sigma_dl))
    return fail(ctx, STRIP_E_INVALID, "invalid grad_sigma arguments");
  if (int rc = set_device(ctx)) return rc;
  Scratch sc;
  float* d_img;
  double* d_w;
  double* d_g;
  CK(sc.get(&d_img, ctx->n_pix));
  CK(sc.get(&d_w, ctx->n_events));
  CK(sc.get(&d_g, 2));
  CK(cudaMemcpyAsync(d_img, rho, ctx->n_pix * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(d_w, w, ctx->n_events * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (int rc = grad_dev(ctx, d_img, d_w, sigma_z, sigma_dl, d_g)) return rc;
  double g[2];
  CK(cudaMemcpyAsync(g, d_g, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *d_sigma_z = g[0];
  *d_sigma_dl = g[1];
  return STRIP_OK;
}

int strip_count_work(strip_ctx* ctx, int64_t* n_bb, int64_t* n_in,
                     int64_t* n_nonempty) {
  if (int rc = check_ready(ctx)) return rc;
  if (int rc = set_device(ctx)) return rc;
  unsigned long long* d = nullptr;
  CK(cudaMalloc(&d, 3 * sizeof(unsigned long long)));
  unsigned long long h[3] = {0, 0, 0};
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof h, ctx->stream);
  if (e == cudaSuccess)
    e = launch_count_work(ctx->s, ctx->d_zu, ctx->d_zd, ctx->d_dl,
                          ctx->n_binned, d, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  CK(e);
  if (n_bb) *n_bb = (int64_t)h[0];
  if (n_in) *n_in = (int64_t)h[1];
  if (n_nonempty) *n_nonempty = (int64_t)h[2];
  return STRIP_OK;
}

int strip_probe_fp32_peak(int device, double* tflops) {
  if (!tflops) return STRIP_E_INVALID;
  strip_ctx* ctx = nullptr;  // for CK (no message storage)
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev <= 0) {
    cudaGetLastError();
    return STRIP_E_NODEVICE;
  }
  CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  float* out = nullptr;
  CK(cudaMalloc(&out, prop.multiProcessorCount * 4 * sizeof(float)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0, flops = 0;
  cudaError_t err = cudaSuccess;
  for (int rep = 0; rep < 4 && err == cudaSuccess; ++rep) {
    cudaEventRecord(e0, 0);
    err = launch_fma_peak(prop.multiProcessorCount, 4096, out, &flops, 0);
    cudaEventRecord(e1, 0);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  CK(err);
  *tflops = best;
  return STRIP_OK;
}

int strip_debug_scale_item_stats(strip_ctx* ctx, float factor) {
  if (!ctx || !(factor > 0.0f) || !std::isfinite(factor)) return STRIP_E_INVALID;
  if (int rc = set_device(ctx)) return rc;
  if (!ctx->d_item_hist || ctx->items.empty()) return STRIP_OK;
  std::vector<float> h(ctx->items.size());
  CK(cudaMemcpyAsync(h.data(), ctx->d_item_hist, h.size() * sizeof(float),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (float& v : h) v *= factor;
  CK(cudaMemcpyAsync(ctx->d_item_hist, h.data(), h.size() * sizeof(float),
                     cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int strip_debug_pixel_sets(strip_ctx* ctx, const float* zu, const float* zd,
                           const float* dl, int64_t n, int32_t* n_bb,
                           int32_t* n_in, uint64_t* digest) {
  if (!ctx) return STRIP_E_INVALID;
  if (n < 0 || (n > 0 && (!zu || !zd || !dl)))
    return fail(ctx, STRIP_E_INVALID, "invalid events");
  if (n == 0) return STRIP_OK;
  if (int rc = set_device(ctx)) return rc;
  char* d = nullptr;
  const size_t fb = n * sizeof(float);
  const size_t need = 3 * fb + 2 * n * sizeof(int32_t) + n * sizeof(uint64_t) + 64;
  CK(cudaMalloc(&d, need));
  float* dzu = (float*)d;
  float* dzd = dzu + n;
  float* ddl = dzd + n;
  uint64_t* ddg = (uint64_t*)(((uintptr_t)(ddl + n) + 15) & ~(uintptr_t)15);
  int32_t* dbb = (int32_t*)(ddg + n);
  int32_t* din = dbb + n;
  cudaError_t e = cudaMemcpyAsync(dzu, zu, fb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dzd, zd, fb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ddl, dl, fb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = launch_debug_sets(ctx->s, dzu, dzd, ddl, n, dbb, din, ddg, ctx->stream);
  if (e == cudaSuccess && n_bb) e = cudaMemcpyAsync(n_bb, dbb, n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && n_in) e = cudaMemcpyAsync(n_in, din, n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && digest) e = cudaMemcpyAsync(digest, ddg, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  CK(e);
  return STRIP_OK;
}

}  // extern "C"

// ---- internal entry points for strip_batch.cu (strip_ctx.h) -------------
namespace stripmlem {

int ctx_fail(strip_ctx* ctx, int code, const char* msg) {
  return fail(ctx, code, "%s", msg);
}

cudaError_t ev_alloc_bytes(strip_ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (ctx->pool) return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 16), ctx->pool,
                                                ctx->stream);
  return cudaMalloc(p, std::max<size_t>(bytes, 16));
}

void ev_free_ptr(strip_ctx* ctx, void* p) {
  if (!p) return;
  if (ctx->pool)
    cudaFreeAsync(p, ctx->stream);
  else
    cudaFree(p);
}

int ctx_prepare_mlem(strip_ctx* ctx, int mode) {
  if (int rc = check_ready(ctx)) return rc;
  if (int rc = set_device(ctx)) return rc;
  if (int rc = ensure_binning(ctx, 1)) return rc;
  if (mode == STRIP_MODE_GPU)
    if (int rc = ensure_sens5(ctx)) return rc;
  return STRIP_OK;
}

LaunchArgs ctx_mlem_args(strip_ctx* ctx, int mode) {
  LaunchArgs a = base_args(ctx);
  a.sens = (mode == STRIP_MODE_GPU) ? ctx->d_sens5 : nullptr;
  if (ctx->sub_item_count.empty()) {
    a.items = ctx->d_items;
    a.n_items = 0;
  } else {
    set_subset(ctx, a, 0);
  }
  return a;
}

int ctx_rebin(strip_ctx* ctx, int tile) {
  if (int rc = check_ready(ctx)) return rc;
  if (int rc = set_device(ctx)) return rc;
  ctx->tile_pref = tile;
  const int n_subsets = ctx->n_subsets;
  ctx->n_subsets = -1;  // force a new binning at the same subset count
  const int rc = ensure_binning(ctx, n_subsets);
  if (rc != STRIP_OK) ctx->n_subsets = n_subsets;
  return rc;
}

}  // namespace stripmlem
