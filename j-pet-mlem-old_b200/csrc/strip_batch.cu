// Batched reconstructions and the schedule autotuner (include/stripmlem.h:
// strip_batch_*, strip_autotune).
//
// A batch advances several contexts -- each with its own geometry, events and
// image -- together: one MLEM step is a tile launch of its own for every
// member with at least two work items per SM, spread over side streams, beside
// one persistent launch per window class over the work items of the smaller
// members (k_tile_batch: CTAs pull items from a global counter, largest
// first), then the global-path launches of members that have overflow events
// and one update launch over all images; the step is captured once as a CUDA
// graph and replayed.  The reference runs one
// reconstruction per process (reconstruction_cmd.cpp:105-301); there is no
// batched counterpart.
//
// The autotuner times one MLEM backprojection of a context's own events for
// each candidate schedule -- pixel tile edge x events a warp takes per
// counter step -- and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <functional>
#include <new>
#include <string>
#include <vector>

#include "strip_ctx.h"

using namespace stripmlem;

// Windows up to this size let two CTAs share an SM.
constexpr int kNarrowSmem = kNarrowSmemBytes;
// Work-item classes: narrow / wide windows, row-major / column-major.
constexpr int kClasses = 4;
inline int class_stride(int c) { return (c & 2) ? kColumnStride : 0; }
// Members with at least this many work items per SM get a tile launch of
// their own (k_tile, arguments in constant parameter space) instead of
// joining the persistent launch, whose per-member arguments are indexed at
// run time and cost registers; the own launches run on kSideStreams streams
// forked from the batch stream, beside the persistent launches that fill
// their tails.
#ifndef STRIP_BATCH_SPLIT_PER_SM
#define STRIP_BATCH_SPLIT_PER_SM 2
#endif
#ifndef STRIP_BATCH_STREAMS
#define STRIP_BATCH_STREAMS 4
#endif
// Members are binned without the cut last wave: the persistent CTAs balance
// the small members' items, and the side streams overlap the own launches'
// tails (measured on 64 instances: 984 Mevent*iter/s unsplit, 938 split).
#ifndef STRIP_BATCH_UNSPLIT
#define STRIP_BATCH_UNSPLIT 1
#endif
constexpr int kSideStreams = STRIP_BATCH_STREAMS;

struct strip_batch {
  int device = 0;
  int mode = STRIP_MODE_CPU;
  int accum = STRIP_ACCUM_KAHAN;
  int sm_count = 148;
  std::vector<strip_ctx*> members;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  BatchArgs* args = nullptr;  // host copy of the kernel parameters (~20 KB)
  // Work items in four classes: members whose windows fit two CTAs per SM
  // and wide-window members (one CTA per SM), each with row-major or
  // column-major windows (class = wide + 2 * column-major).  Each class is one
  // persistent launch, so a wide member does not halve the occupancy of the
  // others.  Class c owns items [cls_begin[c], cls_begin[c] + cls_count[c]).
  BatchItem* d_items = nullptr;
  int n_items = 0;
  int cls_begin[kClasses] = {}, cls_count[kClasses] = {}, cls_smem[kClasses] = {};
  int cls_rows[kClasses] = {};  // the most box rows of a class's events
  int* d_counter = nullptr;  // one counter per class
  // members with a tile launch of their own, and the side stream of each
  std::vector<int> own, own_stream;
  int n_side = 0;
  cudaStream_t side[kSideStreams] = {};
  cudaEvent_t fork = nullptr, join[kSideStreams] = {};
  int64_t n_events = 0;
  int n_work_items = 0;  // of all members, own launches included
  int launches_per_step = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double last_ms = 0;
  std::string err;
};

namespace {

int bfail(strip_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

#define BCK(call)                                                             \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? STRIP_E_NOMEM         \
                                                      : STRIP_E_CUDA,         \
                   std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

void release(strip_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_counter) cudaFree(b->d_counter);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->fork) cudaEventDestroy(b->fork);
  for (int s = 0; s < kSideStreams; ++s) {
    if (b->join[s]) cudaEventDestroy(b->join[s]);
    if (b->side[s]) cudaStreamDestroy(b->side[s]);
  }
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b->args;
  delete b;
}

// One step on the batch stream: counter reset, the own tile launches of the
// large members on the side streams beside the persistent tile launches of
// the others, the members' global-path launches, the batched update.
int enqueue_step(strip_batch* b) {
  BCK(cudaMemsetAsync(b->d_counter, 0, kClasses * sizeof(int), b->stream));
  if (b->n_side > 0) {
    BCK(cudaEventRecord(b->fork, b->stream));
    for (int s = 0; s < b->n_side; ++s) BCK(cudaStreamWaitEvent(b->side[s], b->fork, 0));
    for (size_t k = 0; k < b->own.size(); ++k)
      BCK(launch_tile(OP_MLEM, b->mode, b->accum, b->args->member[b->own[k]],
                      b->side[b->own_stream[k]]));
    for (int s = 0; s < b->n_side; ++s) BCK(cudaEventRecord(b->join[s], b->side[s]));
  }
  for (int c = 0; c < kClasses; ++c)
    if (b->cls_count[c] > 0)
      BCK(launch_tile_batch(b->mode, b->accum, *b->args,
                            b->d_items + b->cls_begin[c], b->cls_count[c],
                            b->d_counter + c, b->cls_smem[c], b->cls_rows[c],
                            class_stride(c), b->sm_count, b->stream));
  for (int s = 0; s < b->n_side; ++s) BCK(cudaStreamWaitEvent(b->stream, b->join[s], 0));
  BatchUpdateArgs u{};
  u.n = (int)b->members.size();
  u.weighted = mlem_weighted(b->mode);
  u.scale = 1.0;
  int64_t max_pix = 0;
  for (int m = 0; m < u.n; ++m) {
    const LaunchArgs& a = b->args->member[m];
    if (a.g_count > 0)
      BCK(launch_global(OP_MLEM, b->mode, b->accum, a, b->stream));
    u.rho[m] = b->members[m]->d_rho;
    u.acc[m] = b->members[m]->d_acc;
    u.n_pix[m] = b->members[m]->n_pix;
    max_pix = std::max(max_pix, u.n_pix[m]);
  }
  BCK(launch_update_batch(u, max_pix, b->stream));
  return STRIP_OK;
}

}  // namespace

extern "C" {

int strip_batch_create(strip_ctx* const* members, int n_members, int mode,
                       strip_batch** out) {
  if (!members || !out || n_members <= 0 || n_members > kMaxBatch ||
      (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU))
    return STRIP_E_INVALID;
  *out = nullptr;
  for (int m = 0; m < n_members; ++m) {
    if (!members[m]) return STRIP_E_INVALID;
    for (int k = 0; k < m; ++k)
      if (members[k] == members[m]) return STRIP_E_INVALID;
    if (members[m]->device != members[0]->device ||
        members[m]->accum != members[0]->accum)
      return ctx_fail(members[m], STRIP_E_INVALID,
                      "strip_batch_create: members differ in device or accumulation");
  }
  strip_batch* b = new (std::nothrow) strip_batch();
  if (!b) return STRIP_E_NOMEM;
  b->args = new (std::nothrow) BatchArgs();
  if (!b->args) {
    delete b;
    return STRIP_E_NOMEM;
  }
  b->device = members[0]->device;
  b->mode = mode;
  b->accum = members[0]->accum;
  b->sm_count = members[0]->sm_count;
  b->members.assign(members, members + n_members);
  int rc = STRIP_OK;
  std::vector<BatchItem> items;
  std::vector<std::pair<int, int>> own;  // (work items, member)
  for (int m = 0; m < n_members && rc == STRIP_OK; ++m) {
    strip_ctx* c = members[m];
    rc = ctx_prepare_mlem(c, mode);
    if (rc != STRIP_OK) {
      b->err = "member " + std::to_string(m) + ": " + c->err;
      break;
    }
    if (STRIP_BATCH_UNSPLIT && c->tail_split) {
      c->tail_split = false;
      rc = ctx_rebin(c, c->tile_pref);
      if (rc != STRIP_OK) {
        b->err = "member " + std::to_string(m) + ": " + c->err;
        break;
      }
    }
    b->args->member[m] = ctx_mlem_args(c, mode);
    const bool own_launch =
        b->args->member[m].n_items >= STRIP_BATCH_SPLIT_PER_SM * b->sm_count;
    const int cls = (c->t.smem_bytes > kNarrowSmem) + (c->t.cs != 0 ? 2 : 0);
    b->cls_smem[cls] = std::max(b->cls_smem[cls], c->t.smem_bytes);
    b->cls_rows[cls] = std::max(b->cls_rows[cls], c->t.max_rows);
    b->n_events += c->n_events;
    b->n_work_items += b->args->member[m].n_items;
    if (own_launch && b->args->member[m].n_items > 0) {
      own.emplace_back(b->args->member[m].n_items, m);
      b->launches_per_step += 1 + (b->args->member[m].g_count > 0);
      continue;
    }
    for (int i = 0; i < b->args->member[m].n_items; ++i) {
      const WorkItem& w = c->items[i];
      items.push_back(BatchItem{m, w.tile, w.count, cls, w.begin, i, 0});
    }
    b->launches_per_step += b->args->member[m].g_count > 0;
  }
  if (rc == STRIP_OK) {
    // by class, then largest items first: the persistent CTAs of a class
    // then finish close together
    std::stable_sort(items.begin(), items.end(),
                     [](const BatchItem& x, const BatchItem& y) {
                       return x.pad != y.pad ? x.pad < y.pad : x.count > y.count;
                     });
    b->n_items = (int)items.size();
    for (const BatchItem& it : items) ++b->cls_count[it.pad];
    for (int c = 1; c < kClasses; ++c) b->cls_begin[c] = b->cls_begin[c - 1] + b->cls_count[c - 1];
    b->launches_per_step += 1;
    for (int c = 0; c < kClasses; ++c) b->launches_per_step += b->cls_count[c] > 0;
    // own launches, largest first, each on the side stream with the fewest
    // work items so far
    std::sort(own.begin(), own.end(), std::greater<std::pair<int, int>>());
    int64_t load[kSideStreams] = {};
    b->n_side = std::min<int>(kSideStreams, (int)own.size());
    for (const auto& o : own) {
      const int s = (int)(std::min_element(load, load + b->n_side) - load);
      load[s] += o.first;
      b->own.push_back(o.second);
      b->own_stream.push_back(s);
    }
    do {
      if (cudaSetDevice(b->device) != cudaSuccess) { rc = STRIP_E_CUDA; break; }
      if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
          cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
        rc = STRIP_E_CUDA;
        break;
      }
      for (int s = 0; s < b->n_side && rc == STRIP_OK; ++s)
        if (cudaStreamCreateWithFlags(&b->side[s], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join[s], cudaEventDisableTiming) != cudaSuccess)
          rc = STRIP_E_CUDA;
      if (rc != STRIP_OK) break;
      if (cudaMalloc(&b->d_items, std::max<size_t>(items.size(), 1) * sizeof(BatchItem)) != cudaSuccess ||
          cudaMalloc(&b->d_counter, kClasses * sizeof(int)) != cudaSuccess) {
        rc = STRIP_E_NOMEM;
        break;
      }
      if (!items.empty() &&
          cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(BatchItem),
                     cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = STRIP_E_CUDA;
        break;
      }
      // the members' own streams may still hold work on their buffers
      for (strip_ctx* c : b->members)
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = STRIP_E_CUDA;
      if (rc != STRIP_OK) break;
      // capture one step as a graph (kernel attributes are set beforehand)
      // (each class has its own kernel: 512-thread CTAs for the narrow
      // windows, 1024-thread CTAs for the wide ones, per window layout)
      bool attr_ok = true;
      for (int c = 0; c < kClasses; ++c)
        if (b->cls_count[c] > 0 &&
            tile_batch_reserve_smem(b->mode, b->accum, b->cls_smem[c], b->cls_rows[c],
                                    class_stride(c)) != cudaSuccess)
          attr_ok = false;
      if (!attr_ok ||
          cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = STRIP_E_CUDA;
        break;
      }
      const int erc = enqueue_step(b);
      const cudaError_t ec = cudaStreamEndCapture(b->stream, &b->graph);
      if (erc != STRIP_OK) { rc = erc; break; }
      if (ec != cudaSuccess ||
          cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
        rc = STRIP_E_CUDA;
        break;
      }
    } while (0);
    if (rc != STRIP_OK && b->err.empty()) b->err = cudaGetErrorString(cudaGetLastError());
  }
  if (rc != STRIP_OK) {
    cudaGetLastError();
    for (strip_ctx* c : b->members)
      if (c->err.empty()) c->err = "strip_batch_create: " + b->err;
    release(b);
    return rc;
  }
  *out = b;
  return STRIP_OK;
}

int strip_batch_iterate(strip_batch* b, int n_iter) {
  if (!b || n_iter < 0) return STRIP_E_INVALID;
  BCK(cudaSetDevice(b->device));
  BCK(cudaEventRecord(b->ev0, b->stream));
  for (int it = 0; it < n_iter; ++it) BCK(cudaGraphLaunch(b->exec, b->stream));
  BCK(cudaEventRecord(b->ev1, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  b->last_ms = ms;
  return STRIP_OK;
}

int strip_batch_stats(strip_batch* b, double* last_iterate_ms, int64_t* n_events,
                      int32_t* n_work_items, int32_t* launches_per_iteration) {
  if (!b) return STRIP_E_INVALID;
  if (last_iterate_ms) *last_iterate_ms = b->last_ms;
  if (n_events) *n_events = b->n_events;
  if (n_work_items) *n_work_items = b->n_work_items;
  if (launches_per_iteration) *launches_per_iteration = b->launches_per_step;
  return STRIP_OK;
}

int strip_batch_last_error(strip_batch* b, char* buf, size_t size) {
  if (!b || !buf || size == 0) return STRIP_E_INVALID;
  std::snprintf(buf, size, "%s", b->err.c_str());
  return STRIP_OK;
}

int strip_batch_destroy(strip_batch* b) {
  if (!b) return STRIP_E_INVALID;
  release(b);
  return STRIP_OK;
}

int strip_autotune(strip_ctx* ctx, int mode, strip_tuning* best) {
  if (!ctx || (mode != STRIP_MODE_CPU && mode != STRIP_MODE_GPU))
    return STRIP_E_INVALID;
  if (int rc = ctx_prepare_mlem(ctx, mode)) return rc;
  static const int kTiles[] = {16, 32, 48, 64};
  static const int kGrabs[] = {4, 8, 16, 32};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return ctx_fail(ctx, STRIP_E_CUDA, "strip_autotune: cudaEventCreate failed");
  }
  double* d_scratch = nullptr;  // the backprojections go here, not into acc
  if (cudaMalloc(&d_scratch, ctx->n_pix * sizeof(double)) != cudaSuccess) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ctx_fail(ctx, STRIP_E_NOMEM, "strip_autotune: no memory for the scratch image");
  }
  strip_tuning top{0, 0, 0.0};
  int rc = STRIP_OK;
  for (int tile : kTiles) {
    if ((rc = ctx_rebin(ctx, tile)) != STRIP_OK) break;
    if (mode == STRIP_MODE_GPU && (rc = ctx_prepare_mlem(ctx, mode)) != STRIP_OK) break;
    for (int grab : kGrabs) {
      ctx->grab = grab;
      LaunchArgs a = ctx_mlem_args(ctx, mode);
      a.acc = d_scratch;
      float best_ms = 1e30f;
      for (int rep = 0; rep < 3 && rc == STRIP_OK; ++rep) {  // the first is a warm-up
        cudaError_t e = cudaEventRecord(e0, ctx->stream);
        if (e == cudaSuccess) e = launch_tile(OP_MLEM, mode, ctx->accum, a, ctx->stream);
        if (e == cudaSuccess) e = launch_global(OP_MLEM, mode, ctx->accum, a, ctx->stream);
        if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
          rc = ctx_fail(ctx, STRIP_E_CUDA, cudaGetErrorString(e));
          break;
        }
        if (rep > 0) best_ms = std::min(best_ms, ms);
      }
      if (rc != STRIP_OK) break;
      if (top.tile == 0 || best_ms < top.ms) top = strip_tuning{tile, grab, best_ms};
    }
    if (rc != STRIP_OK) break;
  }
  cudaFree(d_scratch);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != STRIP_OK) return rc;
  ctx->grab = top.grab;
  if (int r2 = ctx_rebin(ctx, top.tile)) return r2;
  if (best) *best = top;
  return STRIP_OK;
}

int strip_set_schedule(strip_ctx* ctx, int tile, int grab) {
  if (!ctx) return STRIP_E_INVALID;
  if (tile < 8 || tile > 128 || grab < 1 || grab > 32)
    return ctx_fail(ctx, STRIP_E_INVALID, "strip_set_schedule: tile in [8, 128], grab in [1, 32]");
  ctx->grab = grab;
  if (ctx->n_subsets <= 0) {  // no events yet: used by the next binning
    ctx->tile_pref = tile;
    return STRIP_OK;
  }
  return ctx_rebin(ctx, tile);
}

int strip_set_item_events(strip_ctx* ctx, int max_events) {
  if (!ctx) return STRIP_E_INVALID;
  if (max_events < 0 || max_events > kMaxItemEvents)
    return ctx_fail(ctx, STRIP_E_INVALID, "strip_set_item_events: 0 or 1..8000 events");
  ctx->item_events = max_events;
  if (ctx->n_subsets <= 0) return STRIP_OK;  // used by the next binning
  return ctx_rebin(ctx, ctx->tile_pref);
}

}  // extern "C"
