// The strip context (opaque in include/stripmlem.h) and the internal entry
// points strip_batch.cu uses.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "stripmlem.h"
#include "strip_internal.h"

struct strip_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // stream-ordered pool of the event-sized buffers (uploads, binning
  // scratch, binned events): it keeps freed memory for the next binning, so
  // a new set of events costs no device allocations or unmappings
  cudaMemPool_t pool = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  char devname[256] = {0};
  int sm_count = 148;
  int smem_optin = 227 * 1024;
  strip_geometry g{};
  stripmlem::ScannerF s{};
  int accum = STRIP_ACCUM_KAHAN;
  int64_t n_pix = 0;
  float* d_rho = nullptr;
  double* d_acc = nullptr;      // accumulator in use (own or the caller's)
  double* d_acc_own = nullptr;  // the context's own accumulator
  int acc_mode = STRIP_MODE_CPU;  // mode of the last strip_accumulate
  int tile_pref = 32;  // tile edge in pixels (autotuned or 32)
  int grab = 32;       // events a warp takes per counter step (autotuned or 32)
  int item_events = 0;  // largest work item in events (0: chosen per binning)
  bool tail_split = true;  // cut the last wave of items into pieces (binning)
  float* d_sens5 = nullptr;
  float* d_wbin = nullptr;  // adjoint weights in binned order (n_binned, binary32)
  // binned events
  int64_t n_events = 0;   // as given by the caller
  int64_t n_binned = 0;   // events with a non-empty box
  float* d_zu = nullptr;
  float* d_zd = nullptr;
  float* d_dl = nullptr;
  int64_t* d_perm = nullptr;
  int n_subsets = 0;
  stripmlem::Tiling t{};
  int max_w = 0, max_h = 0;
  std::vector<stripmlem::WorkItem> items;
  stripmlem::WorkItem* d_items = nullptr;
  std::vector<int> sub_item_begin, sub_item_count;
  std::vector<int64_t> sub_g_begin, sub_g_count;
  int* d_status = nullptr;
  // per work item: the unweighted window statistic of the last pass (see
  // LaunchArgs::item_hist); zeroed by a new binning and by strip_set_image
  float* d_item_hist = nullptr;
  unsigned long long* d_fallback = nullptr;  // events rerun in a weighted window
  std::vector<cudaEvent_t> tile_marks;
  // pinned staging buffers of the host -> device event uploads, one stream
  // and event each (strip_upload.cu)
  std::vector<void*> stage_buf;
  std::vector<cudaStream_t> stage_stream;
  std::vector<cudaEvent_t> stage_event;
  strip_stats stats{};
  std::string err;
};

namespace stripmlem {

// Records msg as the context's last error and returns code.
int ctx_fail(strip_ctx* ctx, int code, const char* msg);
// Event-sized device buffers from the context's pool (stream-ordered on the
// context's stream; plain cudaMalloc / cudaFree without a pool).
cudaError_t ev_alloc_bytes(strip_ctx* ctx, void** p, size_t bytes);
void ev_free_ptr(strip_ctx* ctx, void* p);
template <class T>
cudaError_t ev_alloc(strip_ctx* ctx, T** p, size_t bytes) {
  return ev_alloc_bytes(ctx, reinterpret_cast<void**>(p), bytes);
}
template <class T>
void ev_free(strip_ctx* ctx, T*& p) {
  ev_free_ptr(ctx, p);
  p = nullptr;
}
// Device selected, events binned for plain MLEM (one subset), the 5-point
// sensitivity present for STRIP_MODE_GPU.
int ctx_prepare_mlem(strip_ctx* ctx, int mode);
// Launch arguments of one MLEM step of the (single) subset.
LaunchArgs ctx_mlem_args(strip_ctx* ctx, int mode);
// Re-bins the events with `tile` x `tile` pixel tiles.
int ctx_rebin(strip_ctx* ctx, int tile);

// strip_upload.cu: host arrays to the device through pinned staging buffers
// filled by several host threads (straight copies for pinned memory).
// upload_soa copies n floats of each array; upload_responses copies n
// triples, splits them on the device and bins them (strip_set_events_device).
int upload_soa(strip_ctx* ctx, const float* zu, const float* zd, const float* dl,
               int64_t n, float* d_zu, float* d_zd, float* d_dl);
int upload_responses(strip_ctx* ctx, const float* zu_zd_dl, int64_t n, int n_subsets);
void release_staging(strip_ctx* ctx);

}  // namespace stripmlem
