// Event input at host-memory bandwidth: the binary event-file reader
// (strip_load_responses_file) and the host -> device path of the event
// setters for pageable host memory.
//
// A plain cudaMemcpy from pageable memory goes through the driver's own small
// staging buffers, one copy at a time, and a single std::ifstream read of a
// 2.4 GB event file into a std::vector runs at one core's memcpy speed before
// the copy even starts.  Here several host threads each own a pinned staging
// buffer and a CUDA stream: a thread fills its buffer with the next chunk
// (pread from the file, or memcpy from the caller's array) and enqueues its
// copy to the device, then fills the buffer again once that copy has
// finished, so the reads of one thread overlap the copies of the others.
// The raw triples land in device memory as they are in the file, and a
// kernel splits them into the z_u / z_d / dl arrays the binning reads.
#include <chrono>
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "strip_ctx.h"

namespace stripmlem {

namespace {

constexpr size_t kStageBytes = size_t(32) << 20;  // one staging buffer
constexpr int kStageThreads = 6;

int upload_fail(strip_ctx* ctx, int code, const std::string& msg) {
  return ctx_fail(ctx, code, msg.c_str());
}

// Pinned staging buffers, streams and events of the context (made once).
int ensure_staging(strip_ctx* ctx) {
  if ((int)ctx->stage_buf.size() == kStageThreads) return STRIP_OK;
  release_staging(ctx);
  for (int t = 0; t < kStageThreads; ++t) {
    void* b = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    if (cudaHostAlloc(&b, kStageBytes, cudaHostAllocPortable) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      if (b) cudaFreeHost(b);
      if (s) cudaStreamDestroy(s);
      cudaGetLastError();
      release_staging(ctx);
      return upload_fail(ctx, STRIP_E_NOMEM, "no pinned memory for the staging buffers");
    }
    ctx->stage_buf.push_back(b);
    ctx->stage_stream.push_back(s);
    ctx->stage_event.push_back(e);
  }
  return STRIP_OK;
}

// Copies `bytes` bytes to d_dst through the staging buffers; fill(off, len,
// buf) writes bytes [off, off + len) of the source into buf and returns
// false on a read error.  Returns a STRIP status.
template <class Fill>
int stage_upload(strip_ctx* ctx, size_t bytes, char* d_dst, const Fill& fill,
                 const char* what) {
  if (bytes == 0) return STRIP_OK;
  if (int rc = ensure_staging(ctx)) return rc;
  const size_t n_chunks = (bytes + kStageBytes - 1) / kStageBytes;
  const int n_threads = (int)std::min<size_t>(kStageThreads, n_chunks);
  std::atomic<size_t> next{0};
  std::atomic<int> read_error{0};
  std::atomic<int> cuda_error{0};
  auto worker = [&](int t) {
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
      cuda_error = 1;
      return;
    }
    char* buf = static_cast<char*>(ctx->stage_buf[t]);
    cudaStream_t st = ctx->stage_stream[t];
    cudaEvent_t ev = ctx->stage_event[t];
    bool pending = false;
    for (;;) {
      const size_t c = next.fetch_add(1);
      if (c >= n_chunks || read_error || cuda_error) break;
      if (pending && cudaEventSynchronize(ev) != cudaSuccess) {  // the buffer is free
        cuda_error = 1;
        break;
      }
      const size_t off = c * kStageBytes, len = std::min(kStageBytes, bytes - off);
      if (!fill(off, len, buf)) {
        read_error = 1;
        break;
      }
      if (cudaMemcpyAsync(d_dst + off, buf, len, cudaMemcpyHostToDevice, st) !=
              cudaSuccess ||
          cudaEventRecord(ev, st) != cudaSuccess) {
        cuda_error = 1;
        break;
      }
      pending = true;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) cuda_error = 1;
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < n_threads; ++t) pool.emplace_back(worker, t);
  worker(0);
  for (auto& th : pool) th.join();
  if (cuda_error) {
    cudaGetLastError();
    return upload_fail(ctx, STRIP_E_CUDA, std::string(what) + ": host to device copy failed");
  }
  if (read_error) return upload_fail(ctx, STRIP_E_INVALID, std::string(what) + ": read failed");
  return STRIP_OK;
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host bytes -> device, straight when the memory is pinned, else staged.
int host_upload(strip_ctx* ctx, const void* src, size_t bytes, char* d_dst,
                const char* what) {
  if (bytes == 0) return STRIP_OK;
  if (is_pinned(src)) {
    if (cudaMemcpyAsync(d_dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      cudaGetLastError();
      return upload_fail(ctx, STRIP_E_CUDA, std::string(what) + ": host to device copy failed");
    }
    return STRIP_OK;
  }
  const char* s = static_cast<const char*>(src);
  return stage_upload(ctx, bytes, d_dst,
                      [s](size_t off, size_t len, char* buf) {
                        std::memcpy(buf, s + off, len);
                        return true;
                      },
                      what);
}

// Triples on the device (3n floats) -> SoA arrays, then the binning of
// strip_set_events_device.
int bin_triples(strip_ctx* ctx, const float* d_aos, int64_t n, int n_subsets) {
  float* d = nullptr;
  const size_t m = (size_t)std::max<int64_t>(n, 1);
  if (ev_alloc(ctx, &d, 3 * m * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return upload_fail(ctx, STRIP_E_NOMEM, "no device memory for the events");
  }
  cudaError_t e = launch_split_triples(d_aos, n, d, d + m, d + 2 * m, ctx->stream);
  int rc = STRIP_OK;
  if (e != cudaSuccess) {
    cudaGetLastError();
    rc = upload_fail(ctx, STRIP_E_CUDA, "splitting the event triples failed");
  } else {
    rc = strip_set_events_device(ctx, d, d + m, d + 2 * m, n, n_subsets);
  }
  ev_free(ctx, d);
  return rc;
}

}  // namespace

void release_staging(strip_ctx* ctx) {
  for (void* b : ctx->stage_buf) cudaFreeHost(b);
  for (cudaStream_t s : ctx->stage_stream) cudaStreamDestroy(s);
  for (cudaEvent_t e : ctx->stage_event) cudaEventDestroy(e);
  ctx->stage_buf.clear();
  ctx->stage_stream.clear();
  ctx->stage_event.clear();
}

int upload_soa(strip_ctx* ctx, const float* zu, const float* zd, const float* dl,
               int64_t n, float* d_zu, float* d_zd, float* d_dl) {
  const size_t bytes = (size_t)n * sizeof(float);
  if (int rc = host_upload(ctx, zu, bytes, reinterpret_cast<char*>(d_zu), "z_u")) return rc;
  if (int rc = host_upload(ctx, zd, bytes, reinterpret_cast<char*>(d_zd), "z_d")) return rc;
  return host_upload(ctx, dl, bytes, reinterpret_cast<char*>(d_dl), "dl");
}

int upload_responses(strip_ctx* ctx, const float* t, int64_t n, int n_subsets) {
  float* d_aos = nullptr;
  const size_t bytes = (size_t)n * 3 * sizeof(float);
  if (ev_alloc(ctx, &d_aos, std::max<size_t>(bytes, 16)) != cudaSuccess) {
    cudaGetLastError();
    return upload_fail(ctx, STRIP_E_NOMEM, "no device memory for the events");
  }
  const auto t0 = std::chrono::steady_clock::now();
  int rc = host_upload(ctx, t, bytes, reinterpret_cast<char*>(d_aos), "responses");
  ctx->stats.last_upload_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (rc == STRIP_OK) rc = bin_triples(ctx, d_aos, n, n_subsets);
  ev_free(ctx, d_aos);
  return rc;
}

}  // namespace stripmlem

extern "C" int strip_load_responses_file(strip_ctx* ctx, const char* path,
                                         int64_t first, int64_t n,
                                         int n_subsets, int64_t* n_loaded) {
  using namespace stripmlem;
  if (!ctx) return STRIP_E_INVALID;
  if (!path || first < 0 || n_subsets < 1 || n_subsets > 4096)
    return ctx_fail(ctx, STRIP_E_INVALID, "strip_load_responses_file: invalid arguments");
  const int fd = open(path, O_RDONLY | O_CLOEXEC);
  if (fd < 0)
    return upload_fail(ctx, STRIP_E_INVALID,
                       std::string("cannot open phantom responses file: ") + path);
  struct stat sb;
  if (fstat(fd, &sb) != 0) {
    close(fd);
    return upload_fail(ctx, STRIP_E_INVALID, std::string("cannot stat ") + path);
  }
  // whole triples only: a trailing partial one ends the reference's reader
  const int64_t in_file = (int64_t)sb.st_size / 12;
  const int64_t avail = std::max<int64_t>(0, in_file - first);
  const int64_t count = n < 0 ? avail : std::min(n, avail);
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    close(fd);
    cudaGetLastError();
    return ctx_fail(ctx, STRIP_E_CUDA, "cudaSetDevice failed");
  }
  posix_fadvise(fd, first * 12, count * 12, POSIX_FADV_SEQUENTIAL);
  float* d_aos = nullptr;
  const size_t bytes = (size_t)count * 12;
  if (ev_alloc(ctx, &d_aos, std::max<size_t>(bytes, 16)) != cudaSuccess) {
    close(fd);
    cudaGetLastError();
    return ctx_fail(ctx, STRIP_E_NOMEM, "no device memory for the events");
  }
  const off_t base = (off_t)first * 12;
  const auto t0 = std::chrono::steady_clock::now();
  int rc = stage_upload(
      ctx, bytes, reinterpret_cast<char*>(d_aos),
      [fd, base](size_t off, size_t len, char* buf) {
        size_t done = 0;
        while (done < len) {
          const ssize_t r = pread(fd, buf + done, len - done, base + (off_t)(off + done));
          if (r < 0 && errno == EINTR) continue;
          if (r <= 0) return false;
          done += (size_t)r;
        }
        return true;
      },
      path);
  close(fd);
  ctx->stats.last_upload_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (rc == STRIP_OK) rc = bin_triples(ctx, d_aos, count, n_subsets);
  ev_free(ctx, d_aos);
  if (rc == STRIP_OK && n_loaded) *n_loaded = count;
  return rc;
}
