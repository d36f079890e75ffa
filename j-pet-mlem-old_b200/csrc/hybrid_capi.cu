// C ABI of the 3D hybrid path (include/hybridmlem.h): context, the host-side
// flattening of the LOR geometry, and the stream-ordered driver of the
// set-up and iteration kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "hybrid_internal.h"
#include "hybridmlem.h"

using namespace hybridmlem;

extern "C" cudaError_t hybridmlem_scan_keep(const int32_t* keep, int64_t* offs, int64_t n,
                                            void* temp, size_t* temp_bytes, cudaStream_t st);

struct hybrid_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int sm_count = 148;
  hybrid_setup setup{};
  GridF g{};
  int64_t n_voxels = 0;
  // geometry
  int32_t n_detectors = 0;
  int64_t n_lors = 0, n_infos = 0;
  std::vector<float> seg;  // 9 floats per LOR
  float4* d_md = nullptr;
  float* d_len = nullptr;
  short2* d_pix = nullptr;
  float* d_pos = nullptr;
  float* d_w_raw = nullptr;  // hits / n_emissions
  float* d_w = nullptr;      // normalised by the sensitivity
  int64_t* d_lbeg = nullptr;
  int64_t* d_lend = nullptr;
  float* d_sens = nullptr;
  double* d_sens_acc = nullptr;
  bool have_sens = false;
  // events
  int64_t n_responses = 0, n_events = 0;
  Frame* d_frames = nullptr;       // kept frame events, response order
  Frame* d_frames_iter = nullptr;  // the same in the iteration kernel's order
  int64_t* d_index = nullptr;
  unsigned long long* d_counts = nullptr;
  // image, z-fast on the device
  float* d_rho_t = nullptr;
  float* d_acc_t = nullptr;
  float* d_tmp = nullptr;  // boundary-layout staging
  float* d_spill = nullptr;  // per-warp weight slabs of k_mlem
  float* d_acc_user = nullptr;  // caller-owned accumulator (hybrid_set_accumulator)
  hybrid_stats stats{};
  std::string err;
};

namespace {

int fail(hybrid_ctx* c, int code, const char* fmt, ...) {
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

template <typename T> void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

inline int64_t lor_index(int64_t first, int64_t second) {
  return first * (first + 1) / 2 + second;
}

// PixelGrid(n_c, n_r, p) / VoxelGrid / GaussianKernel<float> constants.
GridF make_grid(const hybrid_setup& s) {
  GridF g{};
  g.nc = s.n_columns;
  g.nr = s.n_rows;
  g.np = (int16_t)s.n_planes;
  g.p = (float)s.pixel_size;
  g.z_left = (float)s.z_left;
  const float llx = -g.p * (float)g.nc / 2;
  const float lly = -g.p * (float)g.nr / 2;
  g.llc_x = llx + g.p / 2;
  g.llc_y = lly + g.p / 2;
  g.L = (float)s.length;
  const float sz = (float)s.sigma_z, sdl = (float)s.sigma_dl;
  g.ipz = 1 / (sz * sz);
  g.ipdl = 1 / (sdl * sdl);
  g.norm_c = (float)(1 / (2 * M_PI * M_PI) * std::sqrt(g.ipz * g.ipz * g.ipdl));
  g.n_pixels = g.nc * g.nr;
  return g;
}

// LineSegment(start, end) (src/2d/geometry/line_segment.h:18-27).
void make_segment(float sx, float sy, float ex, float ey, float* o) {
  const float vx = ex - sx, vy = ey - sy;
  const float l = std::sqrt(vx * vx + vy * vy);
  o[0] = sx;
  o[1] = sy;
  o[2] = ex;
  o[3] = ey;
  o[4] = (sx + ex) / 2;
  o[5] = (sy + ey) / 2;
  o[6] = vx / l;
  o[7] = vy / l;
  o[8] = std::sqrt(vx * vx + vy * vy);
}

GeometryDev geo_view(const hybrid_ctx* ctx) {
  GeometryDev v;
  v.lor_md = ctx->d_md;
  v.lor_len = ctx->d_len;
  v.pix = ctx->d_pix;
  v.pos = ctx->d_pos;
  v.w = ctx->d_w;
  v.lbeg = ctx->d_lbeg;
  v.lend = ctx->d_lend;
  v.n_lors = ctx->n_lors;
  v.n_infos = ctx->n_infos;
  return v;
}

void free_events(hybrid_ctx* ctx) {
  dfree(ctx->d_frames);
  dfree(ctx->d_frames_iter);
  dfree(ctx->d_index);
  ctx->n_events = 0;
  ctx->n_responses = 0;
}

// The iteration kernel takes the frame events in LOR order: the warps
// resident at one time then work on a few LORs, whose pixel infos, weights
// and image lines they share in L1 and L2 (205.4 against 207.8 ms per
// iteration in response order on the big-barrel workload of 1e7 responses;
// the order of the additions into the volume changes only the binary32
// rounding of the sums).
#ifndef HYBRID_LOR_ORDER
#define HYBRID_LOR_ORDER 1
#endif
int order_for_iterations(hybrid_ctx* ctx) {
  dfree(ctx->d_frames_iter);
  if (!HYBRID_LOR_ORDER || ctx->n_events <= 0) return STRIP_OK;
  if (ctx->n_events > INT32_MAX)
    return fail(ctx, STRIP_E_INVALID, "more than 2^31 - 1 frame events");
  cudaError_t e = cudaMalloc(&ctx->d_frames_iter, ctx->n_events * sizeof(Frame));
  if (e == cudaSuccess)
    e = order_frames_by_lor(ctx->d_frames, (int32_t)ctx->n_events, ctx->n_lors,
                            ctx->d_frames_iter, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    dfree(ctx->d_frames_iter);
    return fail(ctx, e == cudaErrorMemoryAllocation ? STRIP_E_NOMEM : STRIP_E_CUDA,
                "ordering the frame events by LOR: %s", cudaGetErrorString(e));
  }
  return STRIP_OK;
}

const Frame* iter_frames(const hybrid_ctx* ctx) {
  return ctx->d_frames_iter ? ctx->d_frames_iter : ctx->d_frames;
}

void free_geometry(hybrid_ctx* ctx) {
  free_events(ctx);
  dfree(ctx->d_md);
  dfree(ctx->d_len);
  dfree(ctx->d_pix);
  dfree(ctx->d_pos);
  dfree(ctx->d_w_raw);
  dfree(ctx->d_w);
  dfree(ctx->d_lbeg);
  dfree(ctx->d_lend);
  ctx->seg.clear();
  ctx->n_lors = ctx->n_infos = 0;
  ctx->have_sens = false;
}

// Uploads a flattened geometry (host arrays in GeometrySOA order) and
// resets the sensitivity, events and statistics.
int upload_geometry(hybrid_ctx* ctx, int32_t n_detectors, std::vector<float>& seg,
                    const std::vector<int64_t>& lbeg, const std::vector<int64_t>& lend,
                    const std::vector<int16_t>& pix, const std::vector<float>& pos,
                    const std::vector<float>& w, int64_t n_infos) {
  const int64_t n_lors = (int64_t)lbeg.size();
  free_geometry(ctx);
  std::vector<float4> md(n_lors);
  std::vector<float> len(n_lors);
  for (int64_t li = 0; li < n_lors; ++li) {
    const float* sg = seg.data() + li * 9;
    md[li] = make_float4(sg[4], sg[5], sg[6], sg[7]);
    len[li] = sg[8];
  }
  CK(cudaMalloc(&ctx->d_md, n_lors * sizeof(float4)));
  CK(cudaMalloc(&ctx->d_len, n_lors * sizeof(float)));
  CK(cudaMalloc(&ctx->d_lbeg, n_lors * sizeof(int64_t)));
  CK(cudaMalloc(&ctx->d_lend, n_lors * sizeof(int64_t)));
  CK(cudaMalloc(&ctx->d_pix, n_infos * sizeof(short2)));
  CK(cudaMalloc(&ctx->d_pos, n_infos * sizeof(float)));
  CK(cudaMalloc(&ctx->d_w_raw, n_infos * sizeof(float)));
  CK(cudaMalloc(&ctx->d_w, n_infos * sizeof(float)));
  CK(cudaMemcpyAsync(ctx->d_md, md.data(), n_lors * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_len, len.data(), n_lors * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_lbeg, lbeg.data(), n_lors * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_lend, lend.data(), n_lors * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_pix, pix.data(), n_infos * sizeof(short2), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_pos, pos.data(), n_infos * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_w_raw, w.data(), n_infos * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_w, w.data(), n_infos * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->seg.swap(seg);
  ctx->n_detectors = n_detectors;
  ctx->n_lors = n_lors;
  ctx->n_infos = n_infos;
  ctx->stats = hybrid_stats{};
  ctx->stats.n_lors = n_lors;
  ctx->stats.n_pixel_infos = n_infos;
  return STRIP_OK;
}

}  // namespace

extern "C" {

int hybrid_ctx_create(const hybrid_setup* setup, int32_t device, hybrid_ctx** out) {
  if (!setup || !out) return STRIP_E_INVALID;
  *out = nullptr;
  const hybrid_setup& s = *setup;
  if (s.n_columns <= 0 || s.n_rows <= 0 || s.n_planes <= 0 || s.n_columns > 32767 ||
      s.n_rows > 32767 || s.n_planes > 32767 || !(s.pixel_size > 0) || !(s.sigma_z > 0) ||
      !(s.sigma_dl > 0) || !(s.length > 0) || !std::isfinite(s.z_left))
    return STRIP_E_INVALID;
  if ((int64_t)s.n_columns * s.n_rows * s.n_planes >= (int64_t)1 << 31) return STRIP_E_INVALID;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev <= 0) {
    cudaGetLastError();
    return STRIP_E_NODEVICE;
  }
  if (device < 0 || device >= n_dev) return STRIP_E_INVALID;
  hybrid_ctx* ctx = new (std::nothrow) hybrid_ctx();
  if (!ctx) return STRIP_E_NOMEM;
  ctx->device = device;
  ctx->setup = s;
  ctx->g = make_grid(s);
  ctx->n_voxels = (int64_t)s.n_columns * s.n_rows * s.n_planes;
  int rc = STRIP_OK;
  do {
    if (cudaSetDevice(device) != cudaSuccess) { rc = STRIP_E_CUDA; break; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { rc = STRIP_E_CUDA; break; }
    ctx->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
      rc = STRIP_E_CUDA;
      break;
    }
    const size_t vb = ctx->n_voxels * sizeof(float);
    if (cudaMalloc(&ctx->d_rho_t, vb) != cudaSuccess || cudaMalloc(&ctx->d_acc_t, vb) != cudaSuccess ||
        cudaMalloc(&ctx->d_tmp, vb) != cudaSuccess ||
        cudaMalloc(&ctx->d_sens, ctx->g.n_pixels * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&ctx->d_sens_acc, ctx->g.n_pixels * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&ctx->d_counts, 2 * sizeof(unsigned long long)) != cudaSuccess) {
      rc = STRIP_E_NOMEM;
      break;
    }
    // Reconstruction's rho(..., 1) (reconstruction.h:70-75)
    std::vector<float> ones(ctx->n_voxels, 1.0f);
    if (cudaMemcpy(ctx->d_rho_t, ones.data(), vb, cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = STRIP_E_CUDA;
      break;
    }
  } while (0);
  if (rc != STRIP_OK) {
    hybrid_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return STRIP_OK;
}

int hybrid_ctx_destroy(hybrid_ctx* ctx) {
  if (!ctx) return STRIP_E_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_geometry(ctx);
  dfree(ctx->d_sens);
  dfree(ctx->d_sens_acc);
  dfree(ctx->d_counts);
  dfree(ctx->d_rho_t);
  dfree(ctx->d_acc_t);
  dfree(ctx->d_tmp);
  dfree(ctx->d_spill);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return STRIP_OK;
}

const char* hybrid_last_error(const hybrid_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int hybrid_set_geometry_from_matrix(hybrid_ctx* ctx, int32_t n_detectors,
                                    const float* centers_xy, int64_t n_elements,
                                    const uint16_t* lor_a, const uint16_t* lor_b,
                                    const uint16_t* px, const uint16_t* py,
                                    const uint32_t* hits, uint32_t n_emissions,
                                    const int16_t* inactive, int32_t n_inactive) {
  if (!ctx) return STRIP_E_INVALID;
  if (n_detectors <= 0 || n_detectors > 32767 || !centers_xy || n_elements <= 0 || !lor_a ||
      !lor_b || !px || !py || !hits || n_emissions == 0 || n_inactive < 0 ||
      (n_inactive > 0 && !inactive))
    return fail(ctx, STRIP_E_INVALID, "invalid geometry arguments");
  if (ctx->setup.n_columns != ctx->setup.n_rows)
    return fail(ctx, STRIP_E_INVALID, "the matrix geometry needs a square pixel grid");
  if (n_elements >= ((int64_t)1 << 31))
    return fail(ctx, STRIP_E_INVALID, "too many matrix elements");
  CK(cudaSetDevice(ctx->device));
  const int64_t n_lors = lor_index(n_detectors, 0);
  struct El {
    int16_t first, second, x, y;
    uint32_t hits;
  };
  std::vector<El> el(n_elements);
  for (int64_t i = 0; i < n_elements; ++i) {
    if (lor_a[i] >= (uint16_t)n_detectors || lor_b[i] >= (uint16_t)n_detectors)
      return fail(ctx, STRIP_E_INVALID, "element %lld: detector out of range", (long long)i);
    if (px[i] >= (uint16_t)ctx->setup.n_columns || py[i] >= (uint16_t)ctx->setup.n_rows)
      return fail(ctx, STRIP_E_INVALID, "element %lld: pixel out of range", (long long)i);
    const int16_t a = (int16_t)lor_a[i], b = (int16_t)lor_b[i];
    el[i] = El{std::max(a, b), std::min(a, b), (int16_t)px[i], (int16_t)py[i], hits[i]};
  }
  // SparseMatrix::sort_by_lor_n_pixel (sparse_matrix.h:449-454, :585-593)
  std::sort(el.begin(), el.end(), [](const El& a, const El& b) {
    if (a.first != b.first) return a.first < b.first;
    if (a.second != b.second) return a.second < b.second;
    if (a.y != b.y) return a.y < b.y;
    return a.x < b.x;
  });
  std::vector<char> off(n_detectors, 0);
  for (int32_t i = 0; i < n_inactive; ++i)
    if (inactive[i] >= 0 && inactive[i] < n_detectors) off[inactive[i]] = 1;
  std::vector<int64_t> lbeg(n_lors, 0), lend(n_lors, 0);
  std::vector<int16_t> pix(2 * n_elements);
  std::vector<float> w(n_elements), pos(n_elements);
  int64_t cur = -1, index = 0;
  for (const El& e : el) {
    const int64_t li = lor_index(e.first, e.second);
    if (li != cur) {
      if (cur >= 0) lend[cur] = index;
      cur = li;
      lbeg[cur] = index;
    }
    if (n_inactive > 0 && (off[e.first] || off[e.second])) continue;
    pix[2 * index] = e.x;
    pix[2 * index + 1] = e.y;
    w[index] = (float)e.hits / (float)n_emissions;
    ++index;
  }
  lend[cur] = index;
  const int64_t n_infos = index;
  if (n_infos == 0) return fail(ctx, STRIP_E_INVALID, "no active matrix elements");
  // per LOR: the segment between the detector centres and its pixel infos
  // sorted by position along it (geometry_soa.h:135-178)
  std::vector<float> seg(n_lors * 9);
  std::vector<int64_t> indices;
  std::vector<int16_t> sp;
  std::vector<float> sw, spos;
  const GridF& g = ctx->g;
  for (int64_t first = 0; first < n_detectors; ++first) {
    for (int64_t second = 0; second <= first; ++second) {
      const int64_t li = lor_index(first, second);
      float* sg = seg.data() + li * 9;
      make_segment(centers_xy[2 * second], centers_xy[2 * second + 1], centers_xy[2 * first],
                   centers_xy[2 * first + 1], sg);
      const int64_t b = lbeg[li], e = lend[li], n = e - b;
      if (!n) continue;
      indices.resize(n);
      for (int64_t i = 0; i < n; ++i) {
        const int64_t k = b + i;
        const float cx = g.llc_x + (float)pix[2 * k] * g.p;
        const float cy = g.llc_y + (float)pix[2 * k + 1] * g.p;
        pos[k] = ((cx - sg[0]) * sg[6] + (cy - sg[1]) * sg[7]) / sg[8];  // projection_scaled
        indices[i] = k;
      }
      const float* pp = pos.data();
      std::sort(indices.begin(), indices.end(),
                [pp](const int64_t a, const int64_t c) { return pp[a] < pp[c]; });
      sp.resize(2 * n);
      sw.resize(n);
      spos.resize(n);
      for (int64_t i = 0; i < n; ++i) {
        sp[2 * i] = pix[2 * indices[i]];
        sp[2 * i + 1] = pix[2 * indices[i] + 1];
        sw[i] = w[indices[i]];
        spos[i] = pos[indices[i]];
      }
      std::copy(sp.begin(), sp.end(), pix.begin() + 2 * b);
      std::copy(sw.begin(), sw.end(), w.begin() + b);
      std::copy(spos.begin(), spos.end(), pos.begin() + b);
    }
  }
  return upload_geometry(ctx, n_detectors, seg, lbeg, lend, pix, pos, w, n_infos);
}

int hybrid_set_geometry_soa(hybrid_ctx* ctx, int32_t n_detectors, const float* segments,
                            int64_t n_infos, const int16_t* pixels, const float* positions,
                            const float* weights, const uint64_t* lor_begin,
                            const uint64_t* lor_end) {
  if (!ctx) return STRIP_E_INVALID;
  if (n_detectors <= 0 || n_detectors > 32767 || !segments || n_infos <= 0 ||
      n_infos >= ((int64_t)1 << 31) || !pixels || !positions || !weights || !lor_begin ||
      !lor_end)
    return fail(ctx, STRIP_E_INVALID, "invalid geometry arguments");
  CK(cudaSetDevice(ctx->device));
  const int64_t n_lors = lor_index(n_detectors, 0);
  std::vector<float> seg(n_lors * 9);
  std::vector<int64_t> lbeg(n_lors), lend(n_lors);
  for (int64_t li = 0; li < n_lors; ++li) {
    const float* s4 = segments + 4 * li;
    make_segment(s4[0], s4[1], s4[2], s4[3], seg.data() + 9 * li);
    if (lor_begin[li] > lor_end[li] || lor_end[li] > (uint64_t)n_infos)
      return fail(ctx, STRIP_E_INVALID, "LOR %lld: pixel-info range out of bounds",
                  (long long)li);
    lbeg[li] = (int64_t)lor_begin[li];
    lend[li] = (int64_t)lor_end[li];
  }
  std::vector<int16_t> pix(pixels, pixels + 2 * n_infos);
  for (int64_t i = 0; i < n_infos; ++i)
    if (pix[2 * i] < 0 || pix[2 * i] >= ctx->setup.n_columns || pix[2 * i + 1] < 0 ||
        pix[2 * i + 1] >= ctx->setup.n_rows)
      return fail(ctx, STRIP_E_INVALID, "pixel info %lld: pixel out of range", (long long)i);
  std::vector<float> pos(positions, positions + n_infos), w(weights, weights + n_infos);
  return upload_geometry(ctx, n_detectors, seg, lbeg, lend, pix, pos, w, n_infos);
}

int hybrid_get_geometry(hybrid_ctx* ctx, float* seg, int16_t* pix, float* pos, float* weight,
                        int64_t* lbeg, int64_t* lend) {
  if (!ctx) return STRIP_E_INVALID;
  if (!ctx->n_lors) return fail(ctx, STRIP_E_STATE, "no geometry");
  CK(cudaSetDevice(ctx->device));
  if (seg) std::copy(ctx->seg.begin(), ctx->seg.end(), seg);
  const int64_t n = ctx->n_infos, nl = ctx->n_lors;
  if (pix) CK(cudaMemcpyAsync(pix, ctx->d_pix, n * sizeof(short2), cudaMemcpyDeviceToHost, ctx->stream));
  if (pos) CK(cudaMemcpyAsync(pos, ctx->d_pos, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  if (weight) CK(cudaMemcpyAsync(weight, ctx->d_w, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  if (lbeg) CK(cudaMemcpyAsync(lbeg, ctx->d_lbeg, nl * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  if (lend) CK(cudaMemcpyAsync(lend, ctx->d_lend, nl * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int hybrid_set_sensitivity(hybrid_ctx* ctx, int32_t mode, const float* external) {
  if (!ctx) return STRIP_E_INVALID;
  if (!ctx->n_lors) return fail(ctx, STRIP_E_STATE, "set the geometry first");
  if (mode != HYBRID_SENS_CALCULATE && mode != HYBRID_SENS_ONE &&
      mode != HYBRID_SENS_EXTERNAL && mode != HYBRID_SENS_GIVEN)
    return fail(ctx, STRIP_E_INVALID, "unknown sensitivity mode %d", mode);
  if ((mode == HYBRID_SENS_EXTERNAL || mode == HYBRID_SENS_GIVEN) && !external)
    return fail(ctx, STRIP_E_INVALID, "external sensitivity map is null");
  CK(cudaSetDevice(ctx->device));
  const GridF& g = ctx->g;
  if (mode == HYBRID_SENS_CALCULATE) {
    launch_sensitivity(g, ctx->d_pix, ctx->d_w_raw, ctx->n_infos, ctx->d_sens_acc, ctx->d_sens,
                       ctx->stream);
  } else {
    std::vector<float> h(g.n_pixels, 1.0f);
    if (mode != HYBRID_SENS_ONE) std::copy(external, external + g.n_pixels, h.begin());
    CK(cudaMemcpyAsync(ctx->d_sens, h.data(), g.n_pixels * sizeof(float), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  CK(cudaMemcpyAsync(ctx->d_w, ctx->d_w_raw, ctx->n_infos * sizeof(float),
                     cudaMemcpyDeviceToDevice, ctx->stream));
  if (mode != HYBRID_SENS_GIVEN)  // GIVEN: the weights are normalised already
    launch_normalize(g, ctx->d_pix, ctx->d_w, ctx->d_sens, ctx->n_infos, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  free_events(ctx);  // frame events depend on the normalised weights
  ctx->have_sens = true;
  return STRIP_OK;
}

int hybrid_get_sensitivity(hybrid_ctx* ctx, float* sens) {
  if (!ctx || !sens) return STRIP_E_INVALID;
  if (!ctx->have_sens) return fail(ctx, STRIP_E_STATE, "no sensitivity yet");
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(sens, ctx->d_sens, ctx->g.n_pixels * sizeof(float), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int hybrid_set_responses(hybrid_ctx* ctx, const int16_t* first, const int16_t* second,
                         const float* z_up, const float* z_dn, const float* dl, int64_t n) {
  if (!ctx) return STRIP_E_INVALID;
  if (n < 0 || (n > 0 && (!first || !second || !z_up || !z_dn || !dl)))
    return fail(ctx, STRIP_E_INVALID, "invalid responses");
  if (!ctx->have_sens) return fail(ctx, STRIP_E_STATE, "set the geometry and sensitivity first");
  CK(cudaSetDevice(ctx->device));
  free_events(ctx);
  ctx->n_responses = n;
  ctx->stats.n_responses = n;
  ctx->stats.n_events = 0;
  ctx->stats.used_pixels = ctx->stats.used_voxels = 0;
  if (n == 0) return STRIP_OK;
  int16_t *d_a = nullptr, *d_b = nullptr;
  float *d_zu = nullptr, *d_zd = nullptr, *d_dl = nullptr;
  Frame* d_all = nullptr;
  int32_t* d_keep = nullptr;
  int64_t* d_offs = nullptr;
  void* d_tmp = nullptr;
  size_t tmp_bytes = 0;
  int rc = STRIP_OK;
  auto cleanup = [&]() {
    dfree(d_a);
    dfree(d_b);
    dfree(d_zu);
    dfree(d_zd);
    dfree(d_dl);
    dfree(d_all);
    dfree(d_keep);
    dfree(d_offs);
    if (d_tmp) cudaFree(d_tmp);
  };
#define CKR(call)                                                               \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      rc = fail(ctx, e_ == cudaErrorMemoryAllocation ? STRIP_E_NOMEM : STRIP_E_CUDA, \
                "%s: %s", #call, cudaGetErrorString(e_));                       \
      cudaStreamSynchronize(ctx->stream);                                       \
      cleanup();                                                                \
      return rc;                                                                \
    }                                                                           \
  } while (0)
  CKR(cudaMalloc(&d_a, n * sizeof(int16_t)));
  CKR(cudaMalloc(&d_b, n * sizeof(int16_t)));
  CKR(cudaMalloc(&d_zu, n * sizeof(float)));
  CKR(cudaMalloc(&d_zd, n * sizeof(float)));
  CKR(cudaMalloc(&d_dl, n * sizeof(float)));
  CKR(cudaMalloc(&d_all, n * sizeof(Frame)));
  CKR(cudaMalloc(&d_keep, n * sizeof(int32_t)));
  CKR(cudaMalloc(&d_offs, (n + 1) * sizeof(int64_t)));
  CKR(cudaMemcpyAsync(d_a, first, n * sizeof(int16_t), cudaMemcpyHostToDevice, ctx->stream));
  CKR(cudaMemcpyAsync(d_b, second, n * sizeof(int16_t), cudaMemcpyHostToDevice, ctx->stream));
  CKR(cudaMemcpyAsync(d_zu, z_up, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CKR(cudaMemcpyAsync(d_zd, z_dn, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CKR(cudaMemcpyAsync(d_dl, dl, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  launch_frames(ctx->g, geo_view(ctx), d_a, d_b, d_zu, d_zd, d_dl, n, d_all, d_keep, ctx->stream);
  CKR(cudaGetLastError());
  CKR(hybridmlem_scan_keep(d_keep, d_offs, n, nullptr, &tmp_bytes, ctx->stream));
  CKR(cudaMalloc(&d_tmp, tmp_bytes));
  CKR(hybridmlem_scan_keep(d_keep, d_offs, n, d_tmp, &tmp_bytes, ctx->stream));
  int64_t last_off = 0;
  int32_t last_keep = 0;
  CKR(cudaMemcpyAsync(&last_off, d_offs + (n - 1), sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  CKR(cudaMemcpyAsync(&last_keep, d_keep + (n - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CKR(cudaStreamSynchronize(ctx->stream));
  const int64_t kept = last_off + last_keep;
  if (kept > 0) {
    CKR(cudaMalloc(&ctx->d_frames, kept * sizeof(Frame)));
    CKR(cudaMalloc(&ctx->d_index, kept * sizeof(int64_t)));
    launch_compact(d_all, d_keep, d_offs, n, ctx->d_frames, ctx->d_index, ctx->stream);
    CKR(cudaGetLastError());
    launch_event_counts(ctx->d_frames, kept, ctx->d_counts, ctx->stream);
    CKR(cudaGetLastError());
    unsigned long long counts[2] = {0, 0};
    CKR(cudaMemcpyAsync(counts, ctx->d_counts, sizeof counts, cudaMemcpyDeviceToHost, ctx->stream));
    CKR(cudaStreamSynchronize(ctx->stream));
    ctx->stats.used_pixels = (int64_t)counts[0];
    ctx->stats.used_voxels = (int64_t)counts[1];
  }
#undef CKR
  cleanup();
  ctx->n_events = kept;
  ctx->stats.n_events = kept;
  return order_for_iterations(ctx);
}

int hybrid_set_frames(hybrid_ctx* ctx, int64_t n, const int32_t* lor, const int64_t* info_begin,
                      const int64_t* info_end, const int16_t* plane_begin,
                      const int16_t* plane_end, const float* up, const float* right,
                      const float* tan, const float* sec) {
  if (!ctx) return STRIP_E_INVALID;
  if (n < 0 || (n > 0 && (!lor || !info_begin || !info_end || !plane_begin || !plane_end ||
                          !up || !right || !tan || !sec)))
    return fail(ctx, STRIP_E_INVALID, "invalid frame events");
  if (!ctx->n_lors) return fail(ctx, STRIP_E_STATE, "set the geometry first");
  CK(cudaSetDevice(ctx->device));
  std::vector<Frame> h(n);
  std::vector<int64_t> index(n);
  for (int64_t i = 0; i < n; ++i) {
    if (lor[i] < 0 || lor[i] >= ctx->n_lors || info_begin[i] < 0 ||
        info_end[i] > ctx->n_infos || plane_begin[i] < 0 || plane_end[i] > ctx->g.np)
      return fail(ctx, STRIP_E_INVALID, "frame event %lld out of range", (long long)i);
    Frame& f = h[i];
    f.lor = lor[i];
    f.info_begin = (int32_t)info_begin[i];
    f.info_end = (int32_t)info_end[i];
    f.plane_begin = plane_begin[i];
    f.plane_end = plane_end[i];
    f.up = up[i];
    f.right = right[i];
    f.tan = tan[i];
    f.sec = sec[i];
    index[i] = i;
  }
  free_events(ctx);
  ctx->n_responses = n;
  ctx->stats.n_responses = n;
  ctx->stats.n_events = 0;
  ctx->stats.used_pixels = ctx->stats.used_voxels = 0;
  if (n == 0) return STRIP_OK;
  CK(cudaMalloc(&ctx->d_frames, n * sizeof(Frame)));
  CK(cudaMalloc(&ctx->d_index, n * sizeof(int64_t)));
  CK(cudaMemcpyAsync(ctx->d_frames, h.data(), n * sizeof(Frame), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_index, index.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice,
                     ctx->stream));
  launch_event_counts(ctx->d_frames, n, ctx->d_counts, ctx->stream);
  CK(cudaGetLastError());
  unsigned long long counts[2] = {0, 0};
  CK(cudaMemcpyAsync(counts, ctx->d_counts, sizeof counts, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->stats.used_pixels = (int64_t)counts[0];
  ctx->stats.used_voxels = (int64_t)counts[1];
  ctx->n_events = n;
  ctx->stats.n_events = n;
  return order_for_iterations(ctx);
}

int hybrid_get_frames(hybrid_ctx* ctx, int32_t* lor_index_out, int64_t* info_begin,
                      int64_t* info_end, int16_t* plane_begin, int16_t* plane_end,
                      int64_t* response_index) {
  if (!ctx) return STRIP_E_INVALID;
  CK(cudaSetDevice(ctx->device));
  const int64_t n = ctx->n_events;
  if (!n) return STRIP_OK;
  std::vector<Frame> h(n);
  CK(cudaMemcpyAsync(h.data(), ctx->d_frames, n * sizeof(Frame), cudaMemcpyDeviceToHost, ctx->stream));
  if (response_index)
    CK(cudaMemcpyAsync(response_index, ctx->d_index, n * sizeof(int64_t), cudaMemcpyDeviceToHost,
                       ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int64_t i = 0; i < n; ++i) {
    if (lor_index_out) lor_index_out[i] = h[i].lor;
    if (info_begin) info_begin[i] = h[i].info_begin;
    if (info_end) info_end[i] = h[i].info_end;
    if (plane_begin) plane_begin[i] = h[i].plane_begin;
    if (plane_end) plane_end[i] = h[i].plane_end;
  }
  return STRIP_OK;
}

int hybrid_iterate(hybrid_ctx* ctx, int32_t n_iterations, hybrid_progress_cb progress, void* user) {
  if (!ctx) return STRIP_E_INVALID;
  if (n_iterations < 0) return fail(ctx, STRIP_E_INVALID, "negative iteration count");
  if (!ctx->have_sens) return fail(ctx, STRIP_E_STATE, "set the geometry and sensitivity first");
  CK(cudaSetDevice(ctx->device));
  const size_t vb = ctx->n_voxels * sizeof(float);
  const int blocks = ctx->sm_count * mlem_blocks_per_sm();
  if (!ctx->d_spill) CK(cudaMalloc(&ctx->d_spill, mlem_spill_floats(blocks) * sizeof(float)));
  for (int32_t it = 0; it < n_iterations; ++it) {
    if (progress) progress(ctx->stats.iterations, 0, user);
    CK(cudaMemsetAsync(ctx->d_acc_t, 0, vb, ctx->stream));
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (ctx->n_events > 0)
      launch_mlem(ctx->g, geo_view(ctx), ctx->d_sens, iter_frames(ctx), ctx->n_events, ctx->d_rho_t,
                  ctx->d_acc_t, ctx->d_spill, blocks, ctx->stream);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    std::swap(ctx->d_rho_t, ctx->d_acc_t);  // rho = sum of the thread images
    ctx->stats.last_iteration_ms = ms;
    ctx->stats.iterations++;
    if (progress) progress(ctx->stats.iterations - 1, 1, user);
  }
  return STRIP_OK;
}

int hybrid_set_accumulator(hybrid_ctx* ctx, float* device_acc) {
  if (!ctx) return STRIP_E_INVALID;
  ctx->d_acc_user = device_acc;
  return STRIP_OK;
}

int hybrid_accumulate(hybrid_ctx* ctx) {
  if (!ctx) return STRIP_E_INVALID;
  if (!ctx->have_sens) return fail(ctx, STRIP_E_STATE, "set the geometry and sensitivity first");
  CK(cudaSetDevice(ctx->device));
  float* acc = ctx->d_acc_user ? ctx->d_acc_user : ctx->d_acc_t;
  const int blocks = ctx->sm_count * mlem_blocks_per_sm();
  if (!ctx->d_spill) CK(cudaMalloc(&ctx->d_spill, mlem_spill_floats(blocks) * sizeof(float)));
  CK(cudaMemsetAsync(acc, 0, ctx->n_voxels * sizeof(float), ctx->stream));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if (ctx->n_events > 0)
    launch_mlem(ctx->g, geo_view(ctx), ctx->d_sens, iter_frames(ctx), ctx->n_events, ctx->d_rho_t,
                acc, ctx->d_spill, blocks, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaEventSynchronize(ctx->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->stats.last_iteration_ms = ms;
  return STRIP_OK;
}

int hybrid_update(hybrid_ctx* ctx) {
  if (!ctx) return STRIP_E_INVALID;
  CK(cudaSetDevice(ctx->device));
  const float* acc = ctx->d_acc_user ? ctx->d_acc_user : ctx->d_acc_t;
  CK(cudaMemcpyAsync(ctx->d_rho_t, acc, ctx->n_voxels * sizeof(float), cudaMemcpyDeviceToDevice,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->stats.iterations++;
  return STRIP_OK;
}

int hybrid_set_image(hybrid_ctx* ctx, const float* rho) {
  if (!ctx || !rho) return STRIP_E_INVALID;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(ctx->d_tmp, rho, ctx->n_voxels * sizeof(float), cudaMemcpyHostToDevice,
                     ctx->stream));
  launch_to_zfast(ctx->g, ctx->d_tmp, ctx->d_rho_t, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int hybrid_get_image(hybrid_ctx* ctx, float* rho) {
  if (!ctx || !rho) return STRIP_E_INVALID;
  CK(cudaSetDevice(ctx->device));
  launch_from_zfast(ctx->g, ctx->d_rho_t, ctx->d_tmp, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(rho, ctx->d_tmp, ctx->n_voxels * sizeof(float), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return STRIP_OK;
}

int hybrid_get_stats(hybrid_ctx* ctx, hybrid_stats* out) {
  if (!ctx || !out) return STRIP_E_INVALID;
  *out = ctx->stats;
  return STRIP_OK;
}

int hybrid_debug_atan2(int32_t device, const float* a, const float* b, int64_t n,
                       int32_t which, float* out) {
  if (n < 0 || (n > 0 && (!a || !b || !out)) || (which != 0 && which != 1))
    return STRIP_E_INVALID;
  if (n == 0) return STRIP_OK;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return STRIP_E_NODEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return STRIP_E_CUDA;
  float* d = nullptr;
  const size_t bytes = (size_t)n * sizeof(float);
  if (cudaMalloc(&d, 3 * bytes) != cudaSuccess) {
    cudaGetLastError();
    return STRIP_E_NOMEM;
  }
  cudaError_t e = cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n, b, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_atan2_probe(d, d + n, n, which, d + 2 * n, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(out, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return STRIP_E_CUDA;
  }
  return STRIP_OK;
}

}  // extern "C"
