/*
 * stripmlem.h -- C ABI of the B200 (sm_100a) strip list-mode TOF MLEM library.
 *
 * Drop-in boundary for the 2D strip reconstruction path of
 * JPETTomography/j-pet-mlem-old.  The reference has no FFI; its operator API is
 *   (1) the C++ template Reconstruction<F, Kernel> with public members
 *       scanner / rho / sensitivity / responses and operator()(progress,
 *       n_iterations, n_iterations_so_far)   (src/2d/strip/reconstruction.h:42-154)
 *   (2) the GPU entry point PET2D::Strip::GPU::Reconstruction::run<F>(scanner,
 *       responses, n_responses, rho_io, n_blocks, n_iterations_in_block,
 *       output_cb, progress_cb, device, cuda_blocks, cuda_threads,
 *       device_name_cb)                      (src/2d/strip/cuda/reconstruction.h:32-44)
 *   (3) the 2d_strip_reconstruction CLI      (src/2d/strip/reconstruction_cmd.cpp:105-301)
 * Each entry point below names the piece it replaces.
 *
 * Conventions: every function returns STRIP_OK (0) or a negative STRIP_E*
 * code and never throws or aborts; the message of the last failure on a
 * context is strip_last_error().  The caller owns every host buffer.  One
 * context per host thread; all device work of a context is ordered on the
 * context's own CUDA stream, and every call returns after that work is done.
 *
 * Image layout everywhere: row-major binary32, n_y_pixels rows of
 * n_z_pixels; row 0 is the top (y = +size_y/2), column 0 is z = -size_z/2
 * (scanner.h:136-144, reconstruction.h:67-72).
 */
#ifndef STRIPMLEM_H
#define STRIPMLEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STRIPMLEM_ABI_VERSION 1

enum strip_status {
  STRIP_OK = 0,
  STRIP_E_INVALID = -1,    /* bad argument (null pointer, size, geometry)    */
  STRIP_E_CUDA = -2,       /* a CUDA runtime call failed                      */
  STRIP_E_NOMEM = -3,      /* device or host allocation failed                */
  STRIP_E_STATE = -4,      /* call out of order (e.g. iterate before events)  */
  STRIP_E_KERNEL = -5,     /* a kernel reported an error through its status word */
  STRIP_E_NODEVICE = -6    /* no CUDA device / driver                          */
};

/* Reconstruction semantics.
 * STRIP_MODE_CPU: the reference CPU path -- GaussianKernel, no sensitivity:
 *   rho'_j = sum_e K_ej rho_j / sum_k K_ek rho_k   (reconstruction.h:220-298)
 * STRIP_MODE_GPU: the reference --gpu path -- AnalyticKernel with the 5-point
 *   pixel sensitivity in the denominator (warp_granularity.cuh:347-399):
 *   rho'_j = sum_e K_ej rho_j / sum_k K_ek s_k rho_k
 *   i.e. the sensitivity-normalised LM-MLEM update with P = K * s.
 * Both use the CPU's rule for an all-zero denominator (contribution 0). */
enum strip_mode { STRIP_MODE_CPU = 0, STRIP_MODE_GPU = 1 };

/* Accumulation of the per-event normalisation sums D_e = sum_k P_ek rho_k.
 * FP32: plain binary32 per-lane sums; KAHAN: compensated binary32 per-lane
 * sums; FP64: binary64 per-lane sums.  The cross-lane reduction and the
 * global image/likelihood reductions are binary64 in every mode. */
enum strip_accum { STRIP_ACCUM_FP32 = 0, STRIP_ACCUM_KAHAN = 1, STRIP_ACCUM_FP64 = 2 };

/* Scanner parameters, in the units of the event file (the CLI's millimetres).
 * Replaces Scanner<F, S>'s constructor arguments (scanner.h:39-67, options.h:42-50);
 * the library narrows them to binary32 / int16 exactly as Scanner<float, short>
 * does, so pixel sets match the reference bit for bit. */
typedef struct strip_geometry {
  double radius;              /* R: half the distance between the strips   */
  double scintillator_length; /* L                                         */
  int32_t n_y_pixels;
  int32_t n_z_pixels;
  double pixel_height;
  double pixel_width;
  double sigma_z;             /* TOF sigma along z                         */
  double sigma_dl;            /* TOF sigma of delta-l                       */
  double center_y;
  double center_z;
} strip_geometry;

typedef struct strip_ctx strip_ctx;

/* Iteration progress; replaces the run()'s progress delegate
 * (cuda/reconstruction.h:38-39).  `finished` is 0 before and 1 after an
 * iteration.  Return non-zero to stop after the current iteration. */
typedef int (*strip_progress_cb)(int completed, int finished, void* user);

/* Statistics of the last set_events / iterate. */
typedef struct strip_stats {
  int64_t n_events;          /* events held by the context                    */
  int64_t n_empty;           /* events whose clamped box is empty (skipped)   */
  int64_t n_overflow;        /* events processed on the global-memory path   */
  int32_t n_tiles_z, n_tiles_y, tile_z, tile_y, halo_z, halo_y;
  int32_t n_work_items;      /* (tile, event chunk) items per full pass        */
  int32_t n_subsets;         /* subsets of the current binning                */
  int32_t max_box_w, max_box_h;
  int32_t smem_bytes;        /* dynamic shared memory per CTA                 */
  int32_t kernel_launches;   /* launches of the last strip_iterate             */
  double last_iterate_ms;    /* device time of the last strip_iterate          */
  double last_setup_ms;      /* device time of the last set_events binning     */
  double last_tile_ms;       /* device time of the tile-kernel launches of the
                                last strip_iterate (CUDA events on the stream) */
  int64_t n_fallback;        /* events of the last strip_iterate / accumulate
                                that a tile's unweighted fixed-point window had
                                no room for (rerun in a weighted window)       */
  int32_t max_item_events;   /* events of the largest tile work item           */
  int32_t reserved;
  double last_upload_ms;     /* host wall time of the last set_events /
                                set_responses / load_responses_file copy of
                                the events into device memory (file reads
                                included), before the binning               */
} strip_stats;

/* ---- context ------------------------------------------------------------ */

/* Creates a context on `device`.  Replaces the device selection and
 * per-run state of GPU::Reconstruction::run (cuda/reconstruction.cu:54-74).
 * The image starts at 1 everywhere, as Reconstruction's rho (reconstruction.h:59). */
int strip_ctx_create(const strip_geometry* geometry, int device, strip_ctx** out);
int strip_ctx_destroy(strip_ctx* ctx);
/* Copies the last error message (NUL-terminated, truncated to size). */
int strip_last_error(const strip_ctx* ctx, char* buf, size_t size);
/* Device name, as run()'s device_name delegate (cuda/reconstruction.cu:55-57). */
int strip_device_name(const strip_ctx* ctx, char* buf, size_t size);
int strip_set_accumulation(strip_ctx* ctx, int accum);
int strip_get_stats(const strip_ctx* ctx, strip_stats* out);

/* ---- events ------------------------------------------------------------- */

/* Host SoA events: z_u, z_d, dl.  Replaces ResponsesSOA (cuda/gpu_events_soa.h:15-44)
 * and Reconstruction::responses.  Copies to the device, sorts the events into
 * image tiles (n_subsets OSEM subsets: event e goes to subset e % n_subsets)
 * and keeps them resident. */
int strip_set_events(strip_ctx* ctx, const float* z_u, const float* z_d,
                     const float* dl, int64_t n, int n_subsets);
/* Host AoS events: n triples (z_u, z_d, dl), the reference's Response<float>
 * layout and binary event-file layout (response.h:13-20, reconstruction.h:156-167). */
int strip_set_responses(strip_ctx* ctx, const float* zu_zd_dl, int64_t n,
                        int n_subsets);
/* Reads events of a binary event file -- raw little-endian binary32 triples
 * z_u z_d dl, the reference's format (response.h:13-20, read until the end
 * of the file by reconstruction.h:156-167; a trailing partial triple is
 * ignored) -- from event `first` on, at most n of them (n < 0: to the end),
 * straight into device memory, and bins them as strip_set_events.  Several
 * host threads read chunks into pinned staging buffers while earlier chunks
 * are being copied to the device.  *n_loaded (may be NULL) receives the
 * number of events.  Replaces the reference CLI's whole-file read
 * (reconstruction_cmd.cpp:168-186) for one binary input file. */
int strip_load_responses_file(strip_ctx* ctx, const char* path, int64_t first,
                              int64_t n, int n_subsets, int64_t* n_loaded);
/* Same as strip_set_events with device pointers (already resident in HBM). */
int strip_set_events_device(strip_ctx* ctx, const float* d_z_u,
                            const float* d_z_d, const float* d_dl, int64_t n,
                            int n_subsets);

/* ---- image -------------------------------------------------------------- */

/* rho in / out (host, n_y * n_z floats); Reconstruction::rho / run()'s rho_io.
 * An activity image is non-negative and finite: strip_set_image rejects
 * anything else with STRIP_E_INVALID (the reference does not check). */
int strip_set_image(strip_ctx* ctx, const float* rho);
int strip_get_image(strip_ctx* ctx, float* rho);
/* Sensitivity image: five_point = 1 gives Scanner::pixel_sensitivity
 * (scanner.h:174-185, the --gpu path's texture); 0 gives the centre value
 * Scanner::sensitivity (the CPU Reconstruction::sensitivity, reconstruction.h:67-73). */
int strip_get_sensitivity(strip_ctx* ctx, int five_point, float* out);

/* ---- reconstruction ------------------------------------------------------ */

/* Runs n_iter MLEM iterations (n_subsets == 1) or OSEM iterations (each
 * visits every subset once; subset update rho_j <- n_subsets * rho_j *
 * sum_{e in subset} P_ej / D_e).  Replaces Reconstruction::operator()
 * (reconstruction.h:109-154) and the iteration loop of run()
 * (cuda/reconstruction.cu:79-110).  n_subsets must equal the binning of
 * set_events, or the events are re-binned first.  `first` numbers the
 * progress callbacks (n_iterations_so_far). */
int strip_iterate(strip_ctx* ctx, int n_iter, int mode, int n_subsets,
                  int first, strip_progress_cb progress, void* user);

/* ---- split iteration: one MLEM/OSEM step as backprojection + update ----
 * For event sets sharded over several processes or GPUs, each holding the
 * same image: every shard runs strip_accumulate for the subset, the shards
 * sum their accumulators (an all-reduce of n_y * n_z binary64 values, e.g.
 * ncclAllReduce on the buffer given to strip_set_accumulator), and every
 * shard applies strip_update.  One strip_iterate step of n_subsets == 1 is
 * strip_accumulate(ctx, mode, 1, 0) followed by strip_update(ctx, 1.0); an
 * OSEM step visits s = 0 .. n_subsets - 1, each followed by an update with
 * scale n_subsets.  The reference's loop is single-process
 * (reconstruction.h:109-154); its per-thread images summed before the update
 * (reconstruction.h:137-148) are the single-node form of this exchange. */

/* Makes the caller's DEVICE buffer of n_y * n_z binary64 values (on the
 * context's device) the backprojection accumulator of every later call, and
 * zero-fills it; NULL returns to the context's own buffer.  The caller keeps
 * the buffer alive while it is in use. */
int strip_set_accumulator(strip_ctx* ctx, double* d_acc);
/* acc_j += sum_{e in subset} P_ej / D_e over the context's events of subset
 * `subset` (event e belongs to subset e % n_subsets); rho is not changed. */
int strip_accumulate(strip_ctx* ctx, int mode, int n_subsets, int subset);
/* rho_j <- rho_j * acc_j * scale, then acc_j <- 0. */
int strip_update(strip_ctx* ctx, double scale);

/* ---- differentiable projections (pixel sets fixed by the geometry's sigmas) */

/* y_e = sum_j P_ej rho_j for every event, in the caller's event order, with
 * the kernel evaluated at (sigma_z, sigma_dl).  rho and y are host buffers. */
int strip_forward(strip_ctx* ctx, const float* rho, double sigma_z,
                  double sigma_dl, int mode, double* y);
/* g_j = sum_e P_ej w_e (adjoint / backprojection), w in event order. */
int strip_adjoint(strip_ctx* ctx, const double* w, double sigma_z,
                  double sigma_dl, int mode, double* g);
/* d/d(sigma_z, sigma_dl) of sum_e w_e y_e, STRIP_MODE_CPU kernel. */
int strip_grad_sigma(strip_ctx* ctx, const float* rho, const double* w,
                     double sigma_z, double sigma_dl, double* d_sigma_z,
                     double* d_sigma_dl);
/* The same three with DEVICE buffers on the context's device (rho: n_y * n_z
 * floats, y and w: one double per event of set_events, g: n_y * n_z doubles,
 * grad: 2 doubles {d/dsigma_z, d/dsigma_dl}); no host copies.  The reference
 * has no projection operators; these serve a differentiable model whose
 * tensors live on the GPU. */
int strip_forward_device(strip_ctx* ctx, const float* d_rho, double sigma_z,
                         double sigma_dl, int mode, double* d_y);
int strip_adjoint_device(strip_ctx* ctx, const double* d_w, double sigma_z,
                         double sigma_dl, int mode, double* d_g);
int strip_grad_sigma_device(strip_ctx* ctx, const float* d_rho,
                            const double* d_w, double sigma_z,
                            double sigma_dl, double* d_grad);

/* ---- batches of reconstructions ----------------------------------------- */

/* Several contexts -- each with its own geometry, events and image -- advanced
 * together: one MLEM step is a tile launch of its own for every member with
 * at least two work items per SM (on side streams), one persistent launch of
 * the tile kernel over the work items of the smaller members, the global-path
 * launches of members with oversized event boxes, and one update launch over
 * all images; the step is
 * captured once as a CUDA graph and replayed.  The reference runs one
 * reconstruction per process; there is no counterpart.
 * Members (at most 64) share the device and the accumulation mode; their
 * events are re-binned for plain MLEM (one subset), without the last wave
 * of work items cut into pieces.  A batch holds the
 * members' buffers as they were at creation: re-create it after
 * strip_set_events, strip_set_accumulator or a re-binning of a member
 * (strip_set_image keeps the buffers).  While a batch iterates its members
 * must not be used on other threads. */
typedef struct strip_batch strip_batch;
int strip_batch_create(strip_ctx* const* members, int n_members, int mode,
                       strip_batch** out);
/* n_iter MLEM iterations of every member (no progress callbacks). */
int strip_batch_iterate(strip_batch* b, int n_iter);
/* Device time of the last strip_batch_iterate, the members' total events,
 * the tile work items of one step and the kernel launches of one step. */
int strip_batch_stats(strip_batch* b, double* last_iterate_ms,
                      int64_t* n_events, int32_t* n_work_items,
                      int32_t* launches_per_iteration);
int strip_batch_last_error(strip_batch* b, char* buf, size_t size);
int strip_batch_destroy(strip_batch* b);

/* ---- schedule --------------------------------------------------------------- */

/* A tile-kernel schedule: pixel tile edge, events a warp takes per counter
 * step, and the measured device time of one backprojection with it. */
typedef struct strip_tuning {
  int32_t tile;
  int32_t grab;
  double ms;
} strip_tuning;
/* Times one MLEM backprojection of the context's events (into scratch: the
 * image and accumulator are untouched) for every schedule of tile edge
 * {16, 32, 48, 64} x grab {4, 8, 16, 32}, keeps the fastest (events re-binned
 * for it) and reports it in *best (may be NULL). */
int strip_autotune(strip_ctx* ctx, int mode, strip_tuning* best);
/* Sets the schedule by hand (tile edge 8..128, grab 1..32); re-bins the
 * events when the context has some.  Defaults: tile 32, grab 32. */
int strip_set_schedule(strip_ctx* ctx, int tile, int grab);
/* Largest tile work item, in events (1..8000); 0 (the default) picks it per
 * binning: enough items for about eight waves of the device, at least 2048
 * and at most 8000 events, the last wave's worth of each subset's items cut
 * into quarter pieces.  Re-bins the events when the context has some.
 * The item size changes the work decomposition and the fixed-point scale of
 * each item's window, not the result beyond rounding; a small event set
 * binned with 8000-event items runs the arithmetic of a large one. */
int strip_set_item_events(strip_ctx* ctx, int max_events);

/* ---- parity ----------------------------------------------------------- */

/* For n host events (z_u, z_d, dl): bbox pixels tested, in-ellipse pixels and
 * the order-free set digest sum_p mix64(index_p + 1) (mod 2^64), where
 * mix64 is the splitmix64 finaliser -- computed on the device by the same
 * enumeration code the reconstruction kernels run.  Any output may be NULL.
 * Replaces the DEBUG pixel dump of bb_update (reconstruction.h:257-286). */
int strip_debug_pixel_sets(strip_ctx* ctx, const float* z_u, const float* z_d,
                           const float* dl, int64_t n, int32_t* n_bb,
                           int32_t* n_in, uint64_t* digest);

/* Multiplies the per-work-item statistics that size the unweighted
 * fixed-point windows of the next MLEM pass by `factor` (> 0).  A factor
 * below 1 makes the next pass's windows too fine for their events, so events
 * run out of room and take the weighted rerun (strip_stats.n_fallback): a
 * test of that path.  Results stay correct for any factor; only the
 * speed changes.  No counterpart in the reference. */
int strip_debug_scale_item_stats(strip_ctx* ctx, float factor);

/* ---- allocation-free iteration ----------------------------------------- */

/* Largest image (n_y * n_z pixels) strip_iterate_noalloc accepts. */
#define STRIP_NOALLOC_MAX_PIXELS (1 << 20)

/* One MLEM iteration that allocates no device memory, for callers that cannot
 * call cudaMalloc: code inside a host framework that owns all device memory
 * through its own pool under a fixed budget, and pipelines that must not hit
 * cudaMalloc / cudaFree because they can synchronise the device.  No
 * counterpart in the reference.
 *
 * Inputs and outputs are caller-owned DEVICE buffers on the current device:
 * n events (z_u, z_d, dl), the image rho_in and the result rho_out
 * (n_y * n_z floats each; rho_out may equal rho_in).  `mode` as
 * strip_iterate; accumulation as STRIP_ACCUM_KAHAN.  The work is enqueued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) and the call
 * returns without waiting for it.  Events are processed unbinned, one warp
 * per event, straight from global memory.
 *
 * Scratch is a fixed file-scope device array (a binary64 accumulator and a
 * binary32 sensitivity image of STRIP_NOALLOC_MAX_PIXELS entries each, 12 MiB
 * held by every GPU that loads the library until exit).  The first call in a
 * CUDA context of a device looks up the scratch's device address and caches
 * it with the context's unique id, so make that first call before any stream
 * capture; a call in a new context (after cudaDeviceReset, or under another
 * driver-API context) looks it up again.  All calls share the scratch: calls that overlap
 * on the GPU race.  Images larger than STRIP_NOALLOC_MAX_PIXELS are rejected
 * with STRIP_E_INVALID, as are invalid geometries and null pointers. */
int strip_iterate_noalloc(const strip_geometry* geometry, const float* d_z_u,
                          const float* d_z_d, const float* d_dl, int64_t n,
                          const float* d_rho_in, float* d_rho_out, int mode,
                          void* stream);

/* ---- diagnostics ---------------------------------------------------------- */

/* Totals over the context's events of the bounding-box pixels tested and the
 * in-ellipse pixels (kernel evaluations) of one full pass, and the number of
 * events with a non-empty pixel set.  Replaces ReconstructionStats'
 * n_pixels_processed / n_kernel_calls (reconstruction_stats.h:7-89,
 * reconstruction.h:260,272), which the reference can only collect in a
 * special build. */
int strip_count_work(strip_ctx* ctx, int64_t* n_bb, int64_t* n_in,
                     int64_t* n_nonempty);

/* Measures the device's binary32 FMA throughput (TFLOP/s, FMA = 2 flops) with
 * a register-resident FMA chain kernel: the denominator of the roofline
 * fraction of the (FP32-bound) reconstruction kernels.  No counterpart in the
 * reference. */
int strip_probe_fp32_peak(int device, double* tflops);

/* ---- synthetic input ----------------------------------------------------- */

/* Ellipse phantom region (the reference's phantom-file line
 * "ellipse x y a b angle intensity", phantom.h:137-181; x is z). */
typedef struct strip_ellipse {
  double z, y, a, b, angle_deg, activity;
} strip_ellipse;

/* A phantom region of the reference's phantom description
 * (phantom.h:137-181; z is the file's x): ellipse (centre, axes a, b,
 * rotation in degrees), rectangle (centre, half sides a, b) or point
 * (centre); intensity per unit area (per point). */
enum strip_region_kind {
  STRIP_REGION_ELLIPSE = 0,
  STRIP_REGION_RECTANGLE = 1,
  STRIP_REGION_POINT = 2
};
typedef struct strip_region {
  int32_t kind;
  int32_t reserved;
  double z, y, a, b, angle_deg, intensity;
} strip_region;

/* Seeded host generator of list-mode events in the reference's event format.
 * Emission points are uniform in the union of the ellipses, overlaps
 * exclusive with the first-listed ellipse on top (phantom.h:193-204);
 * tan(theta) is uniform in (-L/(2R), L/(2R)); an emission counts only if both
 * hits land on the strips (|z_u|,|z_d| < L/2, scanner.h:196-214); hits are
 * then smeared by N(0, sigma_z) on z_u, z_d and N(0, sigma_dl) on dl
 * (scanner.h:257-267).  Counter-based (Philox-4x32-10), so event i depends
 * only on (seed, i) and the result does not depend on the thread count. */
int strip_generate_events(const strip_geometry* g, const strip_ellipse* ellipses,
                          int n_ellipses, uint64_t seed, int64_t n,
                          float* z_u, float* z_d, float* dl);

/* Same detection and smearing with emission points drawn from an activity
 * image rho (n_y * n_z, the image layout above, non-negative): pixel with
 * probability rho_j / sum rho, point uniform in the pixel.  uniform_angle = 0
 * draws tan(theta) uniformly over the acceptance as above; 1 draws the angle
 * uniformly in (-pi/2, pi/2) as the reference's phantom tool does
 * (phantom.h:213), the emission model the strip kernel assumes.  The
 * reference generates only from phantom shapes (phantom.h:120-215); an image
 * source is what a list-mode model fit needs, where rho is the truth the
 * forward projection is evaluated on. */
int strip_generate_events_image(const strip_geometry* g, const float* rho,
                                uint64_t seed, int64_t n, int uniform_angle,
                                float* z_u, float* z_d, float* dl);

/* The two generators on the current CUDA device, one thread per event, into
 * DEVICE buffers d_z_u, d_z_d, d_dl of n floats each (rho stays a host
 * image); return after the events are written.  Event i is the host
 * generator's event i: the same Philox counters and the same binary64
 * expressions, evaluated without FMA contraction on both sides, so results
 * can differ only where the device math library rounds log, sin, cos or tan
 * differently from the host's.  Replaces the reference's 2d_strip_phantom
 * Monte Carlo loop (phantom_cmd.cpp:136-444, phantom_monte_carlo.h:29-109)
 * for inputs of 1e8-1e9 events. */
int strip_generate_events_device(const strip_geometry* g,
                                 const strip_ellipse* ellipses, int n_ellipses,
                                 uint64_t seed, int64_t n, float* d_z_u,
                                 float* d_z_d, float* d_dl);
int strip_generate_events_image_device(const strip_geometry* g,
                                       const float* rho, uint64_t seed,
                                       int64_t n, int uniform_angle,
                                       float* d_z_u, float* d_z_d, float* d_dl);

/* The reference's phantom Monte Carlo (2d_strip_phantom: phantom_cmd.cpp:
 * 136-444, phantom_monte_carlo.h:29-109, phantom.h:120-215) on the current
 * CUDA device, one thread per emission index:
 *   additive       overlapping regions add up instead of the first-listed
 *                  region covering the later ones (--additive)
 *   uniform_angle  emission angle uniform in (-pi/2, pi/2), the tool's
 *                  model; 0: tan(theta) uniform over the acceptance
 *   count_emitted  n counts emissions and only the detected ones are
 *                  written, in emission order (the tool without --detected);
 *                  0: n detected events (--detected)
 *   d_emitted, d_detected  optional DEVICE images of n_z x n_y counts
 *                  (uint32) of the emission points of all / the detected
 *                  emissions, on the tool's pixel grid of pixel_size centred
 *                  at (origin_z, origin_y): column = floor((z - z0) / s),
 *                  row = floor((y - y0) / s), row 0 at the bottom; counts
 *                  are added to what the images hold.
 * Events go to DEVICE buffers of n floats each; *n_written receives their
 * number and *n_emitted the number of emissions (either may be NULL).
 * Random streams: Philox-4x32-10 counters (seed, index), not the reference's
 * tausworthe generator, so the events are the reference's in distribution,
 * not in value. */
typedef struct strip_simulation {
  int32_t additive;
  int32_t uniform_angle;
  int32_t count_emitted;
  int32_t reserved;
  uint32_t* d_emitted;
  uint32_t* d_detected;
  double pixel_size, origin_z, origin_y;
} strip_simulation;
int strip_simulate_device(const strip_geometry* g, const strip_region* regions,
                          int n_regions, const strip_simulation* options,
                          uint64_t seed, int64_t n, float* d_z_u, float* d_z_d,
                          float* d_dl, int64_t* n_written, int64_t* n_emitted);
/* The same with HOST buffers on CUDA device `device`: z_u, z_d, dl hold n
 * floats each (the first *n_written are set); emitted / detected are
 * n_y x n_z hit images (may be NULL; the d_ fields of options are ignored). */
int strip_simulate(const strip_geometry* g, const strip_region* regions,
                   int n_regions, const strip_simulation* options,
                   uint64_t seed, int64_t n, int device, float* z_u,
                   float* z_d, float* dl, uint32_t* emitted, uint32_t* detected,
                   int64_t* n_written, int64_t* n_emitted);

#ifdef __cplusplus
}
#endif

#endif /* STRIPMLEM_H */
