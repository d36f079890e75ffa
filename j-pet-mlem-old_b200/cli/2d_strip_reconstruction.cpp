// 2d_strip_reconstruction -- drop-in for the reference command of the same
// name (src/2d/strip/reconstruction_cmd.cpp:105-301, options
// src/2d/strip/options.cpp:13-124), running the list-mode TOF MLEM on the
// B200 through the C ABI of libstripmlem (include/stripmlem.h).
//
// Same options, `-c/--config` files and automatic `<input>.cfg` loading, same
// input formats and output names.  Without -G/--gpu the reference CPU
// semantics are used (GaussianKernel, no sensitivity); with it the reference
// GPU semantics (AnalyticKernel with the pixel sensitivity) -- both run on the
// GPU.
#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "stripmlem.h"
#include "strip_io.h"
#include "strip_options.h"

namespace {

using strip_cli::Options;
using strip_cli::add_index;
using strip_cli::ext_of;
using strip_cli::wo_ext;
using strip_cli::wo_path;

// reconstruction_cmd.cpp:114-115 and options.cpp:44-76 on top of the shared
// scanner options
void add_reconstruction_options(Options& cl) {
  cl.add_scanner_options();
  cl.add("3d-response", 0, false, false, "", "input response contains additional LOR information");
  cl.add("dl-is-time", 0, false, false, "", "delta is time, convert using speed of light");
  cl.add("speed-of-light", 0, true, false, "299792458", "speed of light");
  cl.add("scale-length", 0, true, false, "1", "scale input length values");
  cl.add("scale-time", 0, true, false, "1", "scale input time values");
  cl.add("blocks", 'i', true, false, "0", "number of iteration blocks");
  cl.add("iterations", 'I', true, false, "1", "number of iterations (per block)");
  cl.add("output", 'o', true, true, "", "output files prefix (png)");
  cl.add("png-max", 0, true, false, "0", "maximum value mapped to 255 in PNG");
  cl.add("gpu", 'G', false, false, "", "use the reference's GPU semantics");
  cl.add("cuda-device", 'D', true, false, "0", "CUDA device");
  cl.add("cuda-blocks", 'B', true, false, "64", "CUDA blocks (accepted, unused)");
  cl.add("cuda-threads", 'W', true, false, "512", "CUDA threads per block (accepted, unused)");
  cl.add("rho", 0, true, false, "", "start rho (eg. existing iteration)");
  cl.add("rho-is-int", 0, false, false, "", "start rho uses integer representation (not float)");
  cl.add("dump-responses", 0, true, true, "",
         "write the responses as read (after unit conversion) to this binary file and exit");
}

// util::progress (util/progress.h:63-127) for -v (estimate) and -vv
// (benchmark table: "# it     time (ms)", one line per iteration, "# av").
class Progress {
 public:
  Progress(int verbosity, int total) : v_(verbosity), total_(total) {
    if (v_ >= 2) std::cout << "# it     time (ms)" << std::endl;
  }
  void operator()(int completed, bool finished) {
    if (!v_) return;
    using clock = std::chrono::high_resolution_clock;
    if (v_ >= 2) {
      if (!finished) {
        start_ = clock::now();
        return;
      }
      const double ms = std::chrono::duration<double>(clock::now() - start_).count() * 1000;
      total_ms_ += ms;
      std::cout << std::setiosflags(std::ios::fixed) << std::setprecision(2)
                << std::setw(4) << (completed + 1) << ' ' << std::setw(10) << ms << std::endl;
      if (completed == total_ - 1)
        std::cout << "# av " << std::setw(10) << total_ms_ / total_ << "   total "
                  << total_ms_ << std::endl;
      std::cout << std::resetiosflags(std::ios::fixed) << std::setprecision(6);
      return;
    }
    if (finished) {
      if (completed < total_ - 1) return;
      ++completed;
    }
    if (completed == last_) return;
    last_ = completed;
    std::cerr << ' ' << (int)std::round(100.0 * completed / std::max(total_, 1)) << "% "
              << completed << "/" << total_ << (finished && completed == total_ ? "\n" : "\r");
  }

 private:
  int v_, total_;
  int last_ = -1;
  double total_ms_ = 0;
  std::chrono::high_resolution_clock::time_point start_;
};

struct Ctx {
  strip_ctx* p = nullptr;
  ~Ctx() {
    if (p) strip_ctx_destroy(p);
  }
};

void check(strip_ctx* ctx, int rc, const char* what) {
  if (rc == STRIP_OK) return;
  char msg[512] = {0};
  if (ctx) strip_last_error(ctx, msg, sizeof msg);
  throw std::string(what) + " failed (" + std::to_string(rc) + ")" + (msg[0] ? ": " : "") + msg;
}

int progress_cb(int completed, int finished, void* user) {
  (*static_cast<Progress*>(user))(completed, finished != 0);
  return 0;
}

int run(int argc, char** argv) {
  Options cl;
  add_reconstruction_options(cl);
  std::vector<std::string> args(argv + 1, argv + argc);
  cl.parse(args, false);
  if (cl.exist("help")) {
    std::cerr << cl.usage(argv[0]);
    return 0;
  }
  // calculate_scanner_options (options.cpp:106-124), before the .cfg loading
  strip_cli::calculate_scanner_options(cl);
  if (cl.rest.empty()) {
    if (argc == 1) {
      std::cerr << cl.usage(argv[0]);
      return 0;
    }
    throw std::string("at least one responses input file expected, consult --help");
  }
  // cmdline::load_accompanying_config (cmdline_hooks.cpp:110-123)
  for (const auto& fn : std::vector<std::string>(cl.rest)) {
    const std::string cfg = wo_ext(fn) + ".cfg";
    if (std::ifstream(cfg).is_open()) cl.load(cfg);
  }
  if (cl.exist("n-threads")) omp_set_num_threads(cl.integer("n-threads"));

  strip_geometry g{};
  g.radius = cl.num("radius");
  g.scintillator_length = cl.num("length");
  g.n_y_pixels = cl.integer("n-y-pixels");
  g.n_z_pixels = cl.integer("n-z-pixels");
  g.pixel_height = cl.num("s-pixel");
  g.pixel_width = cl.num("s-pixel");
  g.sigma_z = cl.num("s-z");
  g.sigma_dl = cl.num("s-dl");
  const int W = g.n_z_pixels, H = g.n_y_pixels;
  const size_t n_pix = (size_t)W * H;

  const int verbose = cl.count("verbose");
  if (verbose) std::cout << "# image: " << H << "x" << W << std::endl;

  std::vector<float> rho(n_pix, 1.0f);  // reconstruction.h:59
  if (cl.exist("rho")) {
    const std::string rn = cl.str("rho");
    if (ext_of(rn) == ".txt") {
      // The reference reads a text start image into copies of the pixels
      // (pixel_map.h:127-132), so it has no effect; kept as is.
      std::ifstream txt(rn);
    } else {
      std::ifstream bin(rn, std::ios::binary);
      if (cl.exist("rho-is-int")) {
        std::vector<int32_t> iv(n_pix, 0);
        bin.read(reinterpret_cast<char*>(iv.data()), (std::streamsize)(n_pix * 4));
        for (size_t i = 0; i < n_pix; ++i) rho[i] = (float)(iv[i] + 1000);
      } else {
        bin.read(reinterpret_cast<char*>(rho.data()), (std::streamsize)(n_pix * 4));
      }
    }
  }

  const bool is_3d = cl.exist("3d-response");
  std::vector<float> zu, zd, dl;
  // One binary event file with no unit conversion goes from the file to the
  // device through the library's staged reader (strip_load_responses_file);
  // everything else is read here first.
  const bool direct = cl.rest.size() == 1 && ext_of(cl.rest[0]) != ".txt" && !is_3d &&
                      !cl.exist("scale-length") && !cl.exist("dl-is-time") &&
                      !cl.exist("dump-responses");
  for (const auto& fn : cl.rest) {
    if (direct) break;
    if (ext_of(fn) == ".txt") {
      strip_cli::read_events_text(fn, is_3d, zu, zd, dl);
    } else {
      if (is_3d) throw std::string("3D input must have .txt extension");
      strip_cli::read_events_binary(fn, zu, zd, dl);
    }
    if (verbose)
      std::cerr << "# read " << zu.size() << " responsess from " << fn << std::endl;
    // unit conversion, applied to all responses read so far (reference order)
    const bool dl_is_time = cl.exist("dl-is-time");
    if (cl.exist("scale-length")) {
      const double scale = cl.num("scale-length");
      for (size_t i = 0; i < zu.size(); ++i) {
        zu[i] = (float)(zu[i] * scale);
        zd[i] = (float)(zd[i] * scale);
        if (!dl_is_time) dl[i] = (float)(dl[i] * scale);
      }
    }
    if (dl_is_time) {
      const double scale = cl.num("scale-time"), c = cl.num("speed-of-light");
      for (size_t i = 0; i < dl.size(); ++i) dl[i] = (float)(dl[i] * c * scale);
    }
  }

  if (cl.exist("dump-responses")) {
    std::vector<float> t(3 * zu.size());
    for (size_t i = 0; i < zu.size(); ++i) {
      t[3 * i] = zu[i];
      t[3 * i + 1] = zd[i];
      t[3 * i + 2] = dl[i];
    }
    strip_cli::write_raw(cl.str("dump-responses"), t.data(), t.size() * 4);
    return 0;
  }

  const int n_blocks = cl.integer("blocks");
  const int n_in_block = cl.integer("iterations");
  const int n_iterations = n_blocks * n_in_block;
  const std::string output = cl.str("output");
  const std::string base = wo_ext(output), out_ext = ext_of(output);
  const bool out_txt = out_ext == ".txt";
  const bool gpu = cl.exist("gpu");
  Progress progress(verbose, n_iterations);

  Ctx ctx;
  check(nullptr, strip_ctx_create(&g, cl.integer("cuda-device"), &ctx.p), "strip_ctx_create");
  if (direct) {
    int64_t n_read = 0;
    check(ctx.p, strip_load_responses_file(ctx.p, cl.rest[0].c_str(), 0, -1, 1, &n_read),
          "strip_load_responses_file");
    if (verbose)
      std::cerr << "# read " << n_read << " responsess from " << cl.rest[0] << std::endl;
  } else {
    check(ctx.p, strip_set_events(ctx.p, zu.data(), zd.data(), dl.data(), (int64_t)zu.size(), 1),
          "strip_set_events");
  }
  check(ctx.p, strip_set_image(ctx.p, rho.data()), "strip_set_image");

  if (gpu) {
    // GPU::Reconstruction::run (cuda/reconstruction.cu:32-113) and its output
    // delegate (reconstruction_cmd.cpp:232-252)
    if (verbose) {
      char name[256];
      strip_device_name(ctx.p, name, sizeof name);
      std::cerr << "# device: " << name << std::endl;
    }
    auto emit = [&](int iteration, const std::vector<float>& img) {
      if (base.empty()) return;
      const std::string fn = iteration >= 0 ? add_index(base, iteration, n_iterations)
                                            : base + "_sensitivity";
      strip_cli::write_png(fn + ".png", img.data(), W, H, 0);
      if (out_txt) strip_cli::write_text_map(fn + ".txt", img.data(), W, H);
      else if (out_ext != ".png") strip_cli::write_raw(fn + out_ext, img.data(), n_pix * 4);
      strip_cli::write_nrrd_header(fn + ".nrrd", wo_path(fn) + out_ext, W, H, out_txt);
    };
    std::vector<float> img(n_pix);
    check(ctx.p, strip_get_sensitivity(ctx.p, 1, img.data()), "strip_get_sensitivity");
    emit(-1, img);
    for (int block = 0; block < n_blocks; ++block) {
      for (int i = 0; i < n_in_block; ++i) {
        const int it = block * n_in_block + i;
        check(ctx.p, strip_iterate(ctx.p, 1, STRIP_MODE_GPU, 1, it, progress_cb, &progress),
              "strip_iterate");
        if (!block && i < n_in_block - 1 &&
            (i < 5 || i == 9 || i == 14 || i == 19 || i == 29 || i == 49 || i == 99)) {
          check(ctx.p, strip_get_image(ctx.p, img.data()), "strip_get_image");
          emit(i + 1, img);
        }
      }
      check(ctx.p, strip_get_image(ctx.p, img.data()), "strip_get_image");
      emit((block + 1) * n_in_block, img);
    }
    progress(n_iterations, false);
  } else {
    // CPU branch (reconstruction_cmd.cpp:264-292)
    std::vector<float> img(n_pix);
    if (!base.empty()) {
      check(ctx.p, strip_get_sensitivity(ctx.p, 0, img.data()), "strip_get_sensitivity");
      strip_cli::write_png(base + "_sensitivity.png", img.data(), W, H, 0);
    }
    for (int block = 0; block < n_blocks; ++block) {
      check(ctx.p, strip_iterate(ctx.p, n_in_block, STRIP_MODE_CPU, 1, block * n_in_block,
                                 progress_cb, &progress),
            "strip_iterate");
      if (base.empty()) continue;
      check(ctx.p, strip_get_image(ctx.p, img.data()), "strip_get_image");
      const std::string fn = add_index(base, (block + 1) * n_in_block, n_iterations);
      strip_cli::write_png(fn + ".png", img.data(), W, H, cl.num("png-max"));
      if (out_txt) {
        strip_cli::write_tuples(fn + ".txt", img.data(), W, H);
      } else if (out_ext != ".png") {
        strip_cli::write_raw(fn + out_ext, img.data(), n_pix * 4);
        strip_cli::write_nrrd_header(fn + ".nrrd", wo_path(fn) + out_ext, W, H, false);
      }
    }
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return run(argc, argv);
  } catch (const std::string& e) {
    std::cerr << "error: " << e << std::endl;
  } catch (const char* e) {
    std::cerr << "error: " << e << std::endl;
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
  }
  return 1;
}
