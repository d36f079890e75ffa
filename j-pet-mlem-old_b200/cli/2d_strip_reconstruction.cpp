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

namespace {

// ---------------------------------------------------------------------------
// options: the reference's option set (options.cpp:13-76, reconstruction_cmd
// .cpp:114-115, common/options.cpp:5-20) and its parser semantics
// (lib/cmdline: --name=value, --name value, -x value, -abc flags; config
// files hold one argument per line, '#' lines ignored; options marked
// not_from_file ignore config files).
// ---------------------------------------------------------------------------
struct Option {
  std::string name;
  char short_name;
  bool has_value;
  bool not_from_file;
  std::string def;
  std::string help;
  std::string value;
  int count = 0;
};

class Options {
 public:
  Options() {
    add("config", 'c', true, false, "", "load config file");
    add("radius", 'r', true, false, "0.5", "R distance between scintillator");
    add("length", 'l', true, false, "1", "scintillator length");
    add("s-pixel", 'p', true, false, "0.01", "pixel size");
    add("n-pixels", 'n', true, false, "0", "number of pixels");
    add("n-z-pixels", 0, true, false, "", "number of z pixels");
    add("n-y-pixels", 0, true, false, "", "number of y pixels");
    add("s-z", 0, true, false, "0.015", "TOF sigma along z axis");
    add("s-dl", 0, true, false, "0.06", "TOF sigma delta-l");
    add("n-emissions", 'e', true, true, "0", "number of emissions");
    add("verbose", 'v', false, false, "", "print progress information (-v) or benchmark (-vv)");
    add("n-threads", 'T', true, false, "", "number of host threads");
    add("3d-response", 0, false, false, "", "input response contains additional LOR information");
    add("dl-is-time", 0, false, false, "", "delta is time, convert using speed of light");
    add("speed-of-light", 0, true, false, "299792458", "speed of light");
    add("scale-length", 0, true, false, "1", "scale input length values");
    add("scale-time", 0, true, false, "1", "scale input time values");
    add("blocks", 'i', true, false, "0", "number of iteration blocks");
    add("iterations", 'I', true, false, "1", "number of iterations (per block)");
    add("output", 'o', true, true, "", "output files prefix (png)");
    add("png-max", 0, true, false, "0", "maximum value mapped to 255 in PNG");
    add("gpu", 'G', false, false, "", "use the reference's GPU semantics");
    add("cuda-device", 'D', true, false, "0", "CUDA device");
    add("cuda-blocks", 'B', true, false, "64", "CUDA blocks (accepted, unused)");
    add("cuda-threads", 'W', true, false, "512", "CUDA threads per block (accepted, unused)");
    add("rho", 0, true, false, "", "start rho (eg. existing iteration)");
    add("rho-is-int", 0, false, false, "", "start rho uses integer representation (not float)");
    add("help", 'h', false, false, "", "print this message");
    add("dump-responses", 0, true, true, "",
        "write the responses as read (after unit conversion) to this binary file and exit");
  }

  void parse(const std::vector<std::string>& args, bool from_file) {
    for (size_t i = 0; i < args.size(); ++i) {
      const std::string& a = args[i];
      if (a.compare(0, 2, "--") == 0) {
        const auto eq = a.find('=');
        const std::string name = a.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
        Option& o = get(name);
        if (eq != std::string::npos) {
          set(o, a.substr(eq + 1), from_file);
        } else if (o.has_value) {
          if (i + 1 >= args.size()) throw "option needs value: --" + name;
          set(o, args[++i], from_file);
        } else {
          set(o, "", from_file);
        }
      } else if (a.size() > 1 && a[0] == '-') {
        for (size_t j = 1; j < a.size(); ++j) {
          Option& o = get_short(a[j]);
          const bool last = j + 1 == a.size();
          if (last && o.has_value && i + 1 < args.size()) {
            set(o, args[++i], from_file);
          } else if (o.has_value) {
            throw std::string("option needs value: -") + a[j];
          } else {
            set(o, "", from_file);
          }
        }
      } else if (a != "-") {
        rest.push_back(a);
      }
    }
  }

  // cmdline::load (cmdline_hooks.cpp:50-96): relative paths resolve against
  // the including config file's directory.
  void load(const std::string& arg) {
    std::string path = arg;
    if (!dir_stack_.empty() && !path.empty() && path[0] != '/')
      path = dir_stack_.back() + path;
    if (exist("verbose")) std::cout << "# load: " << path << std::endl;
    std::ifstream in(path);
    if (!in.is_open()) throw "cannot open input config file: " + path;
    const auto sep = path.find_last_of('/');
    dir_stack_.push_back(sep == std::string::npos ? std::string() : path.substr(0, sep + 1));
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(in, line))
      if (!line.empty() && line[0] != '#') lines.push_back(line);
    const size_t n_rest = rest.size();
    parse(lines, true);
    rest.resize(n_rest);  // positional lines of a config file are ignored
    dir_stack_.pop_back();
  }

  bool exist(const std::string& name) const { return opts_.at(name).count > 0; }
  int count(const std::string& name) const { return opts_.at(name).count; }
  std::string str(const std::string& name) const {
    const Option& o = opts_.at(name);
    return o.count ? o.value : o.def;
  }
  double num(const std::string& name) const {
    const std::string s = str(name);
    // vector options (--radius) keep their first comma-separated element
    return std::strtod(s.substr(0, s.find(',')).c_str(), nullptr);
  }
  int integer(const std::string& name) const { return (int)std::strtol(str(name).c_str(), nullptr, 10); }
  void set_int(const std::string& name, int v) {
    Option& o = opts_.at(name);
    o.value = std::to_string(v);
    if (!o.count) o.count = 1;
  }

  std::string usage(const char* prog) const {
    std::ostringstream os;
    os << "usage: " << prog << " [options] ... response ...\n"
       << "note: All length options below should be expressed in milimeters.\n"
       << "options:\n";
    for (const auto& name : order_) {
      const Option& o = opts_.at(name);
      os << "  ";
      if (o.short_name) os << "-" << o.short_name << ", "; else os << "    ";
      os << "--" << std::left << std::setw(16) << o.name << o.help;
      if (o.has_value && !o.def.empty()) os << " (=" << o.def << ")";
      os << "\n";
    }
    return os.str();
  }

  std::vector<std::string> rest;

 private:
  void add(const std::string& name, char s, bool has_value, bool nff,
           const std::string& def, const std::string& help) {
    Option o;
    o.name = name;
    o.short_name = s;
    o.has_value = has_value;
    o.not_from_file = nff;
    o.def = def;
    o.help = help;
    opts_[name] = o;
    order_.push_back(name);
  }
  Option& get(const std::string& name) {
    auto it = opts_.find(name);
    if (it == opts_.end()) throw "undefined option: --" + name;
    return it->second;
  }
  Option& get_short(char c) {
    for (auto& kv : opts_)
      if (kv.second.short_name == c) return kv.second;
    throw std::string("undefined short option: -") + c;
  }
  void set(Option& o, const std::string& v, bool from_file) {
    if (from_file && o.not_from_file) return;
    if (o.name == "config") {
      load(v);
      return;
    }
    o.value = v;
    ++o.count;
  }

  std::map<std::string, Option> opts_;
  std::vector<std::string> order_;
  std::vector<std::string> dir_stack_;
};

// path helpers (cmdline_types.h): extension, name without extension / path,
// and add_index(index, max) -> "_<index>" zero-padded to the digits of max.
std::string ext_of(const std::string& p) {
  const auto sep = p.find_last_of("\\/"), dot = p.find_last_of('.');
  if (dot == std::string::npos || (sep != std::string::npos && sep > dot)) return "";
  return p.substr(dot);
}
std::string wo_ext(const std::string& p) { return p.substr(0, p.size() - ext_of(p).size()); }
std::string wo_path(const std::string& p) {
  const auto sep = p.find_last_of("\\/");
  return sep == std::string::npos ? p : p.substr(sep + 1);
}
std::string add_index(const std::string& p, int index, int max) {
  int digits = 1;
  for (int m = 10; m <= max; m *= 10) ++digits;
  std::ostringstream os;
  os << p << "_" << std::setw(digits) << std::setfill('0') << index;
  return os.str();
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
  std::vector<std::string> args(argv + 1, argv + argc);
  cl.parse(args, false);
  if (cl.exist("help")) {
    std::cerr << cl.usage(argv[0]);
    return 0;
  }
  // calculate_scanner_options (options.cpp:106-124), before the .cfg loading
  if (cl.exist("n-pixels")) {
    cl.set_int("n-z-pixels", cl.integer("n-pixels"));
    cl.set_int("n-y-pixels", cl.integer("n-pixels"));
  } else {
    if (!cl.exist("n-z-pixels"))
      cl.set_int("n-z-pixels", (int)std::ceil(cl.num("length") / cl.num("s-pixel")));
    if (!cl.exist("n-y-pixels"))
      cl.set_int("n-y-pixels", (int)std::ceil(2 * cl.num("radius") / cl.num("s-pixel")));
  }
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
  for (const auto& fn : cl.rest) {
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
  check(ctx.p, strip_set_events(ctx.p, zu.data(), zd.data(), dl.data(), (int64_t)zu.size(), 1),
        "strip_set_events");
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
