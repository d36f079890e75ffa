// 2d_strip_phantom -- drop-in for the reference command of the same name
// (src/2d/strip/phantom_cmd.cpp:136-444, options src/2d/strip/options.cpp:
// 78-104): simulates the strip scanner's responses to a phantom on the GPU
// (strip_simulate) and writes the reference's outputs -- the response
// file (binary triples, or text for a .txt name), <base>.cfg for
// 2d_strip_reconstruction, and the emitted / detected / naive count images
// (raw int32 + NRRD + PNG).
//
// Same options and phantom description format ("ellipse x y a b angle
// intensity", "rectangle x y a b intensity", "point x y intensity"; x is z).
// The events follow the reference's Monte Carlo in distribution (uniform
// emission angle, exclusive or --additive regions, detection on the exact
// hits, Gaussian smearing after detection) from Philox counter streams
// (--seed), not from the reference's tausworthe generator.  --tan-bins,
// --kernel-point and --full are not supported.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "stripmlem.h"
#include "strip_io.h"
#include "strip_options.h"

namespace {

using strip_cli::Options;

void add_phantom_options(Options& cl) {
  cl.add_scanner_options();
  cl.add("scale", 0, true, false, "1", "Scale phantom with given constant");
  cl.add("additive", 0, false, false, "", "phantom regions are additive, not disjunctive");
  cl.add("tan-bins", 0, true, false, "", "not supported");
  cl.add("kernel-point", 0, true, false, "", "not supported");
  cl.add("full", 0, false, false, "", "not supported");
  cl.add("no-responses", 0, false, false, "", "Do not emit responses");
  cl.add("point", 0, true, false, "", "Add point phantom x,y[,intensity]");
  cl.add("output", 'o', true, true, "phantom.bin", "responses file");
  cl.add("detected", 0, false, false, "", "collects detected emissions");
  cl.add("image-origin", 0, true, false, "", "Image origin x,y (default 0,0)");
  cl.add("seed", 0, true, false, "1", "random stream seed (Philox counters)");
  cl.add("uniform-tan", 0, false, false, "",
         "draw tan(theta) uniformly over the acceptance instead of a uniform angle");
  cl.add("cuda-device", 'D', true, false, "0", "CUDA device");
}

std::vector<double> parse_list(const std::string& s) {
  std::vector<double> v;
  std::stringstream ss(s);
  std::string el;
  while (std::getline(ss, el, ',')) v.push_back(std::strtod(el.c_str(), nullptr));
  return v;
}

// Phantom::operator<< (phantom.h:137-181): a malformed line ends the file,
// an unknown shape is an error; ellipses and rectangles are scaled, points
// are not.
void read_phantom(const std::string& fn, double scale, std::vector<strip_region>& out) {
  std::ifstream in(fn);
  if (!in.is_open()) throw "cannot open phantom description: " + fn;
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream iss(line);
    std::string type;
    iss >> type;
    strip_region r{};
    if (type == "ellipse") {
      double x, y, a, b, angle, intensity;
      if (!(iss >> x >> y >> a >> b >> angle >> intensity)) break;
      r = strip_region{STRIP_REGION_ELLIPSE, 0, x * scale, y * scale, a * scale,
                       b * scale, angle, intensity};
    } else if (type == "rectangle") {
      double x, y, a, b, intensity;
      if (!(iss >> x >> y >> a >> b >> intensity)) break;
      r = strip_region{STRIP_REGION_RECTANGLE, 0, x * scale, y * scale, a * scale,
                       b * scale, 0, intensity};
    } else if (type == "point") {
      double x, y, intensity;
      if (!(iss >> x >> y >> intensity)) break;
      r = strip_region{STRIP_REGION_POINT, 0, x, y, 0, 0, 0, intensity};
    } else {
      throw "unknown phantom type: " + type;
    }
    out.push_back(r);
  }
}

// the tool's pixel grid (pixel_grid.h:59-69) in binary32 as the reference
struct Grid {
  int nz, ny;
  float llz, lly, s;
  bool at(float z, float y, int& col, int& row) const {
    col = (int)std::floor((z - llz) / s);
    row = (int)std::floor((y - lly) / s);
    return col >= 0 && col < nz && row >= 0 && row < ny;
  }
};

void write_image(const std::string& base, const std::vector<int32_t>& img, int nz, int ny) {
  strip_cli::write_raw(base, img.data(), img.size() * sizeof(int32_t));
  strip_cli::write_nrrd_header(base + ".nrrd", strip_cli::wo_path(base), nz, ny, false, "int");
  std::vector<float> f(img.begin(), img.end());
  strip_cli::write_png(base + ".png", f.data(), nz, ny, 0.0);
}

int run(int argc, char** argv) {
  Options cl;
  add_phantom_options(cl);
  std::vector<std::string> args(argv + 1, argv + argc);
  cl.parse(args, false);
  if (cl.exist("help")) {
    std::cerr << cl.usage(argv[0], "phantom_description");
    return 0;
  }
  strip_cli::calculate_scanner_options(cl);
  if (cl.rest.empty() && !cl.exist("point")) {
    if (argc == 1) {
      std::cerr << cl.usage(argv[0], "phantom_description");
      return 0;
    }
    throw std::string("at least one input phantom description expected, consult --help");
  }
  for (const char* unsupported : {"tan-bins", "kernel-point", "full"})
    if (cl.exist(unsupported)) throw std::string("--") + unsupported + " is not supported";

  const long long n = strip_cli::parse_count(cl.str("n-emissions"));
  const int verbose = cl.count("verbose");
  const double scale = cl.num("scale");
  std::vector<strip_region> regions;
  for (const auto& fn : cl.rest) read_phantom(fn, scale, regions);
  if (cl.exist("point")) {
    const auto p = parse_list(cl.str("point"));
    if (p.size() < 2 || p.size() > 3) throw std::string("--point must specifcy 2 or 3 values x,y[,intensity]");
    regions.push_back(strip_region{STRIP_REGION_POINT, 0, p[0], p[1], 0, 0, 0,
                                   p.size() == 3 ? p[2] : 1.0});
  }
  if (regions.empty()) throw std::string("must specify at least one region");

  strip_geometry g{};
  g.radius = cl.num("radius");
  g.scintillator_length = cl.num("length");
  g.n_y_pixels = cl.integer("n-y-pixels");
  g.n_z_pixels = cl.integer("n-z-pixels");
  g.pixel_height = g.pixel_width = cl.num("s-pixel");
  g.sigma_z = cl.num("s-z");
  g.sigma_dl = cl.num("s-dl");
  double origin[2] = {0, 0};
  if (cl.exist("image-origin")) {
    const auto o = parse_list(cl.str("image-origin"));
    if (o.size() != 2) throw std::string("--image-origin must specify two values for x,y");
    origin[0] = o[0];
    origin[1] = o[1];
  }
  if (verbose) {
    const double size_z = g.n_z_pixels * g.pixel_width, size_y = g.n_y_pixels * g.pixel_height;
    std::cerr << "    image size: " << g.n_z_pixels << " x " << g.n_y_pixels << "\n"
              << "    pixel size: " << g.pixel_width << " x " << g.pixel_height << "\n"
              << "    space size: " << size_z << " x " << size_y << "\n"
              << "space top left: " << -size_z / 2 + g.pixel_width / 2 << " x "
              << size_y / 2 - g.pixel_height / 2 << std::endl;
  }

  const size_t n_pix = (size_t)g.n_y_pixels * g.n_z_pixels;
  const size_t ne = (size_t)std::max<long long>(n, 1);
  std::vector<float> zu(ne), zd(ne), dl(ne);
  std::vector<uint32_t> em(n_pix), det(n_pix);
  strip_simulation opt{};
  opt.additive = cl.exist("additive");
  opt.uniform_angle = !cl.exist("uniform-tan");
  opt.count_emitted = !cl.exist("detected");
  opt.pixel_size = cl.num("s-pixel");
  opt.origin_z = origin[0];
  opt.origin_y = origin[1];
  int64_t written = 0, emitted = 0;
  const int rc = strip_simulate(&g, regions.data(), (int)regions.size(), &opt,
                                (uint64_t)std::strtoull(cl.str("seed").c_str(), nullptr, 10),
                                n, cl.integer("cuda-device"), zu.data(), zd.data(), dl.data(),
                                em.data(), det.data(), &written, &emitted);
  if (rc != STRIP_OK) throw "strip_simulate failed (" + std::to_string(rc) + ")";
  if (verbose)
    std::cerr << " emitted: " << emitted << " events" << std::endl
              << "detected: " << written << " events" << std::endl;

  const std::string output = cl.str("output");
  const std::string base = strip_cli::wo_ext(output);
  const bool text = strip_cli::ext_of(output) == ".txt";
  if (!base.empty() && !cl.exist("no-responses")) {
    if (text) {
      std::ofstream out(output);
      if (!out.is_open()) throw "cannot create output file: " + output;
      for (int64_t i = 0; i < written; ++i) out << zu[i] << ' ' << zd[i] << ' ' << dl[i] << '\n';
    } else {
      std::vector<float> t(3 * (size_t)written);
      for (int64_t i = 0; i < written; ++i) {
        t[3 * i] = zu[i];
        t[3 * i + 1] = zd[i];
        t[3 * i + 2] = dl[i];
      }
      strip_cli::write_raw(output, t.data(), t.size() * sizeof(float));
    }
  }
  if (!base.empty()) {
    {
      std::ofstream cfg(base + ".cfg");
      cl.save(cfg, {"config", "n-pixels", "output", "n-emissions", "tan-bins",
                    "kernel-point", "full", "no-responses", "image-origin",
                    "cuda-device", "help"},
              {"s-z", "s-dl", "scale", "n-z-pixels", "n-y-pixels"});
    }
    // the naive image: the smeared responses' points (from_projection_space_tan,
    // scanner.h:116-134)
    Grid grid{g.n_z_pixels, g.n_y_pixels,
              (float)(-opt.pixel_size * g.n_z_pixels / 2 + origin[0]),
              (float)(-opt.pixel_size * g.n_y_pixels / 2 + origin[1]), (float)opt.pixel_size};
    std::vector<int32_t> naive(n_pix, 0);
    const float R = (float)g.radius;
    for (int64_t i = 0; i < written; ++i) {
      const float tan = (zu[i] - zd[i]) / (2 * R);
      const float y = -0.5f * dl[i] / std::sqrt(1 + tan * tan);
      const float z = 0.5f * (zu[i] + zd[i] + 2 * y * tan);
      int c, r;
      if (grid.at(z, y, c, r)) ++naive[(size_t)r * g.n_z_pixels + c];
    }
    write_image(base + "_detected", std::vector<int32_t>(det.begin(), det.end()), g.n_z_pixels,
                g.n_y_pixels);
    write_image(base + "_emitted", std::vector<int32_t>(em.begin(), em.end()), g.n_z_pixels,
                g.n_y_pixels);
    write_image(base + "_naive", naive, g.n_z_pixels, g.n_y_pixels);
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
  }
  return 1;
}
