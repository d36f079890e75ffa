// Event and image file formats of the 2d_strip_reconstruction command.
//
// Event files (the reference's two formats, reconstruction_cmd.cpp:169-211):
//   binary: raw little-endian float32 triples z_u z_d dl, no header
//           (util::ibstream, bstream.h:23-26; a trailing partial triple is
//           dropped, as the reference's read-until-eof loop does);
//   text (.txt): one response per line, "z_u z_d dl" (or "i j z_u z_d dl"
//           with --3d-response), parsed with the arithmetic of the
//           reference's fast parser (util::text_parser, text_parser.h:139-175)
//           so that the binary32 values are the ones the reference reads.
// Image files: raw float32 (PixelMap bin, pixel_map.h:149-157), NRRD headers
// (nrrd_writer.h:18-27), text maps and tuples (pixel_map.h:134-147,
// reconstruction.h:203-213), and 8-bit grey PNG (png_writer.h:40-61).
#pragma once

#include <cstdint>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

namespace strip_cli {

// Appends the events of a file to z_u / z_d / dl; throws std::string on error.
void read_events_binary(const std::string& path, std::vector<float>& z_u,
                        std::vector<float>& z_d, std::vector<float>& dl);
void read_events_text(const std::string& path, bool is_3d,
                      std::vector<float>& z_u, std::vector<float>& z_d,
                      std::vector<float>& dl);

// One binary32 value with the reference fast parser's arithmetic; advances p.
float parse_fp_reference(const char*& p);

// path helpers (cmdline_types.h): extension, name without extension / path,
// and add_index(index, max) -> "_<index>" zero-padded to the digits of max.
inline std::string ext_of(const std::string& p) {
  const auto sep = p.find_last_of("\\/"), dot = p.find_last_of('.');
  if (dot == std::string::npos || (sep != std::string::npos && sep > dot)) return "";
  return p.substr(dot);
}
inline std::string wo_ext(const std::string& p) { return p.substr(0, p.size() - ext_of(p).size()); }
inline std::string wo_path(const std::string& p) {
  const auto sep = p.find_last_of("\\/");
  return sep == std::string::npos ? p : p.substr(sep + 1);
}
inline std::string add_index(const std::string& p, int index, int max) {
  int digits = 1;
  for (int m = 10; m <= max; m *= 10) ++digits;
  std::ostringstream os;
  os << p << "_" << std::setw(digits) << std::setfill('0') << index;
  return os.str();
}

void write_raw(const std::string& path, const void* data, size_t bytes);
// type: the NRRD element type ("float" for images, "int" for hit counts)
void write_nrrd_header(const std::string& path, const std::string& data_file,
                       int width, int height, bool textual,
                       const char* type = "float");
// PixelMap text: values separated by ' ', '\n' after each row.
void write_text_map(const std::string& path, const float* data, int width,
                    int height);
// "x y value" for value >= 1e-12, fixed with 12 decimals.
void write_tuples(const std::string& path, const float* data, int width,
                  int height);
// 8-bit grey PNG, value 0 -> white; scale_max 0 = the image maximum.
void write_png(const std::string& path, const float* data, int width,
               int height, double scale_max);

}  // namespace strip_cli
