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

void write_raw(const std::string& path, const void* data, size_t bytes);
void write_nrrd_header(const std::string& path, const std::string& data_file,
                       int width, int height, bool textual);
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
