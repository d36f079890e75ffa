#include "strip_io.h"

#include "text_parse.h"

#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>

namespace strip_cli {

// ---------------------------------------------------------------------------
// events
// ---------------------------------------------------------------------------

void read_events_binary(const std::string& path, std::vector<float>& z_u,
                        std::vector<float>& z_d, std::vector<float>& dl) {
  std::ifstream in(path, std::ios::binary);
  if (!in.is_open()) throw "cannot open phantom responses file: " + path;
  in.seekg(0, std::ios::end);
  const std::streamoff bytes = in.tellg();
  in.seekg(0, std::ios::beg);
  const size_t n = (size_t)(bytes / 12);
  std::vector<float> t(3 * n);
  if (n && !in.read(reinterpret_cast<char*>(t.data()), (std::streamsize)(12 * n)))
    throw "cannot read phantom responses file: " + path;
  const size_t base = z_u.size();
  z_u.resize(base + n);
  z_d.resize(base + n);
  dl.resize(base + n);
  for (size_t i = 0; i < n; ++i) {
    z_u[base + i] = t[3 * i];
    z_d[base + i] = t[3 * i + 1];
    dl[base + i] = t[3 * i + 2];
  }
}

namespace {

int parse_int_field(const char*& p) { return striptext::parse_int(p); }

}  // namespace

// The reference fast parser's arithmetic lives in the library (text_parse.h).
float parse_fp_reference(const char*& p) {
  float v = 0.0f;
  const char* err = nullptr;
  if (!striptext::parse_fp(p, v, &err)) throw std::string(err);
  return v;
}

void read_events_text(const std::string& path, bool is_3d,
                      std::vector<float>& z_u, std::vector<float>& z_d,
                      std::vector<float>& dl) {
  // util::text_parser::read_lines: 16 KiB buffer, a line is complete at '\n';
  // an unterminated last line is not read.
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd == -1) throw std::string("cannot open input file: ") + path;
  static const size_t kBuffer = 16 * 1024;
  std::vector<char> buf(kBuffer + 1);
  size_t prev = 0;
  for (;;) {
    const ssize_t got = ::read(fd, buf.data() + prev, kBuffer - prev);
    if (got < 0) {
      ::close(fd);
      throw std::string("read failed");
    }
    if (got == 0) break;
    char* end = buf.data() + prev + got;
    char* line = buf.data();
    for (char* nl; (nl = (char*)memchr(line, '\n', end - line)); line = nl + 1) {
      *nl = 0;
      const char* p = line;
      try {
        if (is_3d) {
          parse_int_field(p);
          parse_int_field(p);
        }
        const float a = parse_fp_reference(p);
        const float b = parse_fp_reference(p);
        const float c = parse_fp_reference(p);
        z_u.push_back(a);
        z_d.push_back(b);
        dl.push_back(c);
      } catch (const std::string& e) {
        ::close(fd);
        throw std::string("error line: ") + line + " (" + e + ")";
      }
    }
    prev = end - line;
    if (prev) std::memmove(buf.data(), line, prev);
    if (prev >= kBuffer) {  // a line longer than the buffer
      ::close(fd);
      throw std::string("line too long in ") + path;
    }
  }
  ::close(fd);
}

// ---------------------------------------------------------------------------
// images
// ---------------------------------------------------------------------------

void write_raw(const std::string& path, const void* data, size_t bytes) {
  std::ofstream out(path, std::ios::binary);
  if (!out.is_open()) throw "cannot create output file: " + path;
  out.write(static_cast<const char*>(data), (std::streamsize)bytes);
}

void write_nrrd_header(const std::string& path, const std::string& data_file,
                       int width, int height, bool textual, const char* type) {
  std::ofstream out(path);
  if (!out.is_open()) throw "cannot create output file: " + path;
  out << "NRRD0001" << std::endl
      << "type: " << type << std::endl
      << "endian: little" << std::endl
      << "dimension: 2" << std::endl
      << "sizes: " << width << " " << height << std::endl
      << "data file: ./" << data_file << std::endl
      << "encoding: " << (textual ? "ascii" : "raw") << std::endl;
}

void write_text_map(const std::string& path, const float* data, int width,
                    int height) {
  std::ofstream out(path);
  if (!out.is_open()) throw "cannot create output file: " + path;
  const size_t n = (size_t)width * height;
  for (size_t i = 0; i < n; ++i) {
    out << data[i];
    out << (((i + 1) % (size_t)width) == 0 ? "\n" : " ");
  }
}

void write_tuples(const std::string& path, const float* data, int width,
                  int height) {
  std::ofstream out(path);
  if (!out.is_open()) throw "cannot create output file: " + path;
  out.precision(12);
  out << std::fixed;
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      const float v = data[(size_t)y * width + x];
      if (v >= (float)0.000000000001) out << x << ' ' << y << ' ' << v << std::endl;
    }
}

namespace {

uint32_t crc32(const uint8_t* p, size_t n, uint32_t crc = 0) {
  static std::array<uint32_t, 256> table = [] {
    std::array<uint32_t, 256> t{};
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      t[i] = c;
    }
    return t;
  }();
  crc = ~crc;
  for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
  return ~crc;
}

void put32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back(x >> 24);
  v.push_back(x >> 16);
  v.push_back(x >> 8);
  v.push_back(x);
}

void chunk(std::ofstream& out, const char* type, const std::vector<uint8_t>& body) {
  std::vector<uint8_t> c;
  put32(c, (uint32_t)body.size());
  c.insert(c.end(), type, type + 4);
  c.insert(c.end(), body.begin(), body.end());
  put32(c, crc32(c.data() + 4, c.size() - 4));
  out.write(reinterpret_cast<const char*>(c.data()), (std::streamsize)c.size());
}

}  // namespace

void write_png(const std::string& path, const float* data, int width,
               int height, double scale_max) {
  // pixel = max(0, 255 - gain * value), gain = 255 / max (png_writer.h:40-61)
  double out_max = scale_max;
  if (out_max == 0)
    for (size_t i = 0; i < (size_t)width * height; ++i)
      out_max = std::max(out_max, (double)data[i]);
  const double gain = 255.0 / out_max;
  std::vector<uint8_t> raw;
  raw.reserve((size_t)(width + 1) * height);
  for (int y = 0; y < height; ++y) {
    raw.push_back(0);  // filter: none
    for (int x = 0; x < width; ++x) {
      const double v = std::max(0.0, 255.0 - gain * data[(size_t)y * width + x]);
      raw.push_back((uint8_t)v);
    }
  }
  // zlib stream of stored deflate blocks
  std::vector<uint8_t> z = {0x78, 0x01};
  size_t pos = 0;
  uint32_t a = 1, b = 0;
  for (uint8_t c : raw) {
    a = (a + c) % 65521u;
    b = (b + a) % 65521u;
  }
  do {
    const size_t len = std::min<size_t>(65535, raw.size() - pos);
    const bool last = pos + len == raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back(len & 0xFF);
    z.push_back(len >> 8);
    z.push_back(~len & 0xFF);
    z.push_back((~len >> 8) & 0xFF);
    z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + len);
    pos += len;
  } while (pos < raw.size());
  put32(z, (b << 16) | a);
  std::ofstream out(path, std::ios::binary);
  if (!out.is_open()) throw "cannot create output file: " + path;
  static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
  out.write(reinterpret_cast<const char*>(sig), 8);
  std::vector<uint8_t> ihdr;
  put32(ihdr, (uint32_t)width);
  put32(ihdr, (uint32_t)height);
  ihdr.insert(ihdr.end(), {8, 0, 0, 0, 0});  // 8-bit grey
  chunk(out, "IHDR", ihdr);
  chunk(out, "IDAT", z);
  chunk(out, "IEND", {});
}

}  // namespace strip_cli
