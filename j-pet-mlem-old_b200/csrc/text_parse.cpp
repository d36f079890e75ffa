// The reference's fast text parser arithmetic (text_parse.h) and the text
// response reader of the 3D hybrid path (hybrid_parse_responses_text in
// include/hybridmlem.h).
#include "text_parse.h"

#include <array>
#include <cstdint>
#include <cstring>
#include <string>

#include "hybridmlem.h"
#include "stripmlem.h"

namespace striptext {

namespace {

constexpr int kMaxExponent = 300;

int parse_digits(const char*& p, int& n_digits) {
  n_digits = 0;
  uint32_t sum = 0;
  while (*p >= '0' && *p <= '9') {
    sum = sum * 10u + (uint32_t)(*p - '0');
    ++p;
    ++n_digits;
  }
  return (int32_t)sum;
}

int parse_sign(const char*& p) {
  if (*p == '-') {
    ++p;
    return -1;
  }
  if (*p == '+') ++p;
  return 1;
}

float pow10_neg(int e) {
  static const std::array<float, kMaxExponent + 1> cache = [] {
    std::array<float, kMaxExponent + 1> c{};
    c[0] = 1.0f;
    for (int i = 1; i <= kMaxExponent; ++i) c[i] = 0.1f * c[i - 1];
    return c;
  }();
  return cache[e];
}

float pow10_pos(int e) { return e == 0 ? 1.0f : 10.0f * pow10_neg(e - 1); }

}  // namespace

bool parse_fp(const char*& p, float& out, const char** err) {
  while (*p == ' ') ++p;
  int n_whole;
  const int sign = parse_sign(p);
  const int whole = parse_digits(p, n_whole);
  float val = (float)whole;
  if (*p == '.') {
    ++p;
    int n_frac = 0;
    const int frac = parse_digits(p, n_frac);
    if (n_whole == 0 && n_frac == 0) {
      *err = "period with no digits either before or after";
      return false;
    }
    if (n_frac > 0) {
      const float scaled = (float)frac * pow10_neg(n_frac < kMaxExponent ? n_frac : kMaxExponent);
      val = val + scaled;
    }
  } else if (n_whole == 0) {
    *err = "neither whole part nor period";
    return false;
  }
  if (*p == 'e' || *p == 'E') {
    ++p;
    int n_exp;
    const int esign = parse_sign(p);
    const int e = (int)((unsigned)esign * (unsigned)parse_digits(p, n_exp));
    if (n_exp == 0) {
      *err = "found exponent char but no exponent";
      return false;
    }
    if (e > kMaxExponent || e < -kMaxExponent) {
      *err = "exponent out of range";
      return false;
    }
    if (e > 0) val = val * pow10_pos(e);
    else if (e < 0) val = val * pow10_neg(-e);
  }
  out = val * (float)sign;
  return true;
}

int parse_int(const char*& p) {
  while (*p == ' ') ++p;
  const int sign = parse_sign(p);
  int nd;
  return (int)((unsigned)sign * (unsigned)parse_digits(p, nd));
}

}  // namespace striptext

extern "C" int hybrid_parse_responses_text(const char* text, int64_t length, int64_t capacity,
                                           int16_t* first, int16_t* second, float* z_up,
                                           float* z_dn, float* dl, int64_t* n_lines) {
  if (!text || length < 0 || capacity < 0 || !n_lines ||
      (capacity > 0 && (!first || !second || !z_up || !z_dn || !dl)))
    return STRIP_E_INVALID;
  int64_t k = 0;
  const char* end = text + length;
  const char* line = text;
  std::array<char, 512> tmp;
  for (const char* nl; line < end && (nl = (const char*)memchr(line, '\n', end - line));
       line = nl + 1, ++k) {
    if (k >= capacity) continue;  // counting only
    // the parser stops at the first character it does not take; a copy of
    // the line ends it with a NUL, as the reference's buffer does
    const size_t len = (size_t)(nl - line);
    std::string big;
    const char* p;
    if (len < tmp.size()) {
      std::memcpy(tmp.data(), line, len);
      tmp[len] = 0;
      p = tmp.data();
    } else {
      big.assign(line, len);
      p = big.c_str();
    }
    const char* err = nullptr;
    const int a = striptext::parse_int(p);
    const int b = striptext::parse_int(p);
    float u, v, w;
    if (!striptext::parse_fp(p, u, &err) || !striptext::parse_fp(p, v, &err) ||
        !striptext::parse_fp(p, w, &err)) {
      *n_lines = k;
      return STRIP_E_INVALID;
    }
    first[k] = (int16_t)(uint16_t)(uint32_t)a;
    second[k] = (int16_t)(uint16_t)(uint32_t)b;
    z_up[k] = u;
    z_dn[k] = v;
    dl[k] = w;
  }
  *n_lines = k;
  return STRIP_OK;
}
