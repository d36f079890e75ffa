// The reference's fast text parser (util::text_parser, src/util/text_parser.h:
// 82-175) restated with the same binary32 arithmetic, so that text event and
// response files parse to the binary32 values the reference reads: blanks
// skipped, digits accumulated in a wrapping 32-bit int, value = whole +
// frac * 0.1^n_frac with 0.1^n built as 0.1f * 0.1^(n-1), positive exponents
// as 10 * 0.1^(e-1) (only e <= 1 is a true power of ten), the sign applied
// last.  Compiled without FMA contraction.  Internal to the library and its
// command-line tools.
#pragma once

namespace striptext {

// One binary32 value; advances p.  On a malformed number returns false and
// sets *err to a message (the reference's exception text).
bool parse_fp(const char*& p, float& out, const char** err);
// One integer field (blanks, sign, digits; wrapping); advances p.
int parse_int(const char*& p);

}  // namespace striptext
