// Test infrastructure (oracle side only): a no-op stand-in for the
// reference's util::png_writer (src/util/png_writer.h), linked into the
// reference's own 2d_strip_reconstruction when it is compiled under
// oracle/_ref.  The image has no libpng, and the reference's CPU path always
// opens a PNG writer when -o is given (src/2d/strip/reconstruction_cmd.cpp:279),
// so without this shim the reference throws "PNG support is not available".
// Nothing is written; only the class's out-of-line members are defined.
#include <string>

#include "util/png_writer.h"

namespace util {

png_writer::png_writer(std::string fn, double scale_max)
    : priv(nullptr), scale_max(scale_max) {
  (void)fn;
}

void png_writer::priv_write_header(unsigned int, unsigned int, unsigned int) {}

void png_writer::priv_write_row(unsigned char*) {}

png_writer::~png_writer() {}

}  // namespace util
