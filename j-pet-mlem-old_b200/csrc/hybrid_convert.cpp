// Gaussian smearing of converted GATE responses (hybrid_smear_responses in
// include/hybridmlem.h): the reference's 3d_tool_convert draws the errors
// from std::normal_distribution<double> over one std::mt19937_64 seeded with
// --seed (src/3d/tool/convert_cmd.cpp:92-95), in output order: z_up, z_dn,
// dl of the first response, then of the next.  Both are specified by the C++
// standard (the engine exactly; the normal distribution by the standard
// library's algorithm), so the same standard library reproduces its values.
#include <cstdint>
#include <random>

#include "hybridmlem.h"
#include "stripmlem.h"

extern "C" int hybrid_smear_responses(int64_t seed, double sigma_z, double sigma_dl,
                                      int64_t n, double* z_up, double* z_dn, double* dl) {
  if (n < 0 || (n > 0 && (!z_up || !z_dn || !dl)) || !(sigma_z >= 0) || !(sigma_dl >= 0))
    return STRIP_E_INVALID;
  std::normal_distribution<double> z_error(0, sigma_z);
  std::normal_distribution<double> dl_error(0, sigma_dl);
  std::mt19937_64 rng((std::mt19937_64::result_type)seed);
  for (int64_t i = 0; i < n; ++i) {
    z_up[i] += z_error(rng);
    z_dn[i] += z_error(rng);
    dl[i] += dl_error(rng);
  }
  return STRIP_OK;
}
