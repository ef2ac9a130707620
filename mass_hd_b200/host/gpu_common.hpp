// Shared pieces of the GPU model plugins (LyotropicGPU, NematicGPU).
//
// Compiles both inside the reference tree (against its header.hpp,
// models.hpp, random.hpp, error_msg.hpp) and in the standalone build
// (against host/compat/). Talks to the device only through the C ABI of
// include/mass_lb.h.
#ifndef MASS_GPU_COMMON_HPP_
#define MASS_GPU_COMMON_HPP_

#include "mass_lb.h"

#include <array>
#include <cmath>
#include <string>
#include <vector>

namespace mass_gpu {

/** One site of D2Q9 populations, as the frame JSON writes it. */
using Node = std::array<double, 9>;

/** The reference's second-order equilibrium (src/lb.hpp:24-41), same
 * operand order so host-configured states match the reference's bit for
 * bit. */
inline Node equilibrium(double vx, double vy, double nn)
{
  Node fe;
  const double v2 = vx*vx + vy*vy;
  fe[1] = nn*(1./9. + 1./3.*vx + 1./3.*v2 - 1./2.*vy*vy);
  fe[2] = nn*(1./9. - 1./3.*vx + 1./3.*v2 - 1./2.*vy*vy);
  fe[3] = nn*(1./9. + 1./3.*vy - 1./2.*vx*vx + 1./3.*v2);
  fe[4] = nn*(1./9. - 1./3.*vy - 1./2.*vx*vx + 1./3.*v2);
  fe[5] = nn*(1./36. + 1./12.*vx + 1./12.*vy + 1./12.*v2 + 1./4.*vx*vy);
  fe[6] = nn*(1./36. - 1./12.*vx - 1./12.*vy + 1./12.*v2 + 1./4.*vx*vy);
  fe[7] = nn*(1./36. - 1./12.*vx + 1./12.*vy + 1./12.*v2 - 1./4.*vx*vy);
  fe[8] = nn*(1./36. + 1./12.*vx - 1./12.*vy + 1./12.*v2 - 1./4.*vx*vy);
  fe[0] = nn-fe[1]-fe[2]-fe[3]-fe[4]-fe[5]-fe[6]-fe[7]-fe[8];
  return fe;
}

/** |a - b| for unsigned values (the reference's diff, src/tools.hpp). */
inline unsigned udiff(unsigned a, unsigned b) { return a > b ? a - b : b - a; }

/** Periodic distance min(x % L, L - x % L) (the reference's wrap). */
inline unsigned uwrap(unsigned x, unsigned L) { return std::min(x%L, L - x%L); }

/** "fp32" / "fp64" -> MASS_LB_FP32 / MASS_LB_FP64, -1 otherwise. */
inline int precision_code(const std::string& s)
{
  if(s == "fp32" || s == "float" || s == "single") return MASS_LB_FP32;
  if(s == "fp64" || s == "double") return MASS_LB_FP64;
  return -1;
}

/** Text of a failed C-ABI call. */
inline std::string abi_error(const char* what, int code)
{
  return std::string(what) + " failed (" + std::to_string(code) + "): " + mass_lb_last_error();
}

/** Flatten site-major populations to the C-ABI layout ff[9*k + v]. */
inline void flatten(const std::vector<Node>& ff, std::vector<double>& out)
{
  out.resize(9*ff.size());
  for(size_t k = 0; k < ff.size(); ++k)
    for(int v = 0; v < 9; ++v) out[9*k + v] = ff[k][v];
}

inline void unflatten(const std::vector<double>& in, std::vector<Node>& ff)
{
  ff.resize(in.size()/9);
  for(size_t k = 0; k < ff.size(); ++k)
    for(int v = 0; v < 9; ++v) ff[k][v] = in[9*k + v];
}

} // namespace mass_gpu

#endif
