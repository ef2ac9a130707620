// Division / death masks of the lyotropic division models: the circles of
// SetMasks (src/models/lyotropic-with-division.cpp:54-69 and :87-105).
//
// The reference marks site k when, for some centre c,
//   wrap(diff(yk, cy), LY)^2 + wrap(diff(xk, cx), LX)^2 <= ceil(radius^2)
// with wrap(d, L) = min(d % L, L - d % L) (src/tools.hpp:30-63), testing
// every site against every centre: O(sites x centres), which at the shipped
// runcards' 500^2 sites and thousands of centres costs ~100 ms per draw.
// stamp_circles writes the same set by visiting, for each centre, the
// offsets (dx, dy) with dx^2 + dy^2 <= ceil(radius^2):
//  * a stamped site is at periodic distance <= |dx|, |dy| from the centre,
//    so the reference marks it too;
//  * a site the reference marks lies at periodic distances (ddx, ddy) with
//    ddx^2 + ddy^2 <= ceil(radius^2), i.e. at the stamped offset (ddx, ddy)
//    up to sign.
// Cost O(centres x radius^2); the mask is identical bit for bit.
#ifndef MASS_GPU_MASK_DRAW_HPP_
#define MASS_GPU_MASK_DRAW_HPP_

#include <array>
#include <cmath>
#include <vector>

namespace mass_gpu {

inline void stamp_circles(std::vector<bool>& mask,
                          const std::vector<std::array<unsigned, 2>>& centers,
                          double radius, unsigned LX, unsigned LY)
{
  mask.assign(static_cast<size_t>(LX)*LY, false);
  const double r2 = std::ceil(radius*radius);
  if(centers.empty() || !(r2 >= 0)) return;
  const long R = static_cast<long>(std::floor(std::sqrt(r2)));
  const long lx = static_cast<long>(LX), ly = static_cast<long>(LY);
  for(const auto& c : centers)
  {
    for(long dx = -R; dx <= R; ++dx)
    {
      const long x = ((static_cast<long>(c[0]) + dx) % lx + lx) % lx;
      for(long dy = -R; dy <= R; ++dy)
      {
        if(static_cast<double>(dx*dx + dy*dy) > r2) continue;
        const long y = ((static_cast<long>(c[1]) + dy) % ly + ly) % ly;
        mask[static_cast<size_t>(y + ly*x)] = true;
      }
    }
  }
}

} // namespace mass_gpu

#endif
