// stamp_circles (mass_hd_b200/host/mask_draw.hpp) against the reference's
// per-site circle test (src/models/lyotropic-with-division.cpp:54-69):
// every site against every centre with the periodic distance
// min(d % L, L - d % L). Random centres on lattices from 1x1 up, radii from
// 0 to beyond the lattice. Prints the number of cases and exits non-zero on
// the first mismatch.
#include "mask_draw.hpp"

#include <cstdio>
#include <random>

namespace {

unsigned pdist(unsigned a, unsigned b, unsigned L)
{
  const unsigned d = a > b ? a - b : b - a;
  return d % L < L - d % L ? d % L : L - d % L;
}

}

int main()
{
  std::mt19937 gen(12345);
  const unsigned sizes[][2] = {{1, 1}, {1, 7}, {3, 5}, {16, 12}, {40, 36}, {7, 100}, {64, 64}};
  const double radii[] = {0., 0.3, 1., 1.5, 2.2, 3., 4.9, 7.2, 20., 150.};
  int cases = 0;
  for(const auto& sz : sizes)
    for(double radius : radii)
      for(int ncent : {0, 1, 3, 17})
      {
        const unsigned LX = sz[0], LY = sz[1];
        std::vector<std::array<unsigned, 2>> centers;
        for(int i = 0; i < ncent; ++i)
          centers.push_back({static_cast<unsigned>(gen() % LX), static_cast<unsigned>(gen() % LY)});
        std::vector<bool> got;
        mass_gpu::stamp_circles(got, centers, radius, LX, LY);
        const double r2 = std::ceil(radius*radius);
        for(unsigned k = 0; k < LX*LY; ++k)
        {
          const unsigned yk = k % LY, xk = k / LY;
          bool want = false;
          for(const auto& c : centers)
            if(std::pow(pdist(yk, c[1], LY), 2) + std::pow(pdist(xk, c[0], LX), 2) <= r2)
            {
              want = true;
              break;
            }
          if(got[k] != want)
          {
            std::printf("mismatch LX=%u LY=%u radius=%g site %u\n", LX, LY, radius, k);
            return 1;
          }
        }
        ++cases;
      }
  std::printf("%d\n", cases);
  return 0;
}
