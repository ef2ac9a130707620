// The standalone build's random stream (mass_hd_b200/host/compat/random.cpp,
// its own Mersenne Twister) against the standard library's std::mt19937
// with uniform_real_distribution and normal_distribution: for several
// seeds, a mixed sequence of random_real (default and other ranges),
// random_reals in bulk, randu and random_normal must give exactly the
// values the standard engine gives. Prints the number of mismatches.
#include "random.hpp"

#include <cstdio>
#include <random>
#include <vector>

int main()
{
  long bad = 0, n = 0;
  auto same = [&](double a, double b) { ++n; if(!(a == b) && !(a != a && b != b)) ++bad; };
  for(unsigned seed : {0u, 1u, 42u, 1001u, 4294967295u})
  {
    set_seed(seed);
    std::mt19937 g(seed);
    for(int i = 0; i < 3000; ++i) same(random_real(), std::uniform_real_distribution<>(0., 1.)(g));
    for(int i = 0; i < 200; ++i)
      same(random_real(-2., 5.), std::uniform_real_distribution<>(-2., 5.)(g));
    std::vector<double> bulk(100003);
    random_reals(bulk.data(), bulk.size());
    for(double v : bulk) same(v, std::uniform_real_distribution<>(0., 1.)(g));
    for(int i = 0; i < 1000; ++i) same(randu(), g());
    for(int i = 0; i < 1000; ++i) same(random_normal(), std::normal_distribution<>(0., 1.)(g));
    for(int i = 0; i < 500; ++i) same(random_normal(0.3), std::normal_distribution<>(0., 0.3)(g));
    random_reals(bulk.data(), 7);
    for(int i = 0; i < 7; ++i) same(bulk[i], std::uniform_real_distribution<>(0., 1.)(g));
    same(random_real(), std::uniform_real_distribution<>(0., 1.)(g));
    // bulk runs starting at odd word offsets, so pairs straddle the blocks
    for(int k = 0; k < 5; ++k)
    {
      same(randu(), g());
      const size_t m = 311 + 977*k;
      random_reals(bulk.data(), m);
      for(size_t i = 0; i < m; ++i) same(bulk[i], std::uniform_real_distribution<>(0., 1.)(g));
    }
  }
  std::printf("%ld of %ld\n", bad, n);
  return bad != 0;
}
