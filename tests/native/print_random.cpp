// Prints n draws of random_real() after set_seed(seed) from the standalone
// plugin build's random stream (mass_hd_b200/host/compat/random.cpp).
#include "random.hpp"
#include <cstdio>
#include <cstdlib>
int main(int argc, char** argv)
{
  if(argc < 3) return 2;
  set_seed(static_cast<unsigned>(std::atoi(argv[1])));
  const int n = std::atoi(argv[2]);
  for(int i = 0; i < n; ++i) std::printf("%.17g\n", random_real());
  return 0;
}
