#include "random.hpp"

#include <random>

namespace {
std::random_device& device()
{
  static std::random_device rd;
  return rd;
}
std::mt19937& engine()
{
  static std::mt19937 gen(device()());
  return gen;
}
}

double random_real(double min, double max)
{
  return std::uniform_real_distribution<>(min, max)(engine());
}

double random_normal(double sigma)
{
  return std::normal_distribution<>(0., sigma)(engine());
}

unsigned randu() { return engine()(); }

void set_seed(unsigned s) { engine().seed(s); }
