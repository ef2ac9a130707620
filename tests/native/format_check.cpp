// The bulk array formatting of the standalone JSON archive
// (mass_hd_b200/host/compat/serialization.hpp: a %.6g conversion written
// from its definition with std::to_chars for the cases it defers, chunks on
// all threads) against the reference's per-value `std::stringstream << v`:
// arrays of doubles (random bit patterns, values at 6-digit rounding
// boundaries, signed zeros, subnormals, infinities), of 9-double nodes and
// of bools, written both ways and compared as text. Prints the number of
// mismatching arrays (0 expected).
#include "serialization.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <sstream>

namespace {

template<class T>
std::string slow(const std::vector<T>& v)
{
  std::string out = "[ ";
  for(std::size_t i = 0; i < v.size(); ++i)
  {
    if(i) out += ", ";
    std::stringstream ss;
    ss << v[i];
    out += ss.str();
  }
  return out + " ]";
}

std::string slow_nodes(const std::vector<std::array<double, 9>>& v)
{
  std::string out = "[ ";
  for(std::size_t i = 0; i < v.size(); ++i)
  {
    if(i) out += ", ";
    std::vector<double> a(v[i].begin(), v[i].end());
    out += slow(a);
  }
  return out + " ]";
}

}

int main()
{
  std::mt19937_64 g(2024);
  std::uniform_real_distribution<double> u(-1, 1);
  int bad = 0;
  for(int rep = 0; rep < 6; ++rep)
  {
    const std::size_t n = rep == 0 ? 0 : rep == 1 ? 1 : 100000 + 37*rep;
    std::vector<double> v(n);
    for(std::size_t i = 0; i < n; ++i)
    {
      switch(i % 5)
      {
        case 0: { uint64_t b = g(); std::memcpy(&v[i], &b, 8); if(v[i] != v[i]) v[i] = 0.0; break; }
        case 1: v[i] = u(g)*std::pow(10.0, static_cast<int>(g() % 60) - 30); break;
        case 2: v[i] = (std::floor(u(g)*1e6) + 0.5)*std::pow(10.0, static_cast<int>(g() % 20) - 10); break;
        case 3: v[i] = (i & 8) ? -0.0 : 0.0; break;
        default: v[i] = (i & 16) ? 4.9e-324*(1 + g() % 100) : 40.0/9 + u(g)*1e-3;
      }
    }
    if(n > 10) { v[3] = std::numeric_limits<double>::infinity(); v[8] = -v[3]; }
    bool badflag = false;
    if(mass_json::format_array(v, badflag) != slow(v)) ++bad;
    std::vector<std::array<double, 9>> nodes(n/9);
    for(std::size_t i = 0; i < nodes.size(); ++i)
      for(int k = 0; k < 9; ++k) nodes[i][k] = v[9*i + k];
    if(mass_json::format_array(nodes, badflag) != slow_nodes(nodes)) ++bad;
    std::vector<bool> mask(n);
    for(std::size_t i = 0; i < n; ++i) mask[i] = (g() & 3) == 0;
    if(mass_json::format_array(mask, badflag) != slow(mask)) ++bad;
    if(badflag) ++bad;
  }
  // the fast %.6g path against the general-purpose conversion, value by
  // value: random bit patterns, wide magnitudes, values at and next to
  // 6-digit rounding ties, integers
  long single = 0;
  for(int i = 0; i < 400000; ++i)
  {
    double vals[5];
    uint64_t b = g();
    std::memcpy(&vals[0], &b, 8);
    if(vals[0] != vals[0]) vals[0] = 1.0;
    vals[1] = u(g)*std::pow(10.0, static_cast<int>(g() % 80) - 40);
    const double tie = (std::floor(u(g)*1e6) + 0.5)*std::pow(10.0, static_cast<int>(g() % 30) - 15);
    vals[2] = tie;
    vals[3] = std::nextafter(tie, (i & 1) ? 1e300 : -1e300);
    vals[4] = static_cast<double>(static_cast<long>(u(g)*1e9));
    for(double x : vals)
    {
      char a[64], c[64];
      *mass_json::put_value(a, x) = 0;
      *mass_json::put_value_exact(c, x) = 0;
      if(std::strcmp(a, c) != 0) ++single;
    }
  }
  if(single) ++bad;
  std::vector<double> withnan = {1.0, std::nan(""), 2.0};
  bool nanflag = false;
  mass_json::format_array(withnan, nanflag);
  if(!nanflag) ++bad;
  std::printf("%d\n", bad);
  return bad != 0;
}
