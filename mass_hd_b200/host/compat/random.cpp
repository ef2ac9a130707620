#include "random.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>

namespace {

// The block loops below are built twice, for AVX2 and for the baseline
// x86-64 vector unit, and the loader picks the one the CPU runs.
#if defined(__x86_64__) && defined(__GNUC__) && defined(__ELF__) && !defined(MASS_GPU_NO_CLONES)
#define MT_CLONES __attribute__((target_clones("avx2", "default"), noinline))
#else
#define MT_CLONES
#endif

constexpr uint32_t MT_N = 624, MT_M = 397;

inline uint32_t mt_step(uint32_t xk, uint32_t xk1, uint32_t xkm)
{
  const uint32_t y = (xk & 0x80000000u) | (xk1 & 0x7fffffffu);
  return xkm ^ (y >> 1) ^ ((0u - (y & 1u)) & 0x9908b0dfu);
}

// X[k+N] from X[k], X[k+1], X[k+M], in place and in order: the first N-M
// words read words not yet replaced, the rest read replaced ones at least
// N-M = 227 places back
MT_CLONES void mt_twist(uint32_t* x)
{
  for(uint32_t k = 0; k < MT_N - MT_M; ++k) x[k] = mt_step(x[k], x[k + 1], x[k + MT_M]);
  for(uint32_t k = MT_N - MT_M; k < MT_N - 1; ++k) x[k] = mt_step(x[k], x[k + 1], x[k + MT_M - MT_N]);
  x[MT_N - 1] = mt_step(x[MT_N - 1], x[0], x[MT_M - 1]);
}

MT_CLONES void mt_temper(const uint32_t* x, uint32_t* out)
{
  for(uint32_t k = 0; k < MT_N; ++k)
  {
    uint32_t y = x[k];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    out[k] = y;
  }
}

// generate_canonical<double, 53> of n word pairs (a, b) = (w[2j], w[2j+1]):
// the 64-bit integer u = a + b*2^32 rounded to double, times 2^-64, kept
// below 1. Both halves become exact doubles through the exponent field:
// (2^84 + b*2^32) - (2^84 + 2^52) = b*2^32 - 2^52 and 2^52 + a; their sum
// is u with the single rounding of a + b*2^32.
MT_CLONES void mt_canonical_pairs(const uint32_t* w, double* d, size_t n)
{
  for(size_t j = 0; j < n; ++j)
  {
    uint64_t u;
    std::memcpy(&u, w + 2*j, sizeof u);
    const uint64_t hb = (u >> 32) | 0x4530000000000000ull;
    const uint64_t lb = (u & 0xffffffffull) | 0x4330000000000000ull;
    double h, l;
    std::memcpy(&h, &hb, sizeof h);
    std::memcpy(&l, &lb, sizeof l);
    const double r = ((h - 19342813118337666422669312.0) + l)*0x1p-64;
    d[j] = r >= 1.0 ? 0x1.fffffffffffffp-1 : r;
  }
}

// The 32-bit Mersenne Twister of the C++ standard library
// ([rand.eng.mers], [rand.predef]: std::mt19937 has word size 32, n = 624,
// m = 397, r = 31, a = 0x9908b0df, tempering u = 11, d = 0xffffffff,
// s = 7, b = 0x9d2c5680, t = 15, c = 0xefc60000, l = 18 and seeding
// multiplier 1812433253). The whole block of 624 words is advanced and
// tempered at once, in loops without branches that the compiler turns into
// vector code; the sequence is std::mt19937's for every seed. The mask
// draws of the division models take one random_real() per site with
// phi >= .5, so this generator bounds a go-or-grow step on the host.
class Mt32
{
public:
  using result_type = uint32_t;
  static constexpr result_type min() { return 0u; }
  static constexpr result_type max() { return 0xffffffffu; }

  explicit Mt32(uint32_t s = 5489u) { seed(s); }

  void seed(uint32_t s)
  {
    x[0] = s;
    for(uint32_t i = 1; i < N; ++i) x[i] = 1812433253u*(x[i - 1] ^ (x[i - 1] >> 30)) + i;
    pos = N;
  }

  result_type operator()()
  {
    if(pos == N) refill();
    return out[pos++];
  }

  // n uniform doubles in [0, 1), each from two consecutive words as
  // generate_canonical<double, 53> forms it
  template<class F>
  void fill_pairs(double* dst, size_t n, F&& canonical)
  {
    size_t i = 0;
    while(i < n)
    {
      if(pos == N) refill();
      if(pos + 1 < N)
      {
        const size_t k = std::min(n - i, static_cast<size_t>((N - pos)/2));
        mt_canonical_pairs(out + pos, dst + i, k);
        pos += static_cast<uint32_t>(2*k);
        i += k;
      }
      else
      {
        const uint32_t a = (*this)();
        const uint32_t b = (*this)();
        dst[i++] = canonical(a, b);
      }
    }
  }

private:
  static constexpr uint32_t N = MT_N;
  uint32_t x[N];
  uint32_t out[N];
  uint32_t pos = N;

  void refill()
  {
    mt_twist(x);
    mt_temper(x, out);
    pos = 0;
  }
};

std::random_device& device()
{
  static std::random_device rd;
  return rd;
}
Mt32& engine()
{
  static Mt32 gen(device()());
  return gen;
}

// generate_canonical<double, 53> of two consecutive words a, b:
// (a + b*2^32) / 2^64 rounded to double, kept below 1
inline double canonical(uint32_t a, uint32_t b)
{
  const double r = (static_cast<double>(a) + static_cast<double>(b)*4294967296.0)/
                   18446744073709551616.0;
  return r >= 1.0 ? std::nextafter(1.0, 0.0) : r;
}

} // namespace

double random_real(double min, double max)
{
  Mt32& g = engine();
  const uint32_t a = g();
  const uint32_t b = g();
  return canonical(a, b)*(max - min) + min;
}

void random_reals(double* out, size_t n)
{
  // uniform_real_distribution(0, 1) is x*(1 - 0) + 0 = x
  engine().fill_pairs(out, n, canonical);
}

double random_normal(double sigma)
{
  return std::normal_distribution<>(0., sigma)(engine());
}

unsigned randu() { return engine()(); }

void set_seed(unsigned s) { engine().seed(s); }
