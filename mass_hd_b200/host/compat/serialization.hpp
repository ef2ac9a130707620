// JSON archive with the layout of the reference's writer
// (src/serialization.hpp:187-274, src/serialization.cpp:9-92):
//   { "id" : ..., "version" : ..., "data" : { "name" : { "type" : ...,
//   "value" : ... }, ... } }
// two-space indentation, iterables as "[ a, b ]" and typed "array(...)",
// scalars as a default std::stringstream prints them (6 significant
// digits), NaN detection. `auto_name(x)` pairs a member with its source
// name, which becomes the JSON key. Standalone build of the GPU plugin only.
//
// Frames are large (a 500^2 go-or-grow frame is 74 MB of text), so the
// field arrays are not printed value by value through a stringstream as the
// reference does: doubles go through std::to_chars with the general format
// at precision 6, which yields the same characters as `stringstream << v`
// (printf's %.6g), and long arrays are formatted in chunks on all host
// threads, then joined in order. The text is identical.
#ifndef MASS_GPU_COMPAT_SERIALIZATION_HPP_
#define MASS_GPU_COMPAT_SERIALIZATION_HPP_

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <ostream>
#include <sstream>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>
#if __cplusplus >= 201703L
#include <charconv>
#endif

#define auto_name(obj) std::pair<decltype(obj)&, std::string> {obj, #obj}

namespace mass_json {

template<class T> struct tname;
#define MASS_JSON_NAME(T, N) template<> struct tname<T> { static std::string get() { return N; } };
MASS_JSON_NAME(bool, "bool")
MASS_JSON_NAME(int, "int")
MASS_JSON_NAME(unsigned, "unsigned")
MASS_JSON_NAME(long, "long")
MASS_JSON_NAME(unsigned long, "unsigned long")
MASS_JSON_NAME(long long, "long long")
MASS_JSON_NAME(unsigned long long, "unsigned long long")
MASS_JSON_NAME(float, "float")
MASS_JSON_NAME(double, "double")
MASS_JSON_NAME(long double, "long double")
MASS_JSON_NAME(std::string, "string")
#undef MASS_JSON_NAME
template<class T, class A> struct tname<std::vector<T, A>>
{ static std::string get() { return "array(" + tname<T>::get() + ")"; } };
template<class T, std::size_t N> struct tname<std::array<T, N>>
{ static std::string get() { return "array(" + tname<T>::get() + ")"; } };

// one value as `std::stringstream() << v` prints it (printf's %.6g), with
// the general-purpose conversion
inline char* put_value_exact(char* p, double v)
{
#if __cplusplus >= 201703L
  return std::to_chars(p, p + 32, v, std::chars_format::general, 6).ptr;
#else
  return p + std::snprintf(p, 32, "%.6g", v);
#endif
}

// 10^i as the nearest double, i in [-330, 330] (index i + 330)
inline const double* pow10_table()
{
  static const double* t = [] {
    static double a[661];
    for(int i = -330; i <= 330; ++i)
    {
      char b[16];
      std::snprintf(b, sizeof b, "1e%d", i);
      a[i + 330] = std::strtod(b, nullptr);
    }
    return a;
  }();
  return t;
}

// %.6g written from its definition (C11 7.21.6.1): the value rounded to 6
// significant digits d0.d1..d5 x 10^X; fixed notation with 5 - X decimals
// when -4 <= X < 6, else d0.d1..d5e+-XX; trailing zeros and a bare decimal
// point removed. The 6-digit rounding is decided from |v| scaled into
// [1e5, 1e6) by a tabulated power of ten, in double arithmetic, whose error
// (a few ulp, below 1e-9 in absolute terms) only matters when the scaled
// value lies within 1e-9 of a rounding tie; those values, zeros,
// non-finite and extreme magnitudes go to put_value_exact. Same characters
// as put_value_exact for every value.
inline char* put_value(char* p, double v, const double* t)
{
  const double a = v < 0 ? -v : v;
  if(!(a >= 1e-290 && a <= 1e290)) return put_value_exact(p, v);
  uint64_t bits;
  std::memcpy(&bits, &a, sizeof bits);
  const int k = static_cast<int>(bits >> 52) - 1023;     // a in [2^k, 2^(k+1))
  int e = (k*78913) >> 18;                                 // floor(k*log10(2)), within 1 of floor(log10 a)
  double sc = 0;
  for(int it = 0; it < 3; ++it)
  {
    sc = a*t[330 + 5 - e];
    if(sc < 99999.9999) --e;
    else if(sc >= 999999.4999) ++e;
    else break;
  }
  if(!(sc >= 99999.9999 && sc < 999999.4999)) return put_value_exact(p, v);
  const long r = static_cast<long>(sc);                   // floor: sc > 0
  const double frac = sc - static_cast<double>(r);
  if(frac > 0.5 - 1e-9 && frac < 0.5 + 1e-9) return put_value_exact(p, v);
  long m = r + (frac > 0.5 ? 1 : 0);
  int X = e;
  if(m >= 1000000) { m /= 10; ++X; }
  char d[6];
  for(int i = 5; i >= 0; --i) { d[i] = static_cast<char>('0' + m % 10); m /= 10; }
  int nd = 6;                       // significant digits after trailing-zero removal
  while(nd > 1 && d[nd - 1] == '0') --nd;
  if(v < 0) *p++ = '-';
  if(X >= -4 && X < 6)
  {
    if(X >= 0)
    {
      for(int i = 0; i <= X; ++i) *p++ = d[i];
      if(nd > X + 1)
      {
        *p++ = '.';
        for(int i = X + 1; i < nd; ++i) *p++ = d[i];
      }
    }
    else
    {
      *p++ = '0';
      *p++ = '.';
      for(int i = 0; i < -X - 1; ++i) *p++ = '0';
      for(int i = 0; i < nd; ++i) *p++ = d[i];
    }
  }
  else
  {
    *p++ = d[0];
    if(nd > 1)
    {
      *p++ = '.';
      for(int i = 1; i < nd; ++i) *p++ = d[i];
    }
    *p++ = 'e';
    int ex = X;
    if(ex < 0) { *p++ = '-'; ex = -ex; }
    else *p++ = '+';
    if(ex >= 100) { *p++ = static_cast<char>('0' + ex/100); ex %= 100; }
    *p++ = static_cast<char>('0' + ex/10);
    *p++ = static_cast<char>('0' + ex%10);
  }
  return p;
}
inline char* put_value(char* p, double v) { return put_value(p, v, pow10_table()); }
inline char* put_value(char* p, bool b) { *p++ = b ? '1' : '0'; return p; }

// element types formatted in bulk, and the most characters one takes
template<class T> struct flat : std::false_type {};
template<> struct flat<double> : std::true_type { static constexpr std::size_t chars = 34; };
template<> struct flat<bool> : std::true_type { static constexpr std::size_t chars = 3; };
template<std::size_t N> struct flat<std::array<double, N>> : std::true_type
{ static constexpr std::size_t chars = 4 + 34*N; };

inline char* put_elem(char* p, double v, bool& bad)
{
  static const double* const t = pow10_table();
  if(v != v) bad = true;
  return put_value(p, v, t);
}
inline char* put_elem(char* p, bool b, bool&) { return put_value(p, b); }
template<std::size_t N>
inline char* put_elem(char* p, const std::array<double, N>& a, bool& bad)
{
  *p++ = '['; *p++ = ' ';
  for(std::size_t i = 0; i < N; ++i)
  {
    if(i) { *p++ = ','; *p++ = ' '; }
    p = put_elem(p, a[i], bad);
  }
  *p++ = ' '; *p++ = ']';
  return p;
}
// "[ a, b, ... ]" of a whole array, in parallel chunks joined in order
template<class V>
std::string format_array(const V& c, bool& bad)
{
  using T = typename V::value_type;
  const std::size_t n = c.size();
  const std::size_t per = flat<T>::chars;
  const std::size_t chunk = 1 << 15;
  const std::size_t nchunks = (n + chunk - 1)/chunk;
  std::vector<std::string> parts(nchunks);
  std::vector<char> badv(nchunks, 0);
  auto work = [&](std::size_t first, std::size_t stride) {
    std::unique_ptr<char[]> buf(new char[(chunk + 1)*per]);   // not zeroed
    for(std::size_t j = first; j < nchunks; j += stride)
    {
      char* p = buf.get();
      bool b = false;
      const std::size_t lo = j*chunk, hi = std::min(n, lo + chunk);
      typename V::const_iterator it = c.begin();
      std::advance(it, lo);
      for(std::size_t i = lo; i < hi; ++i, ++it)
      {
        if(i) { *p++ = ','; *p++ = ' '; }
        p = put_elem(p, *it, b);
      }
      parts[j].assign(buf.get(), p);
      badv[j] = b;
    }
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const std::size_t nthr = std::min<std::size_t>(hw, nchunks);
  if(nthr <= 1) work(0, 1);
  else
  {
    std::vector<std::thread> th;
    for(std::size_t t = 0; t < nthr; ++t) th.emplace_back(work, t, nthr);
    for(auto& t : th) t.join();
  }
  std::size_t total = 4;
  for(const auto& s : parts) total += s.size();
  std::string out;
  out.reserve(total);
  out += "[ ";
  for(const auto& s : parts) out += s;
  out += " ]";
  for(char b : badv) if(b) bad = true;
  return out;
}

} // namespace mass_json

class oarchive
{
  std::ostream& stream;
  unsigned level = 0;
  bool first = true;
  bool f_bad_value = false;

  void open_group() { stream << "{"; ++level; first = true; }
  void close_group()
  {
    --level;
    stream << "\n" << std::string(2*level, ' ') << "}";
    first = false;
  }
  void new_line()
  {
    if(!first) stream << ',';
    else first = false;
    stream << "\n" << std::string(2*level, ' ');
  }
  void add_key(const std::string& key)
  {
    new_line();
    stream << "\"" << key << "\" : ";
  }

  template<class T>
  void element(const T& v)
  {
    if(v != v) f_bad_value = true;
    std::stringstream ss;
    ss << v;
    stream << ss.str();
  }
  void element(const std::string& s) { stream << "\"" << s << "\""; }
  void element(bool b) { std::stringstream ss; ss << b; stream << ss.str(); }
  template<class C>
  void iterable(const C& c)
  {
    stream << "[ ";
    bool f = true;
    for(const auto& x : c)
    {
      if(f) f = false;
      else stream << ", ";
      value(x);
    }
    stream << " ]";
  }
  template<class T> void value(const T& v) { element(v); }
  template<class T, class A>
  void value(const std::vector<T, A>& v) { vector_value(v, mass_json::flat<T>()); }
  template<class V> void vector_value(const V& v, std::true_type)
  { stream << mass_json::format_array(v, f_bad_value); }
  template<class V> void vector_value(const V& v, std::false_type) { iterable(v); }
  template<class T, std::size_t N> void value(const std::array<T, N>& v) { iterable(v); }

public:
  oarchive(std::ostream& os, const std::string& id, unsigned version = 0)
    : stream(os)
  {
    open_group();
    add_key("id"); element(id);
    add_key("version"); element(version);
    add_key("data");
    open_group();
  }
  ~oarchive()
  {
    close_group();
    if(stream.good()) stream << "\n}";
  }

  template<class T>
  oarchive& operator&(const std::pair<T&, std::string>& t)
  {
    add_key(t.second);
    open_group();
    add_key("type");
    element(mass_json::tname<typename std::remove_cv<T>::type>::get());
    add_key("value");
    value(t.first);
    close_group();
    return *this;
  }

  bool bad_value() const { return f_bad_value; }
};

/** Input archive: not implemented, as in the reference. */
struct iarchive
{
  template<class T>
  iarchive& operator&(const std::pair<T&, std::string>&) { return *this; }
};

#endif
