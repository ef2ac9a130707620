// JSON archive with the layout of the reference's writer
// (src/serialization.hpp:187-274, src/serialization.cpp:9-92):
//   { "id" : ..., "version" : ..., "data" : { "name" : { "type" : ...,
//   "value" : ... }, ... } }
// two-space indentation, iterables as "[ a, b ]" and typed "array(...)",
// scalars through a default std::stringstream (6 significant digits),
// NaN detection. `auto_name(x)` pairs a member with its source name, which
// becomes the JSON key. Standalone build of the GPU plugin only.
#ifndef MASS_GPU_COMPAT_SERIALIZATION_HPP_
#define MASS_GPU_COMPAT_SERIALIZATION_HPP_

#include <array>
#include <ostream>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

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
  template<class T, class A> void value(const std::vector<T, A>& v) { iterable(v); }
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
