// Minimal stand-in for the part of boost::program_options that the MASS
// model translation units use (test infrastructure for the oracle only).
//
// The reference model files declare their runcard options with
//   opt::options_description d("caption");
//   d.add_options()("name", opt::value<T>(&member), "help")("flag", "help");
// and return them as std::vector<options_description> (src/models.hpp:9).
// Boost itself is not installed here, so this header provides exactly that
// surface, plus set_option(name, text) so the oracle harness can assign an
// option by name the way a runcard line `name = text` would.
#ifndef MASS_ORACLE_BOOST_PROGRAM_OPTIONS_SHIM_HPP_
#define MASS_ORACLE_BOOST_PROGRAM_OPTIONS_SHIM_HPP_

#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace boost {
namespace program_options {

struct value_semantic
{
  virtual ~value_semantic() {}
  /** Parse text into the bound variable; false if the text does not parse. */
  virtual bool assign(const std::string& text) = 0;
};

template<class T>
struct typed_value : value_semantic
{
  T* target;
  explicit typed_value(T* t) : target(t) {}
  typed_value* default_value(const T& v) { if(target) *target = v; return this; }
  typed_value* implicit_value(const T& v) { (void)v; return this; }
  bool assign(const std::string& text) override
  {
    std::istringstream is(text);
    T v{};
    is >> v;
    if(is.fail()) return false;
    *target = v;
    return true;
  }
};

template<>
inline bool typed_value<std::string>::assign(const std::string& text)
{
  *target = text;
  return true;
}

template<class T>
typed_value<T>* value(T* t) { return new typed_value<T>(t); }

inline typed_value<bool>* bool_switch(bool* t)
{
  if(t) *t = false;
  return new typed_value<bool>(t);
}

class options_description
{
public:
  struct entry
  {
    std::string name;
    std::shared_ptr<value_semantic> semantic;
    std::string help;
  };

  explicit options_description(const std::string& caption = "")
    : caption_(caption) {}

  struct easy_init
  {
    options_description* owner;
    easy_init& operator()(const char* name, value_semantic* s, const char* help)
    {
      owner->entries_.push_back({name, std::shared_ptr<value_semantic>(s), help});
      return *this;
    }
    easy_init& operator()(const char* name, const char* help)
    {
      owner->entries_.push_back({name, nullptr, help});
      return *this;
    }
  };

  easy_init add_options() { return easy_init{this}; }

  options_description& add(const options_description& other)
  {
    for(const auto& e : other.entries_) entries_.push_back(e);
    return *this;
  }

  const std::string& caption() const { return caption_; }
  const std::vector<entry>& entries() const { return entries_; }

  /** Assign `text` to option `name`. Returns 0 on success, -1 if the name
   * is unknown, -2 if the text does not parse as the option's type. */
  int set_option(const std::string& name, const std::string& text) const
  {
    for(const auto& e : entries_)
    {
      // "threads,t" style names: the long name is before the comma
      const std::string longname = e.name.substr(0, e.name.find(','));
      if(longname == name)
      {
        if(!e.semantic) return -2;
        return e.semantic->assign(text) ? 0 : -2;
      }
    }
    return -1;
  }

private:
  std::string caption_;
  std::vector<entry> entries_;
};

} // namespace program_options
} // namespace boost

#endif
