// Subset of boost::program_options used by MASS model plugins: option
// descriptions built with add_options()(name, value<T>(&member), help), plus
// assignment of an option from its runcard text. Part of the standalone
// build of the GPU model plugin; inside the reference tree real boost is used.
#ifndef MASS_GPU_COMPAT_PROGRAM_OPTIONS_HPP_
#define MASS_GPU_COMPAT_PROGRAM_OPTIONS_HPP_

#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace boost {
namespace program_options {

struct value_semantic
{
  virtual ~value_semantic() {}
  virtual bool assign(const std::string& text) = 0;
  virtual bool is_switch() const { return false; }
};

template<class T>
struct typed_value : value_semantic
{
  T* target;
  explicit typed_value(T* t) : target(t) {}
  typed_value* default_value(const T& v) { *target = v; return this; }
  typed_value* implicit_value(const T&) { return this; }
  bool assign(const std::string& text) override
  {
    std::istringstream is(text);
    T v{};
    is >> v;
    if(is.fail()) return false;
    std::string rest;
    if(is >> rest) return false;
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

template<>
inline bool typed_value<bool>::assign(const std::string& text)
{
  if(text.empty() || text == "1" || text == "true" || text == "on" || text == "yes") *target = true;
  else if(text == "0" || text == "false" || text == "off" || text == "no") *target = false;
  else return false;
  return true;
}

template<class T>
typed_value<T>* value(T* t) { return new typed_value<T>(t); }

struct switch_value : typed_value<bool>
{
  using typed_value<bool>::typed_value;
  bool is_switch() const override { return true; }
};

inline typed_value<bool>* bool_switch(bool* t)
{
  *t = false;
  return new switch_value(t);
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

  explicit options_description(const std::string& caption = "") : caption_(caption) {}

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

  /** Assign runcard text to option `name` ("long,s" names match on the long
   * part). 0: assigned; -1: unknown name; -2: text does not parse. */
  int set_option(const std::string& name, const std::string& text) const
  {
    for(const auto& e : entries_)
    {
      const std::string longname = e.name.substr(0, e.name.find(','));
      const std::string shortname =
        e.name.find(',') == std::string::npos ? "" : e.name.substr(e.name.find(',') + 1);
      if(longname == name || (!shortname.empty() && shortname == name))
      {
        if(!e.semantic) return 0;
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
