// error_msg / warning_msg: exceptions built from a list of printable
// arguments, with the type tags the reference's driver catches
// (reference: src/error_msg.hpp). Standalone build only.
#ifndef MASS_GPU_COMPAT_ERROR_MSG_HPP_
#define MASS_GPU_COMPAT_ERROR_MSG_HPP_

#include <exception>
#include <sstream>
#include <string>
#include <utility>

template<typename Tag>
class inline_msg : public std::exception
{
  std::string msg;
  static void put(std::ostream&) {}
  template<class Head, class... Tail>
  static void put(std::ostream& os, Head&& h, Tail&&... t)
  {
    os << std::forward<Head>(h);
    put(os, std::forward<Tail>(t)...);
  }

public:
  template<class... Args>
  explicit inline_msg(Args&&... args)
  {
    std::ostringstream s;
    put(s, std::forward<Args>(args)...);
    msg = s.str();
  }
  const char* what() const noexcept override { return msg.c_str(); }
};

using error_msg = inline_msg<struct Error>;
using warning_msg = inline_msg<struct Warning>;

#endif
