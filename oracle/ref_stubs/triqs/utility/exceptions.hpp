// Stand-in for TRIQS's exceptions.hpp (test infrastructure).
#pragma once
#include <exception>
#include <sstream>
#include <string>
namespace triqs {
struct runtime_error : std::exception {
  std::string msg;
  template <typename T> runtime_error &operator<<(T const &x) {
    std::ostringstream o;
    o << x;
    msg += o.str();
    return *this;
  }
  const char *what() const noexcept override { return msg.c_str(); }
};
} // namespace triqs
#define TRIQS_RUNTIME_ERROR throw ::triqs::runtime_error{}
