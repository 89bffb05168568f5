// Stand-in for TRIQS's first_include.hpp (test infrastructure; see oracle/ref_stubs/README.md).
#pragma once
#include <complex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <cstdint>
#include <strings.h>
#include <functional>
#include <iostream>
#include <cassert>
#include <cmath>
#define CPP2PY_IGNORE
#define CPP2PY_ARG_AS_DICT
using namespace std::complex_literals;
// TRIQS supplies mixed int/complex arithmetic; keldy's sources rely on it.
inline std::complex<double> operator*(int a, std::complex<double> const &b) { return double(a) * b; }
inline std::complex<double> operator*(std::complex<double> const &b, int a) { return double(a) * b; }
inline std::complex<double> operator+(std::complex<double> const &b, int a) { return b + double(a); }
inline std::complex<double> operator+(int a, std::complex<double> const &b) { return double(a) + b; }
inline std::complex<double> operator-(std::complex<double> const &b, int a) { return b - double(a); }
#include "exceptions.hpp"
