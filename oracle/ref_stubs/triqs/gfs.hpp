// Stand-in for the parts of TRIQS 3.0 (gfs, arrays, h5) that keldy's hot-path sources use.
// Test infrastructure only (see oracle/ref_stubs/README.md).
#pragma once
#include "utility/first_include.hpp"
#include <cmath>
#include <complex>
#include <memory>
#include <string>
#include <vector>

namespace h5 {
struct group {
  group create_group(std::string const &) { return {}; }
  group open_group(std::string const &) const { return {}; }
};
template <typename T> void h5_write(group &, std::string const &, T const &) {}
template <typename T> void h5_read(group &, std::string const &, T &) {}
template <typename T> void h5_write_attribute(group &, std::string const &, T const &) {}
} // namespace h5
using h5::h5_read;
using h5::h5_write;
using h5::h5_write_attribute;

namespace triqs::arrays {

template <typename T> class matrix {
  int n1_ = 0, n2_ = 0;
  std::vector<T> d_;

 public:
  matrix() = default;
  matrix(int n1, int n2) : n1_(n1), n2_(n2), d_(static_cast<size_t>(n1) * n2) {}
  T &operator()(int i, int j) { return d_[static_cast<size_t>(i) * n2_ + j]; }
  T const &operator()(int i, int j) const { return d_[static_cast<size_t>(i) * n2_ + j]; }
  int extent0() const { return n1_; }
  int extent1() const { return n2_; }
};

// Partial-pivot LU in LAPACK zgetf2 order (pivot: first maximum of |re|+|im| in the
// column; multipliers formed with the reciprocal of the pivot), det = product of the
// pivots times the permutation sign.
template <typename T> T determinant(matrix<T> const &m_in) {
  int n = m_in.extent0();
  matrix<T> a = m_in;
  T det = 1.0;
  int swaps = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::abs(a(k, k).real()) + std::abs(a(k, k).imag());
    for (int i = k + 1; i < n; ++i) {
      double v = std::abs(a(i, k).real()) + std::abs(a(i, k).imag());
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (best == 0.0) return T(0.0);
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(a(k, j), a(p, j));
      swaps++;
    }
    T piv = a(k, k);
    det *= piv;
    T inv = T(1.0) / piv;
    for (int i = k + 1; i < n; ++i) a(i, k) *= inv;
    for (int i = k + 1; i < n; ++i) {
      T l = a(i, k);
      for (int j = k + 1; j < n; ++j) a(i, j) -= l * a(k, j);
    }
  }
  return (swaps & 1) ? -det : det;
}

template <typename T> class vector {
  std::vector<T> d_;

 public:
  vector() = default;
  explicit vector(long n) : d_(static_cast<size_t>(n)) {}
  T &operator[](long i) { return d_[static_cast<size_t>(i)]; }
  T const &operator[](long i) const { return d_[static_cast<size_t>(i)]; }
  long size() const { return static_cast<long>(d_.size()); }
  T *data_start() { return d_.data(); }
  T const *data_start() const { return d_.data(); }
  vector &operator()() { return *this; }
  vector &operator/=(T x) {
    for (auto &v : d_) v /= x;
    return *this;
  }
};

} // namespace triqs::arrays

namespace triqs::gfs {

struct retime {};
struct refreq {};
struct matrix_valued {};
struct scalar_real_valued {};

struct stub_linear_mesh {
  double xmin = 0, xmax = 0;
  long L = 0;
  double x_max() const { return xmax; }
  double x_min() const { return xmin; }
  long size() const { return L; }
};

template <typename M, typename T> class gf;

// Matrix-valued Green function on the uniform time mesh; values stored as [L][2][2].
template <typename M> class gf<M, matrix_valued> {
 public:
  stub_linear_mesh m_;
  std::vector<std::complex<double>> data_;

  struct value2x2 {
    std::complex<double> v[2][2];
    std::complex<double> operator()(int i, int j) const { return v[i][j]; }
  };

  gf() = default;
  gf(double xmin, double xmax, long L) : m_{xmin, xmax, L}, data_(static_cast<size_t>(L) * 4) {}

  stub_linear_mesh const &mesh() const { return m_; }
  std::complex<double> &at(long i, int o1, int o2) { return data_[static_cast<size_t>(i) * 4 + o1 * 2 + o2]; }

  // Linear interpolation on the uniform mesh; the last interval is closed at x_max.
  value2x2 operator()(double x) const {
    double delta = (m_.xmax - m_.xmin) / static_cast<double>(m_.L - 1);
    double a = (x - m_.xmin) / delta;
    long i = static_cast<long>(std::floor(a));
    if (i == m_.L - 1) i = m_.L - 2;
    if (i < 0 || i > m_.L - 2) TRIQS_RUNTIME_ERROR << "gf evaluated outside its time window: " << x;
    double w = a - static_cast<double>(i);
    value2x2 r;
    for (int o1 = 0; o1 < 2; ++o1)
      for (int o2 = 0; o2 < 2; ++o2) {
        std::complex<double> g0 = data_[static_cast<size_t>(i) * 4 + o1 * 2 + o2];
        std::complex<double> g1 = data_[static_cast<size_t>(i + 1) * 4 + o1 * 2 + o2];
        r.v[o1][o2] = std::complex<double>((1.0 - w) * g0.real() + w * g1.real(), (1.0 - w) * g0.imag() + w * g1.imag());
      }
    return r;
  }
};

template <typename M> class gf<M, scalar_real_valued> {
 public:
  gf() = default;
};

template <typename M, typename T> class block_gf {
 public:
  std::vector<gf<M, T>> blocks;
  block_gf() = default;
  gf<M, T> const &operator[](int i) const { return blocks[static_cast<size_t>(i)]; }
  gf<M, T> &operator[](int i) { return blocks[static_cast<size_t>(i)]; }
};

} // namespace triqs::gfs
