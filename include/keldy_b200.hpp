// keldy's C++ interface for its QMC hot path, running on the keldy_b200 C ABI.
//
// Header-only. The classes keep keldy's names, signatures and value semantics
// (qrng.hpp, warpers/*.hpp, impurity_oneband/{model,wick_direct,compute_obs}.hpp,
// integrator.hpp) so that code written against keldy compiles against this header; the
// work runs on the GPU through include/keldy_b200.h. Errors that keldy raises with
// TRIQS_RUNTIME_ERROR are thrown as std::runtime_error with keldy's message.
//
// Differences from keldy, all forced by running on the device:
//  * warper_product_1d_simple_t is built by the analytic makers (and the uniform maker
//    make_product_1d_simple_uniform); its constructor from arbitrary std::function
//    objects has no device form and throws.
//  * g0_model is built from tables (g0_model::from_tables); the Python layer builds
//    them from model_param_t (keldy_b200.g0_tables).
//  * integrator::reset_rng accepts "sobol_unshifted" and "sobol"; keldy's boost
//    pseudo-random generators are not on the device.
//  * one process drives one GPU; keldy_b200.parallel shards Sobol blocks over ranks.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <memory>
#include <mutex>
#include <array>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "keldy_b200.h"

namespace keldy_b200 {

inline void check(int status) {
  if (status != KB_OK) throw std::runtime_error(kb_last_error());
}

// One context per device, created on first use and kept for the life of the process.
inline kb_context *default_context(int device = 0) {
  static std::mutex mu;
  static kb_context *ctx[64] = {};
  if (device < 0 || device >= 64) throw std::runtime_error("device index out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (!ctx[device]) check(kb_context_create(device, &ctx[device]));
  return ctx[device];
}

} // namespace keldy_b200

namespace keldy {

using dcomplex = std::complex<double>;
using time_real_t = double;
using orbital_t = int;

enum spin_t { up = 0, down = 1 };
enum keldysh_idx_t { forward = 0, backward = 1 };

// Point of the Keldysh contour (common.hpp:45-55).
class contour_pt_t {
 public:
  time_real_t time{};
  keldysh_idx_t k_idx = forward;
  int timesplit_n = 0;
  bool operator==(const contour_pt_t &o) const {
    return time == o.time && k_idx == o.k_idx && timesplit_n == o.timesplit_n;
  }
};

// Contour order (common.cpp:47-57): < 0 if a is earlier on the contour than b.
inline int compare_3way(const contour_pt_t &a, const contour_pt_t &b) {
  int k3 = a.k_idx - b.k_idx;
  if (k3 != 0) return k3;
  double d = a.time - b.time;
  if (d != 0.0) return (1 - 2 * int(a.k_idx)) * (2 * int(!std::signbit(d)) - 1);
  return (1 - 2 * int(a.k_idx)) * (a.timesplit_n - b.timesplit_n);
}

// keldy::sobol (qrng.hpp:49-114). The state is the index k of the last point drawn;
// operator() returns point k+1 (the first draw after seed(s) is point s+1).
class sobol {
  std::shared_ptr<kb_sobol> gen_;
  int dim_ = 0;
  int log_max_points_ = 31;
  uint32_t k_ = 0;

  void make(int dim, bool do_shift, bool do_scramble, int seed_shift) {
    if (log_max_points_ > 31) throw std::runtime_error("To many points requested from Sobol generator.");
    kb_sobol *s = nullptr;
    keldy_b200::check(kb_sobol_create(keldy_b200::default_context(), dim, log_max_points_, do_shift, do_scramble,
                                      seed_shift, &s));
    gen_ = std::shared_ptr<kb_sobol>(s, kb_sobol_destroy);
    dim_ = dim;
  }

 public:
  sobol(int dim, int rng_state_seed, int log_max_points_ = 31) : log_max_points_(log_max_points_) {
    make(dim, false, false, 0);
    seed(rng_state_seed);
  }
  sobol(int dim, int rng_state_seed, bool do_shift, bool do_scramble, int rng_seed_shift, int log_max_points_ = 31)
     : log_max_points_(log_max_points_) {
    make(dim, do_shift, do_scramble, rng_seed_shift);
    seed(rng_state_seed);
  }

  // one point per call (a device round trip); points(count) draws many in one call
  std::vector<double> operator()() { return points(1); }

  // next `count` points, row-major (an addition to keldy's interface)
  std::vector<double> points(int64_t count) {
    if (count > 0 && (uint64_t)k_ >= (1ull << log_max_points_))
      throw std::runtime_error("More sample points requested then generator can hold.");
    std::vector<double> out((size_t)(count * dim_));
    keldy_b200::check(kb_sobol_points(keldy_b200::default_context(), gen_.get(), k_ + 1, count, out.data()));
    k_ += (uint32_t)count;
    return out;
  }

  void seed(int k) { k_ = (uint32_t)k; }
  void discard(int nr_discard) { k_ += (uint32_t)nr_discard; }

  int dimension() const { return dim_; }
  uint32_t state() const { return k_; }
  void set_state(uint32_t k) { k_ = k; }
  const kb_sobol *handle() const { return gen_.get(); }
};

namespace warpers {

// Coordinate maps of the plasma warper (plasma_uv.hpp:35-51), on the device.
inline std::vector<double> vi_from_ui(double t_max, std::vector<double> const &u_times) {
  kb_warper w{KB_WARPER_PLASMA_UV, 0, t_max, 0.0};
  std::vector<double> out(u_times.size());
  if (u_times.empty()) return out;
  keldy_b200::check(kb_warp(keldy_b200::default_context(), &w, 1, KB_FORWARD, 0, 1, (int)u_times.size(), 1,
                            u_times.data(), out.data(), nullptr));
  return out;
}

inline std::vector<double> ui_from_vi(double t_max, std::vector<double> const &v_times) {
  kb_warper w{KB_WARPER_PLASMA_UV, 0, t_max, 0.0};
  std::vector<double> out(v_times.size());
  if (v_times.empty()) return out;
  keldy_b200::check(kb_warp(keldy_b200::default_context(), &w, 1, KB_REVERSE, 1, 0, (int)v_times.size(), 1,
                            v_times.data(), out.data(), nullptr));
  return out;
}

namespace detail {
// map_reverse / map_forward of a chain of warpers on one point.
inline std::pair<std::vector<double>, double> apply(std::vector<kb_warper> const &chain, int direction, int start,
                                                    int end, std::vector<double> const &x) {
  std::vector<double> out(x.size());
  double jac = 1.0;
  if (x.empty()) {
    // keldy's warpers on an empty vector: identity map, Jacobian 1
    return {out, jac};
  }
  keldy_b200::check(kb_warp(keldy_b200::default_context(), chain.data(), (int)chain.size(), direction, start, end,
                            (int)x.size(), 1, x.data(), out.data(), &jac));
  return {out, jac};
}
} // namespace detail

// The concept of a keldy warper (warpers.hpp): map_reverse, map_forward, ui_from_li,
// li_from_ui, jacobian_reverse, jacobian_forward.
class warper_base {
 protected:
  kb_warper desc_{};
  std::shared_ptr<kb_warper_table> table_; // tabulated warpers: keeps the device tables alive

 public:
  const kb_warper &desc() const { return desc_; }
  std::shared_ptr<kb_warper_table> const &table() const { return table_; }
  std::pair<std::vector<double>, double> map_reverse(std::vector<double> const &li_vec) const {
    return detail::apply({desc_}, KB_REVERSE, 1, 0, li_vec);
  }
  std::pair<std::vector<double>, double> map_forward(std::vector<double> const &ui_vec) const {
    return detail::apply({desc_}, KB_FORWARD, 0, 1, ui_vec);
  }
  std::vector<double> ui_from_li(std::vector<double> const &li_vec) const { return map_reverse(li_vec).first; }
  std::vector<double> li_from_ui(std::vector<double> const &ui_vec) const { return map_forward(ui_vec).first; }
  double jacobian_reverse(std::vector<double> const &li_vec) const { return map_reverse(li_vec).second; }
  double jacobian_forward(std::vector<double> const &ui_vec) const { return map_forward(ui_vec).second; }
};

// warpers/identity.hpp:30-49
class warper_identity_t : public warper_base {
 public:
  warper_identity_t() { desc_ = kb_warper{KB_WARPER_IDENTITY, 0, 0.0, 0.0}; }
};

// warpers/plasma_uv.hpp:55-81
class warper_plasma_uv_t : public warper_base {
 public:
  warper_plasma_uv_t(double t_max_ = 0.0) { desc_ = kb_warper{KB_WARPER_PLASMA_UV, 0, t_max_, 0.0}; }
};

// warpers/product_1d_simple.hpp:44-168, built by the makers below.
class warper_product_1d_simple_t : public warper_base {
 public:
  warper_product_1d_simple_t() { desc_ = kb_warper{KB_WARPER_UNIFORM, 0, 1.0, 0.0}; }
  explicit warper_product_1d_simple_t(kb_warper const &d) { desc_ = d; }
  template <typename F1, typename F2, typename F3>
  warper_product_1d_simple_t(F1 &&, F2 &&, F3 &&, double, bool = true) {
    throw std::runtime_error("warper_product_1d_simple_t from arbitrary functions has no device form; use "
                             "make_product_1d_simple_exponential/inverse/inverse_square/inverse_power/uniform");
  }
  // product of the normalised 1-D densities (product_1d_simple.hpp:161-167)
  double operator()(std::vector<double> const &ui_vec) const { return jacobian_forward(ui_vec); }
};

inline warper_product_1d_simple_t make_product_1d_simple_exponential(double domain_u_max, double w_scale) {
  return warper_product_1d_simple_t(kb_warper{KB_WARPER_EXPONENTIAL, 0, domain_u_max, w_scale});
}
inline warper_product_1d_simple_t make_product_1d_simple_inverse(double domain_u_max, double w_scale) {
  return warper_product_1d_simple_t(kb_warper{KB_WARPER_INVERSE, 0, domain_u_max, w_scale});
}
inline warper_product_1d_simple_t make_product_1d_simple_inverse_square(double domain_u_max, double w_scale) {
  return warper_product_1d_simple_t(kb_warper{KB_WARPER_INVERSE_SQUARE, 0, domain_u_max, w_scale});
}
inline warper_product_1d_simple_t make_product_1d_simple_inverse_power(int power, double domain_u_max,
                                                                         double w_scale) {
  return warper_product_1d_simple_t(kb_warper{KB_WARPER_INVERSE_POWER, power, domain_u_max, w_scale});
}
// f1 = 1/u_max on [0, u_max] (keldy writes it with three lambdas, product_1d_simple_test.cpp:10-23)
inline warper_product_1d_simple_t make_product_1d_simple_uniform(double domain_u_max) {
  return warper_product_1d_simple_t(kb_warper{KB_WARPER_UNIFORM, 0, domain_u_max, 0.0});
}

namespace detail {
inline std::shared_ptr<kb_warper_table> own_table(kb_warper_table *t) {
  return std::shared_ptr<kb_warper_table>(t, [](kb_warper_table *p) { kb_warper_table_destroy(p); });
}
inline int table_dims(kb_warper_table const *t) {
  int n = 0;
  keldy_b200::check(kb_warper_table_info(t, nullptr, &n, nullptr));
  return n;
}
inline std::shared_ptr<kb_warper_table> make_table(std::vector<int> const &npts, std::vector<double> const &u,
                                                   std::vector<double> const &f1) {
  kb_warper_table *t = nullptr;
  keldy_b200::check(kb_warper_table_create(keldy_b200::default_context(), (int)npts.size(), npts.data(), u.data(),
                                           f1.data(), &t));
  return std::shared_ptr<kb_warper_table>(t, [](kb_warper_table *p) { kb_warper_table_destroy(p); });
}
} // namespace detail

// product_1d_simple.hpp:174-330: f1 tabulated on points u (u[0] = 0, increasing), linear
// interpolation of its integral and of the inverse, the same table for every coordinate.
class warper_product_1d_simple_interp_nearest_t : public warper_base {
  std::vector<double> u_, f1_;

  void build() {
    table_ = detail::make_table({(int)u_.size()}, u_, f1_);
    desc_ = kb_warper{KB_WARPER_TABLE, 0, u_.back(), 0.0, table_.get()};
  }

 public:
  warper_product_1d_simple_interp_nearest_t(std::vector<double> times_u_pts, std::vector<double> f1_pts)
     : u_(std::move(times_u_pts)), f1_(std::move(f1_pts)) {
    if (f1_.size() != u_.size()) throw std::runtime_error("times_u_pts and f1_pts should have the same length.");
    build();
  }
  // f1 sampled on nr_sample_points equidistant points of [0, domain_u_max] (:295-318)
  warper_product_1d_simple_interp_nearest_t(std::function<double(double)> const &f1, double domain_u_max,
                                            int nr_sample_points) {
    if (!(nr_sample_points >= 3))
      throw std::runtime_error("Expect nr_sample_points to be >= 3. Given was " + std::to_string(nr_sample_points));
    u_.resize((size_t)nr_sample_points);
    f1_.resize((size_t)nr_sample_points);
    for (int i = 0; i < nr_sample_points; ++i)
      u_[(size_t)i] = 0.0 + static_cast<double>(i) / (nr_sample_points - 1) * (domain_u_max - 0.0);
    u_.back() = domain_u_max;
    for (int i = 0; i < nr_sample_points; ++i) f1_[(size_t)i] = f1(u_[(size_t)i]);
    build();
  }
  std::vector<double> const &get_times_u_pts() const { return u_; }
  std::vector<double> const &get_f1_pts() const { return f1_; }
};

// product_1d.hpp:164-211: one tabulated warper per coordinate.
class warper_product_1d_interp_nearest_t : public warper_base {
  std::vector<warper_product_1d_simple_interp_nearest_t> dims_;

  void rebuild() {
    std::vector<int> npts;
    std::vector<double> u, f1;
    for (auto const &d : dims_) {
      npts.push_back((int)d.get_times_u_pts().size());
      u.insert(u.end(), d.get_times_u_pts().begin(), d.get_times_u_pts().end());
      f1.insert(f1.end(), d.get_f1_pts().begin(), d.get_f1_pts().end());
    }
    table_ = detail::make_table(npts, u, f1);
    desc_ = kb_warper{KB_WARPER_TABLE, 0, u[(size_t)npts[0] - 1], 0.0, table_.get()};
  }

 public:
  warper_product_1d_interp_nearest_t() = default;
  // an already built table with one table per coordinate (make_warper_from_proj)
  explicit warper_product_1d_interp_nearest_t(std::shared_ptr<kb_warper_table> t) {
    table_ = std::move(t);
    desc_ = kb_warper{KB_WARPER_TABLE, 0, 1.0, 0.0, table_.get()};
  }
  void reserve(size_t n) { dims_.reserve(n); }
  int size() const { return (dims_.empty() && table_) ? detail::table_dims(table_.get()) : (int)dims_.size(); }
  void emplace_back(warper_product_1d_simple_interp_nearest_t const &w) {
    dims_.push_back(w);
    rebuild();
  }
  warper_product_1d_simple_interp_nearest_t get_1d_warper(int axis) const {
    if (axis < 0 || axis >= size()) throw std::runtime_error("out of range axis");
    if (dims_.empty()) { // built by make_warper_from_proj: read its points back
      std::vector<int> npts((size_t)size());
      keldy_b200::check(kb_warper_table_info(table_.get(), nullptr, nullptr, npts.data()));
      std::vector<double> u((size_t)npts[(size_t)axis]), f1(u.size());
      keldy_b200::check(kb_warper_table_points(table_.get(), axis, u.data(), f1.data()));
      return warper_product_1d_simple_interp_nearest_t(u, f1);
    }
    return dims_[(size_t)axis];
  }
};

namespace detail {
// Sobol points 1..nr_samples of dimension order (keldy's sobol(order, 0), qrng.hpp:69-109)
// and |warped_integrand| there, on the host (the caller's function).
inline void sample_host(std::function<dcomplex(std::vector<double>)> const &warped_integrand, int order,
                        int nr_samples, std::vector<double> &li, std::vector<double> &values) {
  if (order < 1 || nr_samples < 1) throw std::runtime_error("need order >= 1 and nr_samples >= 1");
  kb_sobol *g = nullptr;
  keldy_b200::check(kb_sobol_create(keldy_b200::default_context(), order, 31, 0, 0, 0, &g));
  li.assign((size_t)nr_samples * order, 0.0);
  int st = kb_sobol_points(keldy_b200::default_context(), g, 1, nr_samples, li.data());
  kb_sobol_destroy(g);
  keldy_b200::check(st);
  values.resize((size_t)nr_samples);
  for (int p = 0; p < nr_samples; ++p)
    values[(size_t)p] = std::abs(warped_integrand(std::vector<double>(li.begin() + (long)p * order,
                                                                      li.begin() + (long)(p + 1) * order)));
}
} // namespace detail

// product_1d.hpp:110-160: one analytic product maker per coordinate.
class warper_product_1d_t : public warper_base {
  std::vector<warper_product_1d_simple_t> dims_;

 public:
  warper_product_1d_t() = default;
  void reserve(size_t n) { dims_.reserve(n); }
  int size() const { return (int)dims_.size(); }
  void emplace_back(warper_product_1d_simple_t const &w) {
    dims_.push_back(w);
    std::vector<kb_warper> d;
    for (auto const &x : dims_) d.push_back(x.desc());
    kb_warper_table *t = nullptr;
    keldy_b200::check(kb_warper_table_analytic(keldy_b200::default_context(), (int)d.size(), d.data(), &t));
    table_ = detail::own_table(t);
    desc_ = kb_warper{KB_WARPER_TABLE, 0, d[0].u_max, 0.0, table_.get()};
  }
  warper_product_1d_simple_t get_1d_warper(int axis) const {
    if (axis < 0 || axis >= size()) throw std::runtime_error("out of range axis");
    return dims_[(size_t)axis];
  }
};

// product_1d.hpp:253-266
inline warper_product_1d_t make_product_1d_inverse_cube_alternate(int order, double time, double warper_scale) {
  warper_product_1d_t result{};
  result.reserve((size_t)order);
  for (int n = 1; n <= order; ++n)
    result.emplace_back(n % 2 == 0 ? make_product_1d_simple_inverse_power(3, time, warper_scale)
                                   : make_product_1d_simple_inverse(time, warper_scale));
  return result;
}

// product_1d.hpp:268-288: the same f1 shapes, tabulated on nr_sample_points points.
inline warper_product_1d_interp_nearest_t make_product_1d_inverse_cube_alternate_interp_nearest(
    int order, double time, double warper_scale, int nr_sample_points_warper) {
  warper_product_1d_interp_nearest_t result{};
  result.reserve((size_t)order);
  auto f1 = [warper_scale](double t) -> double { return warper_scale / (warper_scale + t); };
  auto f2 = [warper_scale](double t) -> double {
    return warper_scale * warper_scale * warper_scale / ((warper_scale + t) * (warper_scale + t) * (warper_scale + t));
  };
  for (int n = 1; n <= order; ++n)
    result.emplace_back(n % 2 == 0 ? warper_product_1d_simple_interp_nearest_t(f2, time, nr_sample_points_warper)
                                   : warper_product_1d_simple_interp_nearest_t(f1, time, nr_sample_points_warper));
  return result;
}

// product_1d_simple.hpp:381-554: f1 in closed form (f1_shape.kind: KB_WARPER_EXPONENTIAL
// exp(-u/w), INVERSE w/(w+u), INVERSE_SQUARE (w/(w+u))^2, INVERSE_POWER (w/(w+u))^power,
// UNIFORM 1; f1_shape.u_max the domain), Simpson integral on nr_sample_points points and
// Steffen splines of the integral and of its inverse. keldy takes f1 as any function; the
// device needs one of these closed forms.
class warper_product_1d_simple_interp_hybrid_t : public warper_base {
  kb_warper shape_{};
  int npts_ = 0;

 public:
  warper_product_1d_simple_interp_hybrid_t(kb_warper const &f1_shape, int nr_sample_points)
     : shape_(f1_shape), npts_(nr_sample_points) {
    kb_warper_table *t = nullptr;
    keldy_b200::check(kb_warper_table_hybrid(keldy_b200::default_context(), 1, &shape_, &npts_, &t));
    table_ = detail::own_table(t);
    desc_ = kb_warper{KB_WARPER_TABLE, 0, shape_.u_max, 0.0, table_.get()};
  }
  kb_warper const &get_f1_shape() const { return shape_; }
  int get_nr_sample_points() const { return npts_; }
};

// product_1d.hpp:213-251: one hybrid warper per coordinate.
class warper_product_1d_interp_hybrid_t : public warper_base {
  std::vector<warper_product_1d_simple_interp_hybrid_t> dims_;

 public:
  warper_product_1d_interp_hybrid_t() = default;
  void reserve(size_t n) { dims_.reserve(n); }
  int size() const { return (int)dims_.size(); }
  void emplace_back(warper_product_1d_simple_interp_hybrid_t const &w) {
    dims_.push_back(w);
    std::vector<kb_warper> shapes;
    std::vector<int> npts;
    for (auto const &x : dims_) {
      shapes.push_back(x.get_f1_shape());
      npts.push_back(x.get_nr_sample_points());
    }
    kb_warper_table *t = nullptr;
    keldy_b200::check(
        kb_warper_table_hybrid(keldy_b200::default_context(), (int)shapes.size(), shapes.data(), npts.data(), &t));
    table_ = detail::own_table(t);
    desc_ = kb_warper{KB_WARPER_TABLE, 0, shapes[0].u_max, 0.0, table_.get()};
  }
  warper_product_1d_simple_interp_hybrid_t get_1d_warper(int axis) const {
    if (axis < 0 || axis >= size()) throw std::runtime_error("out of range axis");
    return dims_[(size_t)axis];
  }
};

// product_1d.hpp:290-309
inline warper_product_1d_interp_hybrid_t make_product_1d_inverse_cube_alternate_interp_hybrid(
    int order, double time, double warper_scale, int nr_sample_points_warper) {
  warper_product_1d_interp_hybrid_t result{};
  result.reserve((size_t)order);
  for (int n = 1; n <= order; ++n)
    result.emplace_back(warper_product_1d_simple_interp_hybrid_t(
        n % 2 == 0 ? kb_warper{KB_WARPER_INVERSE_POWER, 3, time, warper_scale}
                   : kb_warper{KB_WARPER_INVERSE, 0, time, warper_scale},
        nr_sample_points_warper));
  return result;
}

// The binned projection of one axis of a projection warper (binner_t<1, 0, double>):
// mean |f J| and counts per bin.
struct projection_bins {
  double xmin = 0.0, xmax = 1.0;
  std::vector<double> data;
  std::vector<uint64_t> nr_values_added;
  std::vector<double> const &get_data() const { return data; }
  std::vector<uint64_t> const &get_nr_values_added() const { return nr_values_added; }
  int get_nr_bins() const { return (int)data.size(); }
  double get_bin_size() const { return (xmax - xmin) / double(data.size()); }
  std::vector<double> get_bin_coord() const {
    std::vector<double> c(data.size());
    for (size_t i = 0; i < c.size(); ++i) c[i] = xmin + (double(i) + 0.5) * get_bin_size();
    return c;
  }
};

// projection.hpp:176-382: per axis the binned |f J| of nr_samples Sobol points, smoothed
// (width sigma, or optimised), its normalised integral and the integral's inverse.
class warper_projection_t : public warper_base {
  int order_ = 0, num_bins_ = 0;

  void adopt(kb_warper_table *t, int order, int num_bins) {
    table_ = detail::own_table(t);
    desc_ = kb_warper{KB_WARPER_TABLE, 0, 1.0, 0.0, table_.get()};
    order_ = order;
    num_bins_ = num_bins;
  }

 public:
  warper_projection_t(std::function<dcomplex(std::vector<double>)> const &warped_integrand, int order, int num_bins,
                      int nr_samples, double sigma, bool optimize_sigma = true) {
    std::vector<double> li, values;
    detail::sample_host(warped_integrand, order, nr_samples, li, values);
    kb_warper_table *t = nullptr;
    keldy_b200::check(kb_warper_projection_create(keldy_b200::default_context(), order, num_bins, nr_samples,
                                                  li.data(), values.data(), sigma, optimize_sigma, &t));
    adopt(t, order, num_bins);
  }
  // an already built projection warper (see make_projection_warper below)
  explicit warper_projection_t(kb_warper_table *t) {
    int n = detail::table_dims(t);
    std::vector<int> npts((size_t)n);
    keldy_b200::check(kb_warper_table_info(t, nullptr, nullptr, npts.data()));
    adopt(t, n, npts[0]);
  }
  std::vector<double> get_sigmas() const {
    std::vector<double> out((size_t)order_);
    for (int a = 0; a < order_; ++a)
      keldy_b200::check(kb_warper_projection_axis(table_.get(), a, &out[(size_t)a], nullptr, nullptr, nullptr));
    return out;
  }
  // fn on the uniform mesh of [0, 1] with num_bins points
  std::vector<double> get_fi(int axis) const {
    std::vector<double> fn((size_t)num_bins_);
    keldy_b200::check(kb_warper_projection_axis(table_.get(), axis, nullptr, nullptr, nullptr, fn.data()));
    return fn;
  }
  projection_bins get_xi(int axis) const {
    projection_bins b;
    const double delta = 1.0 / (num_bins_ - 1.0);
    b.xmin = -delta / 2;
    b.xmax = 1 + delta / 2;
    b.data.resize((size_t)num_bins_);
    b.nr_values_added.resize((size_t)num_bins_);
    keldy_b200::check(
        kb_warper_projection_axis(table_.get(), axis, nullptr, b.data.data(), b.nr_values_added.data(), nullptr));
    return b;
  }
};

// warpers.hpp:45-137: a chain, applied last to first by map_reverse.
class warper_train_t {
  std::vector<kb_warper> chain_;
  std::vector<std::shared_ptr<kb_warper_table>> keep_; // device tables of tabulated warpers

 public:
  warper_train_t() = default;
  void emplace_back(warper_base const &w) {
    if (chain_.size() >= KB_MAX_CHAIN) throw std::runtime_error("warper train longer than KB_MAX_CHAIN");
    if (w.desc().kind == KB_WARPER_TABLE && !w.table()) throw std::runtime_error("empty tabulated warper");
    chain_.push_back(w.desc());
    keep_.push_back(w.table());
  }
  void reserve(size_t n) { chain_.reserve(n); }
  void clear() {
    chain_.clear();
    keep_.clear();
  }
  size_t size() const { return chain_.size(); }
  std::vector<kb_warper> const &chain() const { return chain_; }

  std::pair<std::vector<double>, double> map_reverse(std::vector<double> const &li_vec, int start_domain_nr,
                                                     int end_domain_nr) const {
    if (chain_.empty()) return {li_vec, 1.0};
    return detail::apply(chain_, KB_REVERSE, start_domain_nr, end_domain_nr, li_vec);
  }
  std::pair<std::vector<double>, double> map_forward(std::vector<double> const &ui_vec, int start_domain_nr,
                                                     int end_domain_nr) const {
    if (chain_.empty()) return {ui_vec, 1.0};
    return detail::apply(chain_, KB_FORWARD, start_domain_nr, end_domain_nr, ui_vec);
  }
  std::pair<std::vector<double>, double> map_reverse(std::vector<double> const &li_vec) const {
    return map_reverse(li_vec, (int)chain_.size(), 0);
  }
  std::pair<std::vector<double>, double> map_forward(std::vector<double> const &ui_vec) const {
    return map_forward(ui_vec, 0, (int)chain_.size());
  }
  double jacobian_reverse(std::vector<double> const &li_vec) const { return map_reverse(li_vec).second; }
  double jacobian_forward(std::vector<double> const &ui_vec) const { return map_forward(ui_vec).second; }
  std::vector<double> ui_from_li(std::vector<double> const &li_vec) const { return map_reverse(li_vec).first; }
  std::vector<double> li_from_ui(std::vector<double> const &ui_vec) const { return map_forward(ui_vec).first; }
};

} // namespace warpers

namespace impurity_oneband {

// model.hpp:37-50
struct model_param_t {
  double beta = 1.0;
  double bias_V = 0.0;
  double eps_d = 0.0;
  double Gamma = 1.0;
  double alpha = 0.0;
  double half_bandwidth = 2.;
  std::string bath_type = "semicircle";
  double time_max = +100.0;
  int nr_time_points_gf = 1000;
  std::string ft_method = "fft";
};

// model.hpp:55-78
class gf_index_t {
 public:
  contour_pt_t contour{};
  spin_t spin = up;
  orbital_t orbital = 0;
  gf_index_t() = default;
  gf_index_t(time_real_t time_, int spin_, int k_idx_) : contour{time_, keldysh_idx_t(k_idx_)}, spin(spin_t(spin_)) {}
  gf_index_t(time_real_t time_, int spin_, int k_idx_, int timesplit_n_)
     : contour{time_, keldysh_idx_t(k_idx_), timesplit_n_}, spin(spin_t(spin_)) {}
  gf_index_t(time_real_t time_, int spin_, int k_idx_, int timesplit_n_, int orbital_)
     : contour{time_, keldysh_idx_t(k_idx_), timesplit_n_}, spin(spin_t(spin_)), orbital(orbital_t(orbital_)) {}
  kb_gf_index abi() const {
    return kb_gf_index{contour.time, int(spin), int(contour.k_idx), contour.timesplit_n, orbital};
  }
};

// g^<(t), g^>(t) tables on the uniform mesh [-time_max, time_max] (model.hpp:178-232).
// Copies share the device tables (immutable after construction).
class g0_model {
  std::shared_ptr<kb_model> m_;
  double time_max_ = 0.0;
  int npts_ = 0;
  double alpha_ = 0.0;

 public:
  bool make_dot_lead = false;
  model_param_t param{};

  g0_model() = default;

  // lesser/greater: npts complex values of spin up, orbital (0,0); the other blocks
  // (spin down, dot-lead orbitals) may be added with set_table.
  static g0_model from_tables(double time_max, std::vector<dcomplex> const &lesser,
                              std::vector<dcomplex> const &greater, double alpha = 0.0) {
    if (lesser.size() != greater.size()) throw std::runtime_error("lesser and greater tables differ in length");
    g0_model g;
    kb_model *m = nullptr;
    keldy_b200::check(kb_model_create(keldy_b200::default_context(), (int)lesser.size(), time_max, alpha, &m));
    g.m_ = std::shared_ptr<kb_model>(m, kb_model_destroy);
    g.time_max_ = time_max;
    g.npts_ = (int)lesser.size();
    g.alpha_ = alpha;
    g.param.time_max = time_max;
    g.param.nr_time_points_gf = g.npts_;
    g.param.alpha = alpha;
    g.set_table(0, 0, 0, lesser, greater);
    return g;
  }

  // A model with no tables yet (npts points on [-time_max, time_max]); fill its blocks with
  // set_table or set_fourier.
  static g0_model empty(double time_max, int npts, double alpha = 0.0) {
    g0_model g;
    kb_model *m = nullptr;
    keldy_b200::check(kb_model_create(keldy_b200::default_context(), npts, time_max, alpha, &m));
    g.m_ = std::shared_ptr<kb_model>(m, kb_model_destroy);
    g.time_max_ = time_max;
    g.npts_ = npts;
    g.alpha_ = alpha;
    g.param.time_max = time_max;
    g.param.nr_time_points_gf = npts;
    g.param.alpha = alpha;
    return g;
  }

  // Block (o1, o2) built on the GPU from quadrature nodes w and weights cl, cg
  // (kb_model_set_fourier: g(t) = sum_k c_k e^{-i w_k t}; flags KB_FT_SYMMETRIC, KB_FT_MIRROR).
  void set_fourier(int o1, int o2, std::vector<double> const &w, std::vector<dcomplex> const &cl,
                   std::vector<dcomplex> const &cg, int flags) {
    if (cl.size() != w.size() || cg.size() != w.size()) throw std::runtime_error("one weight per node");
    keldy_b200::check(kb_model_set_fourier(m_.get(), o1, o2, (int)w.size(), w.data(),
                                           reinterpret_cast<const double *>(cl.data()),
                                           reinterpret_cast<const double *>(cg.data()), flags));
  }

  // keldy's "fft" tables of block (o1, o2) from values on the adjoint frequency mesh
  // (kb_model_set_fft; flags KB_FT_MIRROR)
  void set_fft(int o1, int o2, std::vector<dcomplex> const &gl, std::vector<dcomplex> const &gg, int flags) {
    if (gl.size() != gg.size()) throw std::runtime_error("one lesser and one greater value per frequency");
    keldy_b200::check(kb_model_set_fft(m_.get(), o1, o2, reinterpret_cast<const double *>(gl.data()),
                                       reinterpret_cast<const double *>(gg.data()), flags));
  }

  // block (o1, o2) of a bath with a rational hybridisation in closed form
  // (kb_model_set_rational): per lead its mu and the poles and residues of its rational part
  void set_rational(int o1, int o2, std::vector<double> const &mu, std::vector<std::vector<dcomplex>> const &poles,
                    std::vector<std::vector<dcomplex>> const &residues, double beta, int flags) {
    if (poles.size() != mu.size() || residues.size() != mu.size())
      throw std::runtime_error("one pole list and one residue list per term");
    std::vector<int> n;
    std::vector<dcomplex> z, r;
    for (size_t l = 0; l < mu.size(); ++l) {
      if (poles[l].size() != residues[l].size()) throw std::runtime_error("one residue per pole");
      n.push_back((int)poles[l].size());
      z.insert(z.end(), poles[l].begin(), poles[l].end());
      r.insert(r.end(), residues[l].begin(), residues[l].end());
    }
    keldy_b200::check(kb_model_set_rational(m_.get(), o1, o2, (int)mu.size(), mu.data(), n.data(),
                                            reinterpret_cast<const double *>(z.data()),
                                            reinterpret_cast<const double *>(r.data()), beta, flags));
  }

  // KB_INTERP_LINEAR (keldy's) or KB_INTERP_CUBIC (an extension) between mesh points
  void set_interpolation(int order) { keldy_b200::check(kb_model_set_interpolation(m_.get(), order)); }

  // keldy's public g0_lesser / g0_greater data of one block (model.hpp:184-188)
  std::pair<std::vector<dcomplex>, std::vector<dcomplex>> get_table(int spin, int o1, int o2) const {
    std::vector<dcomplex> l((size_t)npts_), g((size_t)npts_);
    keldy_b200::check(kb_model_get_table(m_.get(), spin, o1, o2, reinterpret_cast<double *>(l.data()),
                                         reinterpret_cast<double *>(g.data())));
    return {l, g};
  }

  void set_table(int spin, int o1, int o2, std::vector<dcomplex> const &lesser, std::vector<dcomplex> const &greater) {
    if ((int)lesser.size() != npts_ || (int)greater.size() != npts_)
      throw std::runtime_error("table length differs from the model's mesh");
    keldy_b200::check(kb_model_set_table(m_.get(), spin, o1, o2, reinterpret_cast<const double *>(lesser.data()),
                                         reinterpret_cast<const double *>(greater.data())));
  }

  double time_max() const { return time_max_; }
  int npts() const { return npts_; }
  double alpha() const { return alpha_; }
  const kb_model *handle() const { return m_.get(); }
};

// model.hpp:238-268
struct g0_keldysh_contour_t {
  g0_model model;
  g0_keldysh_contour_t(g0_model model_) : model(std::move(model_)) {}

  dcomplex operator()(gf_index_t const &a, gf_index_t const &b, bool internal_point = true) const {
    kb_gf_index x = a.abi(), y = b.abi();
    int internal = internal_point ? 1 : 0;
    double out[2];
    keldy_b200::check(kb_g0_eval(keldy_b200::default_context(), model.handle(), &x, &y, &internal, 1, out));
    return {out[0], out[1]};
  }

  double get_time_max() const { return model.time_max(); }
};

// wick_direct.hpp:34-65
class integrand_g_direct {
  g0_keldysh_contour_t g0;
  gf_index_t external_A;
  gf_index_t external_B;
  double cutoff;
  int algo_ = KB_ALGO_AUTO;

  std::pair<dcomplex, int> eval(std::vector<double> const &times, bool keep, bool no_det) const {
    kb_integrand f = abi();
    double out[2];
    int dom = 0;
    int n = (int)times.size();
    if (no_det)
      keldy_b200::check(kb_integrand_eval_no_det(keldy_b200::default_context(), g0.model.handle(), &f, n, 1,
                                                 times.data(), keep, out, &dom));
    else
      keldy_b200::check(kb_integrand_eval(keldy_b200::default_context(), g0.model.handle(), &f, n, 1, times.data(),
                                          keep, algo_, out, &dom, nullptr));
    return {dcomplex(out[0], out[1]), dom};
  }

 public:
  using result_t = dcomplex;

  integrand_g_direct(g0_keldysh_contour_t g0_, gf_index_t external_A_, gf_index_t external_B_, double cutoff_ = 0.)
     : g0(std::move(g0_)), external_A(external_A_), external_B(external_B_), cutoff(cutoff_) {
    if (external_A.contour.time < 0. || external_B.contour.time < 0.)
      throw std::runtime_error("An external point has negative time.");
    double const t_max = g0.get_time_max();
    if (external_A.contour.time > t_max || external_B.contour.time > t_max)
      throw std::runtime_error("An external point is out of g0 time window.");
  }

  // One point per call, as keldy's: each call is a device round trip (tens of
  // microseconds). A loop over many points should call eval_many instead.
  std::pair<result_t, int> operator()(std::vector<double> const &times, bool const keep_u_hypercube = true) const {
    return eval(times, keep_u_hypercube, false);
  }
  // count points of `order` vertex times each (row-major in `times`), one device call:
  // values[p], in_domain[p] (an addition to keldy's interface).
  void eval_many(int order, int64_t count, double const *times, std::vector<result_t> &values,
                 std::vector<int> &in_domain, bool const keep_u_hypercube = true) const {
    kb_integrand f = abi();
    std::vector<double> out((size_t)(2 * count));
    in_domain.assign((size_t)count, 0);
    keldy_b200::check(kb_integrand_eval(keldy_b200::default_context(), g0.model.handle(), &f, order, count, times,
                                        keep_u_hypercube, algo_, out.data(), in_domain.data(), nullptr));
    values.resize((size_t)count);
    for (int64_t p = 0; p < count; ++p) values[(size_t)p] = dcomplex(out[(size_t)(2 * p)], out[(size_t)(2 * p + 1)]);
  }
  std::pair<result_t, int> eval_no_det(std::vector<double> const &times, bool const keep_u_hypercube = true) const {
    return eval(times, keep_u_hypercube, true);
  }

  // algorithm of the device integrand: KB_ALGO_AUTO (default), KB_ALGO_TREE, KB_ALGO_DIRECT
  void set_algorithm(int algo) { algo_ = algo; }
  int algorithm() const { return algo_; }
  kb_integrand abi() const { return kb_integrand{external_A.abi(), external_B.abi(), cutoff}; }
  g0_keldysh_contour_t const &get_g0() const { return g0; }
};

// integrator.hpp:42-136 for the integrand_g_direct observables; runs on the device.
class integrator_g_direct {
 protected:
  int dimension = 1;
  dcomplex result{0.0};
  uint64_t n_points = 0;
  uint64_t n_integrand_evals_in_domain = 0;
  integrand_g_direct integrand;
  sobol rng_;

 public:
  warpers::warper_train_t warper{};

  integrator_g_direct(integrand_g_direct integrand_, int dimension_)
     : dimension(dimension_), integrand(std::move(integrand_)), rng_(dimension_ > 0 ? dimension_ : 1, 0) {
    if (dimension <= 0) throw std::runtime_error("Dimension of the integration space must be > 0.");
  }

  // One point per call, as keldy's (a device round trip); kb_evaluate_warped takes many.
  std::pair<dcomplex, double> evaluate_warped_integrand(std::vector<double> const &li_vec, int start_domain_nr,
                                                        bool keep_u_hypercube = true) const {
    kb_integrand f = integrand.abi();
    double out[2], jac = 1.0;
    int dom = 0;
    auto const &chain = warper.chain();
    keldy_b200::check(kb_evaluate_warped(keldy_b200::default_context(), integrand.get_g0().model.handle(), &f,
                                         chain.data(), (int)chain.size(), start_domain_nr, (int)li_vec.size(), 1,
                                         li_vec.data(), keep_u_hypercube, integrand.algorithm(), out, &jac, &dom));
    return {dcomplex(out[0], out[1]), double(dom)};
  }
  std::pair<dcomplex, double> evaluate_warped_integrand(std::vector<double> const &li_vec) const {
    return evaluate_warped_integrand(li_vec, (int)warper.size(), true);
  }

  // nr_steps Sobol points through the warper train and the integrand, summed (integrator.hpp:81-95)
  void run(int nr_steps) {
    if (nr_steps <= 0) return;
    if ((uint64_t)rng_.state() + (uint64_t)nr_steps > (1ull << 31))
      throw std::runtime_error("More sample points requested then generator can hold.");
    auto const &chain = warper.chain();
    kb_work w{integrand.get_g0().model.handle(), rng_.handle(), chain.data(), (int)chain.size(), integrand.abi(),
              dimension, rng_.state() + 1, nr_steps};
    kb_accum acc{};
    keldy_b200::check(kb_integrate(keldy_b200::default_context(), &w, 1, integrand.algorithm(), &acc));
    rng_.discard(nr_steps);
    result += dcomplex(acc.sum_re, acc.sum_im);
    n_points += acc.n_points;
    n_integrand_evals_in_domain += acc.n_in_domain;
  }

  // integrator.hpp:97-112 ("sobol_unshifted", "sobol"; the boost generators have no device form)
  void reset_rng(std::string rng_name, int rng_state_seed, bool do_shift = false, bool do_scramble = false,
                 int rng_seed_shift = 0) {
    if (rng_name == "sobol_unshifted")
      rng_ = sobol(dimension, rng_state_seed);
    else if (rng_name == "sobol")
      rng_ = sobol(dimension, rng_state_seed, do_shift, do_scramble, rng_seed_shift);
    else if (rng_name == "mt19937_64" || rng_name == "ranlux48" || rng_name == "taus88")
      throw std::runtime_error("rng '" + rng_name + "' has no device form; use sobol_unshifted or sobol");
    else
      throw std::runtime_error("No other rng available.");
  }

  dcomplex reduce_result() const { return result * (1.0 / double(reduce_nr_points_run())); }
  uint64_t reduce_nr_points_run() const { return n_points; }
  uint64_t reduce_nr_points_in_domain() const { return n_integrand_evals_in_domain; }
  dcomplex raw_result() const { return result; }
  integrand_g_direct get_integrand() const { return integrand; }
  warpers::warper_train_t get_warper() const { return warper; }
  sobol const &get_rng() const { return rng_; }
};

// compute_obs.hpp:51-64: charge G^<_{up,up}(t, t)
class compute_charge_Q_direct : public integrator_g_direct {
 public:
  compute_charge_Q_direct(g0_model model, double time, int order, double cutoff_integrand)
     : integrator_g_direct(integrand_g_direct{g0_keldysh_contour_t{std::move(model)}, gf_index_t{time, up, forward},
                                              gf_index_t{time, up, backward}, cutoff_integrand},
                           order) {}
};

// compute_obs.hpp:66-80: current, -2e/hbar gamma Re G^<_{lead,dot}(t, t); needs the
// model's dot-lead blocks (set_table(spin, 1, 0, ...) and (spin, 0, 1, ...)).
class compute_current_J_direct : public integrator_g_direct {
 public:
  compute_current_J_direct(g0_model model, double time, int order, double cutoff_integrand)
     : integrator_g_direct(integrand_g_direct{g0_keldysh_contour_t{std::move(model)},
                                              gf_index_t{time, up, forward, 0, 1},
                                              gf_index_t{time, up, backward, 0, 0}, cutoff_integrand},
                           order) {}
};

// keldy::binner::binner_t<1> (binner.hpp:163-300): a continuous axis [xmin, xmax] in
// nr_bins bins; per bin the sum of the values added and their number; values outside the
// axis counted as dropped.
class binner_1d {
  double xmin_ = 0.0, xmax_ = 1.0, bin_size_ = 1.0;
  std::vector<dcomplex> data_;
  std::vector<long> nr_values_added_;

 public:
  long nr_values_dropped = 0;

  binner_1d(double xmin, double xmax, long nr_bins) : xmin_(xmin), xmax_(xmax) {
    if (xmin >= xmax)
      throw std::runtime_error("Boundaries of binning range are in wrong order (" + std::to_string(xmin) +
                               " >= " + std::to_string(xmax) + ")");
    if (nr_bins < 1 || nr_bins > 4096) throw std::runtime_error("the number of time bins must be in [1, 4096]");
    bin_size_ = (xmax - xmin) / double(nr_bins);
    data_.assign((size_t)nr_bins, dcomplex(0.0));
    nr_values_added_.assign((size_t)nr_bins, 0);
  }
  std::vector<dcomplex> const &get_data() const { return data_; }
  std::vector<long> const &get_nr_values_added() const { return nr_values_added_; }
  long get_nr_values_dropped() const { return nr_values_dropped; }
  int get_nr_bins() const { return (int)data_.size(); }
  double get_bin_size() const { return bin_size_; }
  double get_xmin() const { return xmin_; }
  double get_xmax() const { return xmax_; }
  std::vector<double> get_bin_coord() const {
    std::vector<double> c(data_.size());
    for (size_t i = 0; i < c.size(); ++i) c[i] = xmin_ + (double(i) + 0.5) * bin_size_;
    return c;
  }
  binner_1d &operator*=(dcomplex s) {
    for (auto &v : data_) v *= s;
    return *this;
  }
  // adds kb_integrate_binned's outputs of one work item
  void add(const double *sums, const uint64_t *counts, uint64_t dropped) {
    for (size_t b = 0; b < data_.size(); ++b) {
      data_[b] += dcomplex(sums[2 * b], sums[2 * b + 1]);
      nr_values_added_[b] += (long)counts[b];
    }
    nr_values_dropped += (long)dropped;
  }
};

// integrator<binner_t<1>, integrand_g_direct_time> (wick_direct_time.cpp:42-163,
// integrator.hpp:81-131): the direct integrand, each point's f*J binned by its earliest
// vertex time. evaluate_warped_integrand returns the unbinned value.
class integrator_g_direct_time : public integrator_g_direct {
 protected:
  binner_1d bins_;

 public:
  integrator_g_direct_time(binner_1d bins, integrand_g_direct integrand_, int dimension_)
     : integrator_g_direct(std::move(integrand_), dimension_), bins_(std::move(bins)) {}

  void run(int nr_steps) {
    if (nr_steps <= 0) return;
    if ((uint64_t)rng_.state() + (uint64_t)nr_steps > (1ull << 31))
      throw std::runtime_error("More sample points requested then generator can hold.");
    auto const &chain = warper.chain();
    kb_work w{integrand.get_g0().model.handle(), rng_.handle(), chain.data(), (int)chain.size(), integrand.abi(),
              dimension, rng_.state() + 1, nr_steps};
    kb_time_bins tb{bins_.get_nr_bins(), bins_.get_xmin(), bins_.get_xmax()};
    std::vector<double> sums(2 * (size_t)tb.nbins, 0.0);
    std::vector<uint64_t> counts((size_t)tb.nbins, 0);
    uint64_t dropped = 0;
    kb_accum acc{};
    keldy_b200::check(kb_integrate_binned(keldy_b200::default_context(), &w, 1, integrand.algorithm(), &tb, &acc,
                                          sums.data(), counts.data(), &dropped));
    rng_.discard(nr_steps);
    bins_.add(sums.data(), counts.data(), dropped);
    result += dcomplex(acc.sum_re, acc.sum_im);
    n_points += acc.n_points;
    n_integrand_evals_in_domain += acc.n_in_domain;
  }

  // result / n_points, as integrator::reduce_result (integrator.hpp:123-127)
  binner_1d reduce_result() const {
    binner_1d r = bins_;
    r *= dcomplex(1.0 / double(reduce_nr_points_run()));
    return r;
  }
};

// keldy::binner::binner_t<1, 1> of the kernel method: [xmin, xmax] in nr_bins time bins x
// the Keldysh index (forward, backward).
class binner_2d {
  double xmin_ = 0.0, xmax_ = 1.0, bin_size_ = 1.0;
  std::vector<dcomplex> data_; // [bin][k]
  std::vector<long> nr_values_added_;

 public:
  long nr_values_dropped = 0;
  binner_2d(double xmin, double xmax, long nr_bins) : xmin_(xmin), xmax_(xmax) {
    if (xmin >= xmax)
      throw std::runtime_error("Boundaries of binning range are in wrong order (" + std::to_string(xmin) +
                               " >= " + std::to_string(xmax) + ")");
    if (nr_bins < 1 || nr_bins > 4096) throw std::runtime_error("the number of time bins must be in [1, 4096]");
    bin_size_ = (xmax - xmin) / double(nr_bins);
    data_.assign(2 * (size_t)nr_bins, dcomplex(0.0));
    nr_values_added_.assign(2 * (size_t)nr_bins, 0);
  }
  std::vector<dcomplex> const &get_data_flat() const { return data_; }
  std::vector<long> const &get_nr_values_added_flat() const { return nr_values_added_; }
  long get_nr_values_dropped() const { return nr_values_dropped; }
  int get_nr_bins() const { return (int)(data_.size() / 2); }
  double get_bin_size() const { return bin_size_; }
  double get_xmin() const { return xmin_; }
  double get_xmax() const { return xmax_; }
  std::vector<double> get_bin_coord() const {
    std::vector<double> c(data_.size() / 2);
    for (size_t i = 0; i < c.size(); ++i) c[i] = xmin_ + (double(i) + 0.5) * bin_size_;
    return c;
  }
  binner_2d &operator*=(dcomplex s) {
    for (auto &v : data_) v *= s;
    return *this;
  }
  void add(const double *sums, const uint64_t *counts, uint64_t dropped) {
    for (size_t b = 0; b < data_.size(); ++b) {
      data_[b] += dcomplex(sums[2 * b], sums[2 * b + 1]);
      nr_values_added_[b] += (long)counts[b];
    }
    nr_values_dropped += (long)dropped;
  }
};

// integrand_g_kernel (wick_kernel.cpp:42-138): fixed point X; operator() returns, per
// vertex i and Keldysh index k, the sum of the terms keldy accumulates at (u_i, k).
class integrand_g_kernel {
  g0_keldysh_contour_t g0_;
  gf_index_t X_;

 public:
  integrand_g_kernel(g0_keldysh_contour_t g0, gf_index_t X) : g0_(std::move(g0)), X_(X) {}
  std::pair<std::vector<std::array<dcomplex, 2>>, int> operator()(std::vector<double> const &times,
                                                                    bool keep_u_hypercube = true) const {
    const int n = (int)times.size();
    std::vector<double> out(4 * (size_t)n);
    int dom = 0;
    kb_gf_index x = X_.abi();
    keldy_b200::check(kb_integrand_kernel_eval(keldy_b200::default_context(), g0_.model.handle(), &x, n, 1,
                                               times.data(), keep_u_hypercube, out.data(), &dom));
    std::vector<std::array<dcomplex, 2>> r((size_t)n);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 2; ++k) r[(size_t)i][(size_t)k] = dcomplex(out[4 * i + 2 * k], out[4 * i + 2 * k + 1]);
    return {r, dom};
  }
  g0_keldysh_contour_t const &get_g0() const { return g0_; }
  gf_index_t const &get_X() const { return X_; }
};

// integrator<binner_t<1, 1>, integrand_g_kernel> + compute_gf_kernel (compute_obs.hpp:105-117):
// G(t) by the kernel method, binned over [0, t] x Keldysh index.
class compute_gf_kernel {
  int dimension = 1;
  binner_2d bins_;
  uint64_t n_points = 0;
  uint64_t n_integrand_evals_in_domain = 0;
  integrand_g_kernel integrand;
  sobol rng_;

 public:
  warpers::warper_train_t warper{};

  compute_gf_kernel(g0_model model, double time, int order, int nr_bins = 100)
     : dimension(order), bins_(0.0, time, nr_bins),
       integrand(g0_keldysh_contour_t{std::move(model)}, gf_index_t{time, up, forward}),
       rng_(order > 0 ? order : 1, 0) {
    if (dimension <= 0) throw std::runtime_error("Dimension of the integration space must be > 0.");
  }

  void run(int nr_steps) {
    if (nr_steps <= 0) return;
    if ((uint64_t)rng_.state() + (uint64_t)nr_steps > (1ull << 31))
      throw std::runtime_error("More sample points requested then generator can hold.");
    auto const &chain = warper.chain();
    kb_gf_index x = integrand.get_X().abi();
    kb_work w{integrand.get_g0().model.handle(), rng_.handle(), chain.data(), (int)chain.size(),
              kb_integrand{x, x, 0.0}, dimension, rng_.state() + 1, nr_steps};
    kb_time_bins tb{bins_.get_nr_bins(), bins_.get_xmin(), bins_.get_xmax()};
    std::vector<double> sums(4 * (size_t)tb.nbins, 0.0);
    std::vector<uint64_t> counts(2 * (size_t)tb.nbins, 0);
    uint64_t dropped = 0;
    kb_accum acc{};
    keldy_b200::check(kb_integrate_kernel(keldy_b200::default_context(), &w, 1, &tb, &acc, sums.data(),
                                          counts.data(), &dropped));
    rng_.discard(nr_steps);
    bins_.add(sums.data(), counts.data(), dropped);
    n_points += acc.n_points;
    n_integrand_evals_in_domain += acc.n_in_domain;
  }

  void reset_rng(std::string rng_name, int rng_state_seed, bool do_shift = false, bool do_scramble = false,
                 int rng_seed_shift = 0) {
    if (rng_name == "sobol_unshifted")
      rng_ = sobol(dimension, rng_state_seed);
    else if (rng_name == "sobol")
      rng_ = sobol(dimension, rng_state_seed, do_shift, do_scramble, rng_seed_shift);
    else
      throw std::runtime_error("rng '" + rng_name + "' has no device form; use sobol_unshifted or sobol");
  }

  binner_2d reduce_result() const {
    binner_2d r = bins_;
    r *= dcomplex(1.0 / double(n_points));
    return r;
  }
  uint64_t reduce_nr_points_run() const { return n_points; }
  uint64_t reduce_nr_points_in_domain() const { return n_integrand_evals_in_domain; }
  integrand_g_kernel get_integrand() const { return integrand; }
  warpers::warper_train_t get_warper() const { return warper; }
};

// integrand_g_kernel_single_omega (wick_kernel_single_omega.cpp:42-140): the kernel
// method's terms of a point weighted by e^{i omega t} of their vertex's time and summed.
class integrand_g_kernel_single_omega {
  integrand_g_kernel kernel_;
  double omega_;

 public:
  integrand_g_kernel_single_omega(g0_keldysh_contour_t g0, gf_index_t X, double omega)
     : kernel_(std::move(g0), X), omega_(omega) {}
  std::pair<dcomplex, int> operator()(std::vector<double> const &times, bool keep_u_hypercube = true) const {
    auto [terms, dom] = kernel_(times, keep_u_hypercube);
    if (!dom) return {dcomplex(0.0), 0};
    dcomplex r(0.0);
    for (size_t i = 0; i < times.size(); ++i)
      r += (terms[i][0] + terms[i][1]) * std::exp(dcomplex(0.0, omega_ * times[i]));
    return {r, 1};
  }
  g0_keldysh_contour_t const &get_g0() const { return kernel_.get_g0(); }
  gf_index_t const &get_X() const { return kernel_.get_X(); }
  double get_omega() const { return omega_; }
};

// integrator<dcomplex, integrand_g_kernel_single_omega> + compute_gf_kernel_single_omega
// (compute_obs.hpp:119-133): the kernel method's G at one frequency, X = (time, up, forward).
class compute_gf_kernel_single_omega {
  int dimension = 1;
  dcomplex result{0.0};
  uint64_t n_points = 0;
  uint64_t n_integrand_evals_in_domain = 0;
  integrand_g_kernel_single_omega integrand;
  sobol rng_;

 public:
  warpers::warper_train_t warper{};

  compute_gf_kernel_single_omega(g0_model model, double time, double omega, int order)
     : dimension(order), integrand(g0_keldysh_contour_t{std::move(model)}, gf_index_t{time, up, forward}, omega),
       rng_(order > 0 ? order : 1, 0) {
    if (dimension <= 0) throw std::runtime_error("Dimension of the integration space must be > 0.");
  }

  void run(int nr_steps) {
    if (nr_steps <= 0) return;
    if ((uint64_t)rng_.state() + (uint64_t)nr_steps > (1ull << 31))
      throw std::runtime_error("More sample points requested then generator can hold.");
    auto const &chain = warper.chain();
    kb_gf_index x = integrand.get_X().abi();
    kb_work w{integrand.get_g0().model.handle(), rng_.handle(), chain.data(), (int)chain.size(),
              kb_integrand{x, x, 0.0}, dimension, rng_.state() + 1, nr_steps};
    kb_accum acc{};
    keldy_b200::check(kb_integrate_kernel_single_omega(keldy_b200::default_context(), &w, 1, integrand.get_omega(),
                                                       &acc));
    rng_.discard(nr_steps);
    result += dcomplex(acc.sum_re, acc.sum_im);
    n_points += acc.n_points;
    n_integrand_evals_in_domain += acc.n_in_domain;
  }

  void reset_rng(std::string rng_name, int rng_state_seed, bool do_shift = false, bool do_scramble = false,
                 int rng_seed_shift = 0) {
    if (rng_name == "sobol_unshifted")
      rng_ = sobol(dimension, rng_state_seed);
    else if (rng_name == "sobol")
      rng_ = sobol(dimension, rng_state_seed, do_shift, do_scramble, rng_seed_shift);
    else
      throw std::runtime_error("rng '" + rng_name + "' has no device form; use sobol_unshifted or sobol");
  }

  dcomplex reduce_result() const { return result / double(n_points); }
  uint64_t reduce_nr_points_run() const { return n_points; }
  uint64_t reduce_nr_points_in_domain() const { return n_integrand_evals_in_domain; }
  integrand_g_kernel_single_omega get_integrand() const { return integrand; }
  warpers::warper_train_t get_warper() const { return warper; }
};

// compute_obs.hpp:85-101: charge G^<_{up,up}(t, t) binned over [0, t] in nr_time_slices.
class compute_charge_Q_direct_time : public integrator_g_direct_time {
 public:
  compute_charge_Q_direct_time(g0_model model, double time, int order, int nr_time_slices, double cutoff_integrand)
     : integrator_g_direct_time(binner_1d(0.0, time, nr_time_slices),
                                integrand_g_direct{g0_keldysh_contour_t{std::move(model)}, gf_index_t{time, up, forward},
                                                   gf_index_t{time, up, backward}, cutoff_integrand},
                                order) {}
};

} // namespace impurity_oneband

namespace warpers {
// make_warper_from_proj (make_warper_from_proj.hpp:118-153) for any warped integrand (the
// caller's function, evaluated on the host at Sobol points 1..nr_samples).
inline warper_product_1d_interp_nearest_t make_warper_from_proj(
    std::function<dcomplex(std::vector<double>)> const &warped_integrand, int order, int num_bins, int nr_samples,
    double sigma) {
  std::vector<double> li, values;
  detail::sample_host(warped_integrand, order, nr_samples, li, values);
  kb_warper_table *t = nullptr;
  keldy_b200::check(kb_warper_table_from_samples(keldy_b200::default_context(), order, num_bins, nr_samples,
                                                 li.data(), values.data(), sigma, &t));
  return warper_product_1d_interp_nearest_t(detail::own_table(t));
}

// warper_projection_t for the integrand of `computer` through its current warper train,
// sampled on the GPU (the same tables as warper_projection_t(warped_integrand, ...) with
// warped_integrand = computer.evaluate_warped_integrand(l, train size, keep_u_hypercube)).
inline warper_projection_t make_projection_warper(impurity_oneband::integrator_g_direct const &computer, int order,
                                                  int num_bins, int nr_samples, double sigma,
                                                  bool optimize_sigma = true, bool keep_u_hypercube = true) {
  auto const train = computer.get_warper();
  auto const &chain = train.chain();
  kb_integrand f = computer.get_integrand().abi();
  kb_warper_table *t = nullptr;
  keldy_b200::check(kb_warper_projection_from_integrand(
      keldy_b200::default_context(), computer.get_integrand().get_g0().model.handle(), &f, chain.data(),
      (int)chain.size(), order, num_bins, nr_samples, sigma, optimize_sigma, keep_u_hypercube, &t));
  return warper_projection_t(t);
}

// make_warper_from_proj (make_warper_from_proj.hpp:118-153) for the integrand of
// `computer` through its current warper train: one tabulated warper per axis, built from
// the smoothed projections of |f J| on nr_samples Sobol points; append it to the train.
inline warper_product_1d_interp_nearest_t make_warper_from_proj(impurity_oneband::integrator_g_direct const &computer,
                                                                int order, int num_bins, int nr_samples,
                                                                double sigma, bool keep_u_hypercube = true) {
  auto const train = computer.get_warper(); // a copy: its chain must outlive the call below
  auto const &chain = train.chain();
  kb_integrand f = computer.get_integrand().abi();
  kb_warper_table *t = nullptr;
  keldy_b200::check(kb_warper_table_from_projection(keldy_b200::default_context(),
                                                    computer.get_integrand().get_g0().model.handle(), &f,
                                                    chain.data(), (int)chain.size(), order, num_bins, nr_samples,
                                                    sigma, keep_u_hypercube, &t));
  return warper_product_1d_interp_nearest_t(detail::own_table(t));
}
} // namespace warpers
} // namespace keldy
