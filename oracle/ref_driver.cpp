// C entry points around keldy's own hot-path sources, compiled by oracle/ref_build.sh
// into oracle/_ref/ (never committed). TEST INFRASTRUCTURE ONLY: tests/, smoke() and
// bench.py's reference arm load it as the checker or as the timed CPU baseline.
//
// Compiled from keldy's sources as they are: qrng_details/digitalseq_b2g.hpp,
// warpers/{identity,plasma_uv,product_1d_simple}.hpp, common.cpp and
// impurity_oneband/wick_direct.cpp (against the stand-ins in oracle/ref_stubs/).
// Restated here because their headers pull boost/MPI/projection code: the
// keldy::sobol wrapper (qrng.hpp:49-114), the warper_train_t chain loop
// (warpers.hpp:72-101) and the integrator loop (integrator.hpp:68-95, 123-131).
#include <keldy/common.hpp>
#include <keldy/impurity_oneband/wick_direct.hpp>
#include <keldy/qrng_details/digitalseq_b2g.hpp>
#include <keldy/warpers/identity.hpp>
#include <keldy/warpers/plasma_uv.hpp>
#include <keldy/warpers/product_1d_simple.hpp>

#include <omp.h>

#include <cstdint>
#include <cstring>
#include <random>
#include <variant>
#include <vector>

// Stand-in for the constructor in model.cpp (not compiled here: it needs FFTW, QUADPACK
// and boost). The oracle hands g0 tables to g0_model directly, so only the parameters
// (alpha, time window) matter; the bath functions are never evaluated.
keldy::impurity_oneband::g0_model_omega::g0_model_omega(model_param_t const &parameters) : param_(parameters) {}

using namespace keldy;
using namespace keldy::impurity_oneband;
using namespace keldy::warpers;

namespace {

thread_local std::string g_err;

// keldy::sobol (qrng.hpp:69-109): the generator state after construction with seed.
qmc::digitalseq_b2g<double, std::uint32_t> make_sobol(int dim, int seed, bool do_shift, bool do_scramble,
                                                      int seed_shift, int log_max_points) {
  std::vector<std::uint32_t> Cs(static_cast<size_t>(dim) * log_max_points);
  qmc::JK2008_sobol_matrices(Cs.begin(), dim, log_max_points);
  auto t = qmc::bit_depth(Cs.begin(), Cs.end());
  unsigned t2 = t;
  std::vector<std::uint32_t> shifts(dim);
  std::vector<std::uint32_t> scrambled = Cs;
  std::vector<std::uint32_t> M(static_cast<size_t>(dim) * t);
  if (do_shift || do_scramble) {
    std::mt19937_64 rng(seed_shift);
    std::generate_n(shifts.begin(), dim, rng);
    if (!do_shift) std::fill_n(shifts.begin(), dim, 0);
    if (do_scramble) {
      qmc::generate_random_linear_scramble(dim, t2, t, M.begin(), rng);
      qmc::scramble(dim, t, log_max_points, M.begin(), Cs.begin(), scrambled.begin());
    }
  }
  auto g = qmc::digitalseq_b2g<double, std::uint32_t>(dim, log_max_points, scrambled.begin(), shifts.begin());
  g.set_state(std::uint32_t(seed));
  return g;
}

struct ref_warper_desc {
  int kind;
  int power;
  double u_max;
  double w;
};

using warper_v = std::variant<warper_identity_t, warper_plasma_uv_t, warper_product_1d_simple_t>;

warper_v make_warper(ref_warper_desc const &d) {
  switch (d.kind) {
  case 0: return warper_identity_t{};
  case 1: return warper_plasma_uv_t{d.u_max};
  case 2: return make_product_1d_simple_exponential(d.u_max, d.w);
  case 3: return make_product_1d_simple_inverse(d.u_max, d.w);
  case 4: return make_product_1d_simple_inverse_square(d.u_max, d.w);
  case 5: return make_product_1d_simple_inverse_power(d.power, d.u_max, d.w);
  case 6: {
    double t = d.u_max;
    return warper_product_1d_simple_t([t](double) -> double { return 1. / t; }, [t](double u) -> double { return u / t; },
                                      [t](double l) -> double { return t * l; }, t);
  }
  default: TRIQS_RUNTIME_ERROR << "unknown warper kind " << d.kind;
  }
}

std::vector<warper_v> make_chain(ref_warper_desc const *chain, int len) {
  std::vector<warper_v> v;
  for (int i = 0; i < len; ++i) v.push_back(make_warper(chain[i]));
  return v;
}

std::pair<std::vector<double>, double> chain_reverse(std::vector<warper_v> const &ws, std::vector<double> const &li,
                                                     int start, int end) {
  double jac = 1.0;
  std::vector<double> x = li;
  for (int i = start - 1; i >= end; --i) {
    auto out = std::visit([&x](auto &&w) { return w.map_reverse(x); }, ws[static_cast<size_t>(i)]);
    x = out.first;
    jac *= out.second;
  }
  return {x, jac};
}

std::pair<std::vector<double>, double> chain_forward(std::vector<warper_v> const &ws, std::vector<double> const &ui,
                                                     int start, int end) {
  double jac = 1.0;
  std::vector<double> x = ui;
  for (int i = start; i < end; ++i) {
    auto out = std::visit([&x](auto &&w) { return w.map_forward(x); }, ws[static_cast<size_t>(i)]);
    x = out.first;
    jac *= out.second;
  }
  return {x, jac};
}

struct ref_model {
  g0_model model;
};

struct ref_gf_index {
  double time;
  int spin;
  int k_idx;
  int timesplit;
  int orbital;
};

gf_index_t to_index(ref_gf_index const &x) { return gf_index_t{x.time, x.spin, x.k_idx, x.timesplit, x.orbital}; }

} // namespace

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

int ref_sobol_matrices(int dim, int m, std::uint32_t *Cs) {
  qmc::JK2008_sobol_matrices(Cs, static_cast<unsigned>(dim), static_cast<unsigned>(m));
  return 0;
}

// `count` successive draws of keldy::sobol(dim, seed[, shift...]) (qrng.hpp:51-58).
int ref_sobol_points(int dim, int seed, int do_shift, int do_scramble, int seed_shift, int log_max_points,
                     long count, double *out) {
  try {
    auto g = make_sobol(dim, seed, do_shift != 0, do_scramble != 0, seed_shift, log_max_points);
    for (long p = 0; p < count; ++p) {
      if (g.past_end()) TRIQS_RUNTIME_ERROR << "More sample points requested then generator can hold.";
      auto x = g.next();
      std::memcpy(out + p * dim, x.data(), sizeof(double) * static_cast<size_t>(dim));
    }
  } catch (std::exception const &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

// direction 0: map_reverse(li, start, end); 1: map_forward(ui, start, end).
int ref_warp(ref_warper_desc const *chain, int len, int direction, int start, int end, int n, long count,
             double const *in, double *out, double *jac) {
  try {
    auto ws = make_chain(chain, len);
    for (long p = 0; p < count; ++p) {
      std::vector<double> x(in + p * n, in + (p + 1) * n);
      auto r = direction == 0 ? chain_reverse(ws, x, start, end) : chain_forward(ws, x, start, end);
      std::memcpy(out + p * n, r.first.data(), sizeof(double) * static_cast<size_t>(n));
      jac[p] = r.second;
    }
  } catch (std::exception const &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

// keldy's warper_product_1d_simple_interp_nearest_t(times_u_pts, f1_pts) on count points
// of n coordinates: direction 0 map_reverse, 1 map_forward.
int ref_interp_nearest(int npts, double const *u, double const *f1, int direction, int n, long count,
                       double const *in, double *out, double *jac) {
  try {
    triqs::arrays::vector<double> tu(npts), tf(npts);
    for (int i = 0; i < npts; ++i) {
      tu[i] = u[i];
      tf[i] = f1[i];
    }
    warper_product_1d_simple_interp_nearest_t w(tu, tf);
    for (long p = 0; p < count; ++p) {
      std::vector<double> x(in + p * n, in + (p + 1) * n);
      auto r = direction == 0 ? w.map_reverse(x) : w.map_forward(x);
      std::memcpy(out + p * n, r.first.data(), sizeof(double) * static_cast<size_t>(n));
      jac[p] = r.second;
    }
  } catch (std::exception const &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

// A g0 model whose lesser/greater tables (interleaved complex, orbital (0,0), on the
// mesh [-time_max, time_max] with npts points) are given; spin down = spin up.
void *ref_model_create(int npts, double time_max, double alpha, double const *lesser, double const *greater) {
  auto *m = new ref_model{};
  model_param_t p;
  p.alpha = alpha;
  p.time_max = time_max;
  p.nr_time_points_gf = npts | 1;
  m->model.model_omega = g0_model_omega{p};
  triqs::gfs::gf<triqs::gfs::retime, triqs::gfs::matrix_valued> gl(-time_max, time_max, npts), gg(-time_max, time_max, npts);
  for (long i = 0; i < npts; ++i) {
    gl.at(i, 0, 0) = {lesser[2 * i], lesser[2 * i + 1]};
    gg.at(i, 0, 0) = {greater[2 * i], greater[2 * i + 1]};
  }
  m->model.g0_lesser.blocks = {gl, gl};
  m->model.g0_greater.blocks = {gg, gg};
  return m;
}

void ref_model_destroy(void *m) { delete static_cast<ref_model *>(m); }

int ref_g0(void *mh, ref_gf_index const *a, ref_gf_index const *b, int internal, double *out) {
  try {
    g0_keldysh_contour_t g0{static_cast<ref_model *>(mh)->model};
    auto v = g0(to_index(*a), to_index(*b), internal != 0);
    out[0] = v.real();
    out[1] = v.imag();
  } catch (std::exception const &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

// integrand_g_direct::operator() (or eval_no_det when no_det != 0) on `count` time vectors.
int ref_integrand(void *mh, ref_gf_index const *A, ref_gf_index const *B, double cutoff, int n, long count,
                  double const *times, int keep_u_hypercube, int no_det, double *out, int *in_domain) {
  try {
    integrand_g_direct f{g0_keldysh_contour_t{static_cast<ref_model *>(mh)->model}, to_index(*A), to_index(*B), cutoff};
    for (long p = 0; p < count; ++p) {
      std::vector<double> t(times + p * n, times + (p + 1) * n);
      auto r = no_det ? f.eval_no_det(t, keep_u_hypercube != 0) : f(t, keep_u_hypercube != 0);
      out[2 * p] = r.first.real();
      out[2 * p + 1] = r.first.imag();
      in_domain[p] = r.second;
    }
  } catch (std::exception const &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

// integrator::run(nr_steps) + reduce_result (integrator.hpp:81-95, 123-131) with the
// sobol_unshifted generator of the given seed (or a shifted/scrambled one).
// mode 0 = as shipped: one loop, OpenMP inside the integrand with `threads` threads;
// mode 1 = MPI-equivalent: `threads` workers, worker r keeps point i when
// i % threads == r (integrator.hpp:84-88), the integrand runs single-threaded.
// result[0..1] = sum of f*J, result[2] = points run, result[3] = points in domain.
int ref_integrate(void *mh, ref_gf_index const *A, ref_gf_index const *B, double cutoff, ref_warper_desc const *chain,
                  int len, int n, int seed, int do_shift, int do_scramble, int seed_shift, long nr_steps, int mode,
                  int threads, double *result) {
  try {
    integrand_g_direct f{g0_keldysh_contour_t{static_cast<ref_model *>(mh)->model}, to_index(*A), to_index(*B), cutoff};
    auto ws = make_chain(chain, len);
    if (mode == 0) {
      omp_set_max_active_levels(1);
      omp_set_num_threads(threads);
      auto g = make_sobol(n, seed, do_shift != 0, do_scramble != 0, seed_shift, 31);
      std::complex<double> acc = 0;
      std::uint64_t npts = 0, ndom = 0;
      for (long i = 0; i < nr_steps; ++i) {
        auto li = g.next();
        auto [ui, jac] = chain_reverse(ws, li, len, 0);
        auto [val, dom] = f(ui, true);
        val *= jac;
        acc += val;
        npts++;
        ndom += static_cast<std::uint64_t>(dom);
      }
      result[0] = acc.real();
      result[1] = acc.imag();
      result[2] = static_cast<double>(npts);
      result[3] = static_cast<double>(ndom);
    } else {
      omp_set_max_active_levels(1);
      std::vector<std::complex<double>> acc(static_cast<size_t>(threads));
      std::vector<std::uint64_t> npts(static_cast<size_t>(threads)), ndom(static_cast<size_t>(threads));
#pragma omp parallel num_threads(threads)
      {
        int r = omp_get_thread_num(), size = omp_get_num_threads();
        auto g = make_sobol(n, seed, do_shift != 0, do_scramble != 0, seed_shift, 31);
        std::complex<double> a = 0;
        std::uint64_t np = 0, nd = 0;
        for (long i = 0; i < nr_steps; ++i) {
          auto li = g.next();
          if (i % size != r) continue;
          auto [ui, jac] = chain_reverse(ws, li, len, 0);
          auto [val, dom] = f(ui, true);
          val *= jac;
          a += val;
          np++;
          nd += static_cast<std::uint64_t>(dom);
        }
        acc[static_cast<size_t>(r)] = a;
        npts[static_cast<size_t>(r)] = np;
        ndom[static_cast<size_t>(r)] = nd;
      }
      std::complex<double> s = 0;
      std::uint64_t np = 0, nd = 0;
      for (int r = 0; r < threads; ++r) {
        s += acc[static_cast<size_t>(r)];
        np += npts[static_cast<size_t>(r)];
        nd += ndom[static_cast<size_t>(r)];
      }
      result[0] = s.real();
      result[1] = s.imag();
      result[2] = static_cast<double>(np);
      result[3] = static_cast<double>(nd);
    }
  } catch (std::exception const &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

} // extern "C"
