// C ABI of the device-resident product warpers (kb_warper_table_*, kb_warper_projection_*,
// include/keldy_b200.h). The tables are built once on the host, as keldy builds them:
// * warper_product_1d_simple_interp_nearest_t (integrate_and_inverse,
//   product_1d_simple.hpp:219-253) and make_warper_from_proj (make_warper_from_proj.hpp);
// * warper_projection_t (projection.hpp:176-382): binned |f J| per axis, Gaussian local
//   linear smoothing of its logarithm (optional Brent search of the width), the smoothed
//   projection's integral and its Akima-interpolated inverse on uniform meshes;
// * warper_product_1d_simple_interp_hybrid_t (product_1d_simple.hpp:381-554): Simpson
//   integral of a closed-form f1 and Steffen splines of the integral and its inverse;
// * warper_product_1d_t (product_1d.hpp:110-160): one analytic product maker per axis.
// The warper chain evaluates them on the device (table_reverse / table_forward,
// kb_device.cuh).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <functional>
#include <vector>

#include "kb_host.h"

using namespace kb;

namespace {

// One coordinate's table on the host: the descriptor (device pointers filled at upload)
// and up to four arrays (p0..p3).
struct HostDim {
  TableDimDev meta{};
  std::vector<double> a[4];
  std::vector<double> u_in, f1_in; // nearest tables: the points and f1 as given
};

// ------------------------------------------------------------ interpolation tools

// Interval of the increasing points x[0..n) holding v (GSL's bisection: the last point
// falls in the last interval).
int interval(const double *x, int n, double v) {
  int lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    const int m = (lo + hi) >> 1;
    if (x[m] > v)
      hi = m;
    else
      lo = m;
  }
  return lo;
}

// GSL's linear spline at v (v inside [x[0], x[n-1]]).
double linear_at(const std::vector<double> &x, const std::vector<double> &y, double v) {
  const int i = interval(x.data(), (int)x.size(), v);
  const double dx = x[(size_t)i + 1] - x[(size_t)i];
  return dx > 0.0 ? y[(size_t)i] + (v - x[(size_t)i]) / dx * (y[(size_t)i + 1] - y[(size_t)i]) : y[(size_t)i];
}

// A function on the uniform mesh of [0, 1] with n points, linearly interpolated (TRIQS
// gf<retime> evaluation; the device's mesh_eval). NaN outside the mesh.
double mesh_at(const std::vector<double> &g, double x) {
  const long n = (long)g.size();
  const double delta_inv = 1.0 / (1.0 / (double)(n - 1));
  const double a = x * delta_inv;
  double fi = std::floor(a);
  double w = a - fi;
  long i = (long)fi;
  if (i == n - 1 && std::fabs(w) < 1e-14) {
    i = n - 2;
    w = 1.0;
  }
  if (!(i >= 0 && i < n - 1)) return NAN;
  return (1.0 - w) * g[(size_t)i] + w * g[(size_t)i + 1];
}

// Cubic Hermite interpolation from end values and slopes (the device's table_hermite).
double hermite(double x, double x0, double x1, double y0, double y1, double d0, double d1) {
  const double h = x1 - x0;
  const double s = (y1 - y0) / h;
  const double c2 = (3.0 * s - 2.0 * d0 - d1) / h;
  const double c3 = (d0 + d1 - 2.0 * s) / (h * h);
  const double dx = x - x0;
  return y0 + dx * (d0 + dx * (c2 + dx * c3));
}

// Akima's interpolation (H. Akima, J. ACM 17 (1970) 589): on each interval the cubic
// Hermite polynomial whose node slopes are
//   t_i = (|m_{i+1} - m_i| m_{i-1} + |m_{i-1} - m_{i-2}| m_i) / (|m_{i+1} - m_i| + |m_{i-1} - m_{i-2}|)
// (the mean of m_{i-1} and m_i when both weights vanish), m_k the secant slope of interval
// k, extended past each end by m_{-1} = 2 m_0 - m_1, m_{-2} = 2 m_{-1} - m_0 (and the
// mirror image at the right end). Returns the node slopes.
std::vector<double> akima_slopes(const std::vector<double> &x, const std::vector<double> &y) {
  const int n = (int)x.size();
  std::vector<double> m((size_t)n + 3); // m[k + 2] = slope of interval k, k in [-2, n]
  for (int k = 0; k < n - 1; ++k) m[(size_t)k + 2] = (y[(size_t)k + 1] - y[(size_t)k]) / (x[(size_t)k + 1] - x[(size_t)k]);
  m[1] = 2.0 * m[2] - m[3];
  m[0] = 2.0 * m[1] - m[2];
  m[(size_t)n + 1] = 2.0 * m[(size_t)n] - m[(size_t)n - 1];
  m[(size_t)n + 2] = 2.0 * m[(size_t)n + 1] - m[(size_t)n];
  std::vector<double> t((size_t)n);
  for (int i = 0; i < n; ++i) {
    const double mm2 = m[(size_t)i], mm1 = m[(size_t)i + 1], m0 = m[(size_t)i + 2], mp1 = m[(size_t)i + 3];
    const double wl = std::fabs(mp1 - m0), wr = std::fabs(mm1 - mm2);
    t[(size_t)i] = (wl + wr > 0.0) ? (wl * mm1 + wr * m0) / (wl + wr) : 0.5 * (mm1 + m0);
  }
  return t;
}

// Steffen's monotone interpolation (M. Steffen, Astron. Astrophys. 239 (1990) 443): node
// slopes (sign s_{i-1} + sign s_i) min(|s_{i-1}|, |s_i|, |p_i| / 2) with
// p_i = (s_{i-1} h_i + s_i h_{i-1}) / (h_{i-1} + h_i); at the two ends the end secant (the
// paper's simplest choice).
std::vector<double> steffen_slopes(const double *x, const double *y, int n) {
  std::vector<double> d((size_t)n);
  d[0] = (y[1] - y[0]) / (x[1] - x[0]);
  for (int i = 1; i < n - 1; ++i) {
    const double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
    const double s0 = (y[i] - y[i - 1]) / h0, s1 = (y[i + 1] - y[i]) / h1;
    const double p = (s0 * h1 + s1 * h0) / (h0 + h1);
    d[(size_t)i] = (std::copysign(1.0, s0) + std::copysign(1.0, s1)) *
                   std::min(std::fabs(s0), std::min(std::fabs(s1), 0.5 * std::fabs(p)));
  }
  d[(size_t)n - 1] = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
  return d;
}

// ------------------------------------------------------------ smoothing

// Weighted least-squares line through (x, y) with the weights w > 0 (the others left
// out); its value at x0.
double wlinear_at(const double *x, const double *y, const double *w, int n, double x0) {
  double W = 0.0, mx = 0.0, my = 0.0;
  for (int i = 0; i < n; ++i)
    if (w[i] > 0.0) {
      W += w[i];
      mx += w[i] * x[i];
      my += w[i] * y[i];
    }
  mx /= W;
  my /= W;
  double sxx = 0.0, sxy = 0.0;
  for (int i = 0; i < n; ++i)
    if (w[i] > 0.0) {
      const double dx = x[i] - mx;
      sxx += w[i] * dx * dx;
      sxy += w[i] * dx * (y[i] - my);
    }
  const double c1 = sxy / sxx;
  return (my - mx * c1) + x0 * c1;
}

// local_linear_reg (interfaces/gsl_fit_linear_wrap.hpp:66-113) on x = 0..N-1: at every
// point the weighted linear fit over the kernel window centred on it, the dead points
// (weight 0) left out.
std::vector<double> local_linear_reg(const std::vector<double> &y, const std::vector<double> &kernel,
                                     const std::vector<char> &dead) {
  const int N = (int)y.size();
  const int K = (int)kernel.size();
  const int H = K / 2;
  std::vector<double> x((size_t)N), out((size_t)N), w((size_t)K);
  for (int i = 0; i < N; ++i) x[(size_t)i] = i;
  for (int i = 0; i < N; ++i) {
    const int start_ker = std::max(0, H - i);
    const int end_ker = std::min(N + H - i - 1, K - 1);
    const int size = end_ker - start_ker + 1;
    const int start_x = start_ker - H + i;
    for (int j = 0; j < size; ++j) w[(size_t)j] = dead[(size_t)(start_x + j)] ? 0.0 : kernel[(size_t)(start_ker + j)];
    out[(size_t)i] = wlinear_at(x.data() + start_x, y.data() + start_x, w.data(), size, x[(size_t)i]);
  }
  return out;
}

std::vector<char> dead_points(const std::vector<double> &y) {
  std::vector<char> d(y.size());
  for (size_t i = 0; i < y.size(); ++i) d[i] = !(y[i] > 0.0);
  return d;
}

// kernel_smoothing (make_warper_from_proj.hpp:40-66, projection.hpp:52-78): exp of the
// local linear fit of log y, Gaussian weights exp(-((j - H) / sigma)^2 / 2) on the window
// of H = max(min(int(3 sigma), N), 1) points on each side, sigma in bins.
std::vector<double> kernel_smoothing(const std::vector<double> &y, double sigma) {
  const int N = (int)y.size();
  const int H = std::max(std::min((int)(3 * sigma), N), 1);
  std::vector<double> ker((size_t)(2 * H + 1)), logy((size_t)N);
  for (int j = 0; j <= 2 * H; ++j) ker[(size_t)j] = std::exp(-std::pow((j - H) / sigma, 2) / 2);
  for (int i = 0; i < N; ++i) logy[(size_t)i] = std::log(y[(size_t)i]);
  std::vector<double> out = local_linear_reg(logy, ker, dead_points(y));
  for (auto &v : out) v = std::exp(v);
  return out;
}

// Brent's minimisation without derivatives (R. P. Brent, Algorithms for Minimization
// without Derivatives, 1973, ch. 5): golden-section steps, parabolic steps through the
// three best points when they stay well inside the bracket. Starts from the bracket
// (a, x, b) with f(x) below both ends; stops when the bracket is narrower than abstol or
// after max_iter steps; returns the best point.
int brent_minimize(const std::function<double(double)> &f, double a, double x, double b, double abstol,
                   int max_iter, double &xmin) {
  const double golden = 0.5 * (3.0 - std::sqrt(5.0));
  double fx = f(x);
  const double fa = f(a), fb = f(b);
  if (!std::isfinite(fx) || !std::isfinite(fa) || !std::isfinite(fb)) return fail(KB_E_INVALID, "Function returned Nan or Inf.");
  if (!(fx < fa && fx < fb))
    return fail(KB_E_INVALID, "Endpoints do not enclose a minimum. Make sure f(x_lower) > f(x_guess) < f(x_upper)");
  double v = x, w = x, fv = fx, fw = fx, d = 0.0, e = 0.0;
  for (int it = 0; it < max_iter; ++it) {
    const double mid = 0.5 * (a + b);
    const double tol = std::sqrt(DBL_EPSILON) * std::fabs(x) + 1e-12;
    bool parabolic = false;
    if (std::fabs(e) > tol) {
      double r = (x - w) * (fx - fv);
      double q = (x - v) * (fx - fw);
      double p = (x - v) * q - (x - w) * r;
      q = 2.0 * (q - r);
      if (q > 0.0)
        p = -p;
      else
        q = -q;
      const double e_prev = e;
      e = d;
      if (std::fabs(p) < std::fabs(0.5 * q * e_prev) && p > q * (a - x) && p < q * (b - x)) {
        d = p / q;
        const double u = x + d;
        if (u - a < 2.0 * tol || b - u < 2.0 * tol) d = (x < mid) ? tol : -tol;
        parabolic = true;
      }
    }
    if (!parabolic) {
      e = (x < mid) ? b - x : a - x;
      d = golden * e;
    }
    const double u = (std::fabs(d) >= tol) ? x + d : x + (d > 0.0 ? tol : -tol);
    const double fu = f(u);
    if (!std::isfinite(fu)) return fail(KB_E_INVALID, "Function returned Nan or Inf.");
    if (fu <= fx) {
      if (u < x)
        b = x;
      else
        a = x;
      v = w;
      fv = fw;
      w = x;
      fw = fx;
      x = u;
      fx = fu;
    } else {
      if (u < x)
        a = u;
      else
        b = u;
      if (fu <= fw || w == x) {
        v = w;
        fv = fw;
        w = u;
        fw = fu;
      } else if (fu <= fv || v == x || v == w) {
        v = u;
        fv = fu;
      }
    }
    if (std::fabs(b - a) < abstol) break;
  }
  xmin = x;
  return KB_OK;
}

// optimize_sigma (projection.hpp:82-128): the smoothing width (in bins, >= 0.3) that
// minimises the leave-one-out squared error of the smoothed projection, searched by
// Brent's method on [-upper, upper] from sigma (the cost is even in sigma), 20 steps,
// absolute tolerance 1e-8.
int optimize_sigma(const std::vector<double> &y, double sigma, double upper, double &out) {
  const int N = (int)y.size();
  const double sigma_min = 0.3;
  std::vector<double> log_y((size_t)N);
  const std::vector<char> dead = dead_points(y);
  for (int i = 0; i < N; ++i) log_y[(size_t)i] = dead[(size_t)i] ? 0.0 : std::log(y[(size_t)i]);
  const int H = std::max(std::min((int)(3 * upper), N), 1);
  std::vector<double> kernel((size_t)(2 * H + 1));
  bool bad = false;
  auto cost = [&](double s) -> double {
    s = std::max(std::fabs(s), sigma_min);
    for (int j = 0; j <= 2 * H; ++j) kernel[(size_t)j] = std::exp(-std::pow((j - H) / s, 2) / 2);
    kernel[(size_t)H] = 0.0;
    const double k1 = kernel[(size_t)H + 1];
    for (auto &k : kernel) k /= k1;
    const std::vector<double> fit = local_linear_reg(log_y, kernel, dead);
    double c = 0.0;
    for (int i = 0; i < N; ++i) c += std::pow(std::exp(fit[(size_t)i]) - y[(size_t)i], 2);
    if (std::isnan(c)) bad = true;
    return c;
  };
  double x = 0.0;
  const int st = brent_minimize(cost, -upper, sigma, upper, 1e-8, 20, x);
  if (bad)
    return fail(KB_E_INVALID, "Smoothing procedure returned a Nan. This may be due to a lack of data, try to "
                              "increase the number of samples.");
  if (st) return st;
  out = std::max(std::fabs(x), sigma_min);
  return KB_OK;
}

// ------------------------------------------------------------ builders

// warper_product_1d_simple_interp_nearest_t's integrate_and_inverse: F[n-1] = 0,
// F[i] = F[i+1] - (f1[i+1] + f1[i]) / 2 (u[i+1] - u[i]), normalised by -F[0] (F[0] then
// -1 exactly); f1 on an interval = the mean of its ends; the inverse runs on F[0..cut].
int build_nearest(const double *u, const double *f1, int n, HostDim &h) {
  if (n < 3) return fail(KB_E_INVALID, "Expect nr_sample_points to be >= 3. Given was " + std::to_string(n));
  if (u[0] != 0.0) return fail(KB_E_INVALID, "times_u_pts should start at 0");
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(u[i]) || !std::isfinite(f1[i])) return fail(KB_E_INVALID, "warper table values must be finite");
    if (i > 0 && !(u[i] > u[i - 1])) return fail(KB_E_INVALID, "times_u_pts must be strictly increasing");
  }
  std::vector<double> F((size_t)n, 0.0), f(f1, f1 + n);
  int cut = n - 1;
  bool found = false;
  for (int i = n - 2; i >= 0; --i) {
    F[(size_t)i] = F[(size_t)i + 1] - 0.5 * (f[(size_t)i + 1] + f[(size_t)i]) * (u[i + 1] - u[i]);
    found = found || (F[(size_t)i] != 0);
    if (!found) cut = i;
  }
  if (!found) return fail(KB_E_INVALID, "Model function is flat zero.");
  const double norm = -F[0];
  for (auto &v : F) v /= norm;
  for (auto &v : f) v /= norm;
  F[0] = -1;
  for (int i = 0; i < cut; ++i)
    if (!(F[(size_t)i + 1] > F[(size_t)i]))
      return fail(KB_E_INVALID, "the integral of f1 is not strictly increasing on the warper's support "
                                "(f1 must be > 0 there)");
  h.u_in.assign(u, u + n);
  h.f1_in.assign(f1, f1 + n);
  h.meta.type = TAB_NEAREST;
  h.meta.n = n;
  h.meta.cut = cut;
  h.meta.norm = norm;
  h.a[0].assign(u, u + n);
  h.a[1] = F;
  h.a[2].resize((size_t)n - 1);
  for (int i = 0; i + 1 < n; ++i) h.a[2][(size_t)i] = 0.5 * (f[(size_t)i] + f[(size_t)i + 1]);
  return KB_OK;
}

// The closed-form f1 shapes of the hybrid warpers on the host (the device's hybrid_f1).
double hybrid_f1_host(const SimpleDev &f, double t) {
  switch (f.kind) {
  case KB_WARPER_EXPONENTIAL: return std::exp(-t / f.w);
  case KB_WARPER_INVERSE: return f.w / (f.w + t);
  case KB_WARPER_INVERSE_SQUARE: return f.w * f.w / ((f.w + t) * (f.w + t));
  case KB_WARPER_INVERSE_POWER: {
    double num = f.w, den = f.w + t;
    for (int k = 1; k < f.power; ++k) {
      num *= f.w;
      den *= f.w + t;
    }
    return num / den;
  }
  default: return 1.0;
  }
}

// warper_product_1d_simple_interp_hybrid_t's constructor (product_1d_simple.hpp:424-476):
// equidistant points, F by Simpson's rule from u_max down (f1 at both ends and the middle
// of each interval), normalised; Steffen splines of F(u) and of u(F) on F[0..cut].
int build_hybrid(const kb_warper &spec, int n, HostDim &h) {
  if (!(n >= 3)) return fail(KB_E_INVALID, "Expect nr_sample_points to be >= 3. Given was " + std::to_string(n));
  if (!(spec.u_max > 0.0)) return fail(KB_E_INVALID, "the hybrid warper's domain_u_max must be > 0");
  if (spec.kind != KB_WARPER_EXPONENTIAL && spec.kind != KB_WARPER_INVERSE && spec.kind != KB_WARPER_INVERSE_SQUARE &&
      spec.kind != KB_WARPER_INVERSE_POWER && spec.kind != KB_WARPER_UNIFORM)
    return fail(KB_E_INVALID, "the hybrid warper's f1 must be one of the closed forms (exponential, inverse, "
                              "inverse_square, inverse_power, uniform)");
  if (spec.kind != KB_WARPER_UNIFORM && !(spec.w > 0.0)) return fail(KB_E_INVALID, "w_scale must be > 0");
  if (spec.kind == KB_WARPER_INVERSE_POWER && spec.power < 1) return fail(KB_E_INVALID, "power must be >= 1");
  SimpleDev f{};
  f.kind = spec.kind;
  f.power = spec.power;
  f.u_max = spec.u_max;
  f.w = spec.w;
  const double delta = (spec.u_max - 0.0) / (n - 1);
  std::vector<double> u((size_t)n), F((size_t)n, 0.0);
  for (int i = 0; i < n; ++i) u[(size_t)i] = 0.0 + delta * i;
  u[(size_t)n - 1] = spec.u_max;
  int cut = n - 1;
  bool found = false;
  double f2d = hybrid_f1_host(f, u[(size_t)n - 1]);
  for (int i = n - 2; i >= 0; --i) {
    const double f0d = f2d;
    const double f1d = hybrid_f1_host(f, 0.5 * (u[(size_t)i + 1] + u[(size_t)i]));
    f2d = hybrid_f1_host(f, u[(size_t)i]);
    const double dl = delta / 6. * (f0d + 4 * f1d + f2d);
    F[(size_t)i] = F[(size_t)i + 1] - dl;
    if (dl < 1e-100)
      return fail(KB_E_INVALID, "dl=" + std::to_string(dl) + " < 1e-100 is too small for a cubic interpolator in "
                                                              "double precision.");
    found = found || (F[(size_t)i] != 0);
    if (!found) cut = i;
  }
  if (!found) return fail(KB_E_INVALID, "Model function is flat zero.");
  const double norm = -F[0];
  for (auto &v : F) v /= norm;
  F[0] = -1;
  h.meta.type = TAB_HYBRID;
  h.meta.n = n;
  h.meta.cut = cut;
  h.meta.norm = norm;
  h.meta.f = f;
  h.a[2] = steffen_slopes(u.data(), F.data(), n);
  h.a[3] = steffen_slopes(F.data(), u.data(), cut + 1);
  h.a[0] = u;
  h.a[1] = F;
  return KB_OK;
}

// The binned projections of keldy's gather_data (projection.hpp:190-223,
// make_warper_from_proj.hpp:68-98): per axis the sum of |f J| and the count of the
// samples in each bin of binner_t({xmin, xmax, nb}) (xmin <= x <= xmax kept, x = xmax in
// the last bin), then the mean of every bin with samples.
void gather_axis(const double *li, const double *val, int64_t n, int order, int axis, double xmin, double xmax,
                 int nb, std::vector<double> &data, std::vector<uint64_t> &count) {
  const double bin_size = (xmax - xmin) / nb;
  data.assign((size_t)nb, 0.0);
  count.assign((size_t)nb, 0);
  for (int64_t p = 0; p < n; ++p) {
    const double x = li[(size_t)p * order + axis];
    if (!(xmin <= x && x <= xmax)) continue;
    const int b = (x == xmax) ? nb - 1 : std::min((int)((x - xmin) / bin_size), nb - 1);
    data[(size_t)b] += val[p];
    count[(size_t)b]++;
  }
  for (int b = 0; b < nb; ++b)
    if (count[(size_t)b] > 0) data[(size_t)b] /= (double)count[(size_t)b];
}

struct ProjAxis {
  double sigma = 0.0; // natural units
  std::vector<double> xi;
  std::vector<uint64_t> count;
  std::vector<double> fn;
};

// warper_projection_t's constructor (projection.hpp:225-332) on samples li [n][order] with
// values |f J|: bins of width 1/(nb-1) centred on the mesh points, the width sigma (or the
// optimised one), the smoothed projection fn on the uniform mesh of nb points, its
// integral (midpoint values of fn times the step, partial sums, normalised) and the
// inverse of the integral by Akima's interpolation on 1 + 5 (nb - 1) points.
int build_projection_axis(const double *li, const double *val, int64_t n, int order, int axis, int nb, double sigma,
                          bool optimize, HostDim &h, ProjAxis &info) {
  const double delta = 1.0 / (nb - 1.0);
  const double xmin = -delta / 2, xmax = 1 + delta / 2;
  const double bin_size = (xmax - xmin) / nb;
  gather_axis(li, val, n, order, axis, xmin, xmax, nb, info.xi, info.count);
  double s = sigma / bin_size;
  if (optimize) {
    if (bin_size >= 2) return fail(KB_E_INVALID, "delta too large");
    int st = optimize_sigma(info.xi, s, 1.0 / bin_size, s);
    if (st) return st;
  }
  info.sigma = s * bin_size;
  const std::vector<double> sm = kernel_smoothing(info.xi, s);
  std::vector<double> times((size_t)nb);
  for (int i = 0; i < nb; ++i) times[(size_t)i] = xmin + (i + 0.5) * bin_size;
  times[0] = 0;
  times[(size_t)nb - 1] = 1;
  const double mdelta = (1.0 - 0.0) / (nb - 1);
  std::vector<double> mesh((size_t)nb), fn((size_t)nb), fint((size_t)nb);
  for (int j = 0; j < nb; ++j) mesh[(size_t)j] = 0.0 + j * mdelta;
  for (int j = 0; j < nb; ++j) fn[(size_t)j] = linear_at(times, sm, mesh[(size_t)j]);
  for (int j = 0; j < nb; ++j) fint[(size_t)j] = (j == 0) ? 0.0 : mesh_at(fn, mesh[(size_t)j] - mdelta / 2) * mdelta;
  for (int j = 1; j < nb; ++j) fint[(size_t)j] += fint[(size_t)j - 1];
  const double norm = fint[(size_t)nb - 1];
  for (auto &v : fint) v /= norm;
  for (int j = 0; j < nb; ++j)
    if (!std::isfinite(fn[(size_t)j]) || !(fn[(size_t)j] > 0.0))
      return fail(KB_E_INVALID, "the smoothed projection is not positive and finite on axis " + std::to_string(axis) +
                                    " (too few samples?)");
  for (int j = 1; j < nb; ++j)
    if (!(fint[(size_t)j] > fint[(size_t)j - 1]))
      return fail(KB_E_INVALID, "the integral of the smoothed projection is not strictly increasing");
  const std::vector<double> t = akima_slopes(fint, mesh);
  const int M = 1 + 5 * (nb - 1);
  std::vector<double> inv((size_t)M);
  const double ldelta = (1.0 - 0.0) / (M - 1);
  for (int k = 0; k < M; ++k) {
    const double l = 0.0 + k * ldelta;
    const int i = interval(fint.data(), nb, l);
    inv[(size_t)k] = hermite(l, fint[(size_t)i], fint[(size_t)i + 1], mesh[(size_t)i], mesh[(size_t)i + 1],
                             t[(size_t)i], t[(size_t)i + 1]);
  }
  info.fn = fn;
  h.meta.type = TAB_PROJECTION;
  h.meta.n = nb;
  h.meta.m = M;
  h.meta.norm = norm;
  h.a[0] = fn;
  h.a[1] = fint;
  h.a[2] = inv;
  return KB_OK;
}

// Copies the tables to the device and makes the kb_warper_table.
int upload(kb_context *ctx, std::vector<HostDim> &dims, int type, double u_max, kb_warper_table **out) {
  const int ndims = (int)dims.size();
  size_t total = 0;
  for (auto &d : dims)
    for (auto &a : d.a) total += a.size();
  std::vector<double> host(std::max<size_t>(total, 1));
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  auto *t = new kb_warper_table;
  t->ctx = ctx;
  t->device = ctx->device;
  t->ndims = ndims;
  t->type = type;
  t->u_max = u_max;
  cudaError_t e = device_malloc(&t->d_data, host.size() * sizeof(double));
  if (e == cudaSuccess) e = device_malloc(&t->d_dims, (size_t)ndims * sizeof(TableDimDev));
  std::vector<TableDimDev> meta((size_t)ndims);
  size_t pos = 0;
  for (int d = 0; d < ndims; ++d) {
    meta[(size_t)d] = dims[(size_t)d].meta;
    const double **ptr[4] = {&meta[(size_t)d].p0, &meta[(size_t)d].p1, &meta[(size_t)d].p2, &meta[(size_t)d].p3};
    for (int k = 0; k < 4; ++k) {
      const auto &a = dims[(size_t)d].a[k];
      *ptr[k] = a.empty() ? nullptr : (e == cudaSuccess ? t->d_data + pos : nullptr);
      std::copy(a.begin(), a.end(), host.begin() + (long)pos);
      pos += a.size();
    }
    t->npts.push_back(dims[(size_t)d].meta.n);
    t->pts_u.push_back(dims[(size_t)d].u_in);
    t->pts_f1.push_back(dims[(size_t)d].f1_in);
  }
  // on the library's stream, which does not synchronise with the legacy default stream
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(t->d_data, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(t->d_dims, meta.data(), meta.size() * sizeof(TableDimDev), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(t->d_data);
    cudaFree(t->d_dims);
    delete t;
    return fail(KB_E_CUDA, std::string("kb_warper_table: ") + cudaGetErrorString(e));
  }
  *out = t;
  return KB_OK;
}

// make_warper_from_proj's tables (make_warper_from_proj.hpp:118-153) from samples li
// [n][order] with values |f J|: num_bins bins of [0, 1] per axis, smoothed, turned into
// f1 points f1[0] = 0, f1[i+1] = 2 s_i - f1[i] on the bin edges.
int tables_from_samples(kb_context *ctx, int order, int num_bins, int64_t n, const double *li, const double *val,
                        double sigma, kb_warper_table **out) {
  const double bin_size = 1.0 / num_bins;
  std::vector<double> tu((size_t)num_bins + 1);
  for (int i = 0; i <= num_bins; ++i) tu[(size_t)i] = i * bin_size;
  tu[(size_t)num_bins] = 1.0;
  std::vector<HostDim> dims((size_t)order);
  for (int axis = 0; axis < order; ++axis) {
    std::vector<double> xi;
    std::vector<uint64_t> cnt;
    gather_axis(li, val, n, order, axis, 0.0, 1.0, num_bins, xi, cnt);
    const std::vector<double> sm = kernel_smoothing(xi, sigma / bin_size);
    std::vector<double> f1((size_t)num_bins + 1);
    f1[0] = 0;
    for (int i = 0; i < num_bins; ++i) f1[(size_t)i + 1] = 2 * sm[(size_t)i] - f1[(size_t)i];
    int st = build_nearest(tu.data(), f1.data(), num_bins + 1, dims[(size_t)axis]);
    if (st) return st;
  }
  return upload(ctx, dims, KB_TABLE_NEAREST, 1.0, out);
}

// Sobol points 1..nr_samples of dimension order (keldy's sobol(order, 0), unshifted) and
// |f J| there through `chain` on the GPU.
int gpu_samples(kb_context *ctx, const kb_model *m, const kb_integrand *f, const kb_warper *chain, int chain_len,
                int order, int nr_samples, int keep_u_hypercube, std::vector<double> &li, std::vector<double> &absval) {
  kb_sobol *g = nullptr;
  int st = kb_sobol_create(ctx, order, 31, 0, 0, 0, &g);
  if (st) return st;
  li.assign((size_t)nr_samples * order, 0.0);
  std::vector<double> val(2 * (size_t)nr_samples);
  st = kb_sobol_points(ctx, g, 1, nr_samples, li.data());
  kb_sobol_destroy(g);
  if (st) return st;
  st = kb_evaluate_warped(ctx, m, f, chain, chain_len, chain_len, order, nr_samples, li.data(), keep_u_hypercube,
                          KB_ALGO_AUTO, val.data(), nullptr, nullptr);
  if (st) return st;
  absval.resize((size_t)nr_samples);
  for (int p = 0; p < nr_samples; ++p) absval[(size_t)p] = std::hypot(val[2 * (size_t)p], val[2 * (size_t)p + 1]);
  return KB_OK;
}

int check_params(int order, int num_bins, int64_t n, double sigma, int min_bins) {
  KB_CHECK(order >= 1 && order <= MAX_ORDER, "order must be in [1, 16]");
  KB_CHECK(num_bins >= min_bins && num_bins <= (1 << 20),
           "num_bins must be in [" + std::to_string(min_bins) + ", 2^20]");
  KB_CHECK(n >= 1, "need at least one sample");
  KB_CHECK(sigma > 0.0, "sigma must be > 0");
  return KB_OK;
}

int projection_from_samples(kb_context *ctx, int order, int num_bins, int64_t n, const double *li, const double *val,
                            double sigma, int optimize, kb_warper_table **out) {
  std::vector<HostDim> dims((size_t)order);
  std::vector<ProjAxis> info((size_t)order);
  for (int axis = 0; axis < order; ++axis) {
    int st = build_projection_axis(li, val, n, order, axis, num_bins, sigma, optimize != 0, dims[(size_t)axis],
                                   info[(size_t)axis]);
    if (st) return st;
  }
  int st = upload(ctx, dims, KB_TABLE_PROJECTION, 1.0, out);
  if (st) return st;
  for (auto &a : info) {
    (*out)->sigmas.push_back(a.sigma);
    (*out)->xi.push_back(a.xi);
    (*out)->xi_count.push_back(a.count);
    (*out)->fn.push_back(a.fn);
  }
  return KB_OK;
}

} // namespace

extern "C" {

int kb_warper_table_create(kb_context *ctx, int ndims, const int *npts, const double *u_pts, const double *f1_pts,
                           kb_warper_table **out) {
  KB_CHECK(ctx && npts && u_pts && f1_pts && out, "kb_warper_table_create: null argument");
  KB_CHECK(ndims >= 1 && ndims <= MAX_ORDER, "a tabulated warper has 1 to 16 tables");
  std::vector<HostDim> dims((size_t)ndims);
  size_t off = 0;
  for (int d = 0; d < ndims; ++d) {
    int st = build_nearest(u_pts + off, f1_pts + off, npts[d], dims[(size_t)d]);
    if (st) return st;
    off += (size_t)npts[d];
  }
  return upload(ctx, dims, KB_TABLE_NEAREST, u_pts[npts[0] - 1], out);
}

int kb_warper_table_analytic(kb_context *ctx, int ndims, const kb_warper *dims_in, kb_warper_table **out) {
  KB_CHECK(ctx && dims_in && out, "kb_warper_table_analytic: null argument");
  KB_CHECK(ndims >= 1 && ndims <= MAX_ORDER, "a product warper has 1 to 16 coordinates");
  std::vector<HostDim> dims((size_t)ndims);
  for (int d = 0; d < ndims; ++d) {
    const int k = dims_in[d].kind;
    KB_CHECK(k == KB_WARPER_EXPONENTIAL || k == KB_WARPER_INVERSE || k == KB_WARPER_INVERSE_SQUARE ||
                 k == KB_WARPER_INVERSE_POWER || k == KB_WARPER_UNIFORM,
             "warper_product_1d_t takes the product makers' warpers (exponential, inverse, inverse_square, "
             "inverse_power, uniform)");
    int st = simple_dev(dims_in[d], dims[(size_t)d].meta.f);
    if (st) return st;
    dims[(size_t)d].meta.type = TAB_ANALYTIC;
  }
  return upload(ctx, dims, KB_TABLE_ANALYTIC, dims_in[0].u_max, out);
}

int kb_warper_table_hybrid(kb_context *ctx, int ndims, const kb_warper *f1, const int *npts, kb_warper_table **out) {
  KB_CHECK(ctx && f1 && npts && out, "kb_warper_table_hybrid: null argument");
  KB_CHECK(ndims >= 1 && ndims <= MAX_ORDER, "a hybrid warper has 1 to 16 tables");
  std::vector<HostDim> dims((size_t)ndims);
  for (int d = 0; d < ndims; ++d) {
    int st = build_hybrid(f1[d], npts[d], dims[(size_t)d]);
    if (st) return st;
  }
  return upload(ctx, dims, KB_TABLE_HYBRID, f1[0].u_max, out);
}

int kb_warper_table_destroy(kb_warper_table *t) {
  if (!t) return KB_OK;
  cudaSetDevice(t->device);
  cudaFree(t->d_data);
  cudaFree(t->d_dims);
  delete t;
  return KB_OK;
}

int kb_warper_table_info(const kb_warper_table *t, int *type, int *ndims, int *npts) {
  KB_CHECK(t, "null warper table");
  if (type) *type = t->type;
  if (ndims) *ndims = t->ndims;
  if (npts)
    for (int d = 0; d < t->ndims; ++d) npts[d] = t->npts[(size_t)d];
  return KB_OK;
}

int kb_warper_table_points(const kb_warper_table *t, int d, double *u, double *f1) {
  KB_CHECK(t, "null warper table");
  KB_CHECK(t->type == KB_TABLE_NEAREST, "not an interp-nearest warper");
  KB_CHECK(d >= 0 && d < t->ndims, "out of range axis");
  if (u) std::copy(t->pts_u[(size_t)d].begin(), t->pts_u[(size_t)d].end(), u);
  if (f1) std::copy(t->pts_f1[(size_t)d].begin(), t->pts_f1[(size_t)d].end(), f1);
  return KB_OK;
}

int kb_warper_table_from_samples(kb_context *ctx, int order, int num_bins, int64_t n, const double *li,
                                 const double *values, double sigma, kb_warper_table **out) {
  KB_CHECK(ctx && out && li && values, "kb_warper_table_from_samples: null argument");
  int st = check_params(order, num_bins, n, sigma, 2);
  if (st) return st;
  return tables_from_samples(ctx, order, num_bins, n, li, values, sigma, out);
}

int kb_warper_table_from_projection(kb_context *ctx, const kb_model *m, const kb_integrand *f,
                                    const kb_warper *chain, int chain_len, int order, int num_bins, int nr_samples,
                                    double sigma, int keep_u_hypercube, kb_warper_table **out) {
  KB_CHECK(ctx && m && f && out, "kb_warper_table_from_projection: null argument");
  int st = check_params(order, num_bins, nr_samples, sigma, 2);
  if (st) return st;
  std::vector<double> li, val;
  st = gpu_samples(ctx, m, f, chain, chain_len, order, nr_samples, keep_u_hypercube, li, val);
  if (st) return st;
  return tables_from_samples(ctx, order, num_bins, nr_samples, li.data(), val.data(), sigma, out);
}

int kb_warper_projection_create(kb_context *ctx, int order, int num_bins, int64_t n, const double *li,
                                const double *values, double sigma, int optimize_sigma, kb_warper_table **out) {
  KB_CHECK(ctx && out && li && values, "kb_warper_projection_create: null argument");
  int st = check_params(order, num_bins, n, sigma, 5);
  if (st) return st;
  return projection_from_samples(ctx, order, num_bins, n, li, values, sigma, optimize_sigma, out);
}

int kb_warper_projection_from_integrand(kb_context *ctx, const kb_model *m, const kb_integrand *f,
                                        const kb_warper *chain, int chain_len, int order, int num_bins,
                                        int nr_samples, double sigma, int optimize_sigma, int keep_u_hypercube,
                                        kb_warper_table **out) {
  KB_CHECK(ctx && m && f && out, "kb_warper_projection_from_integrand: null argument");
  std::vector<double> li, val;
  int st = check_params(order, num_bins, nr_samples, sigma, 5);
  if (st) return st;
  st = gpu_samples(ctx, m, f, chain, chain_len, order, nr_samples, keep_u_hypercube, li, val);
  if (st) return st;
  return projection_from_samples(ctx, order, num_bins, nr_samples, li.data(), val.data(), sigma, optimize_sigma, out);
}

int kb_warper_projection_axis(const kb_warper_table *t, int axis, double *sigma, double *xi, uint64_t *xi_count,
                              double *fn) {
  KB_CHECK(t, "null warper table");
  KB_CHECK(t->type == KB_TABLE_PROJECTION, "not a projection warper");
  KB_CHECK(axis >= 0 && axis < t->ndims, "this axis does not exist.");
  const size_t a = (size_t)axis;
  if (sigma) *sigma = t->sigmas[a];
  if (xi) std::copy(t->xi[a].begin(), t->xi[a].end(), xi);
  if (xi_count) std::copy(t->xi_count[a].begin(), t->xi_count[a].end(), xi_count);
  if (fn) std::copy(t->fn[a].begin(), t->fn[a].end(), fn);
  return KB_OK;
}

} // extern "C"
