// Stand-in definitions of GSL's linear spline and lookup accelerator (test infrastructure
// only), so that keldy's warper_product_1d_simple_interp_nearest_t (product_1d_simple.hpp)
// runs in oracle/_ref. GSL's documented behaviour: gsl_interp_accel_find returns the
// index i of the interval x[i] <= v < x[i+1] (the last point belongs to the last interval);
// the linear spline interpolates between the interval's ends; evaluation outside the
// points is a domain error (NaN here). The Steffen spline is not provided.
#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <vector>

#include "gsl/gsl_spline.h"

struct gsl_interp_type {
  int id;
};
struct gsl_interp_accel {
  std::size_t cache;
};
struct gsl_spline {
  const gsl_interp_type *type;
  std::vector<double> x, y;
};

static const gsl_interp_type linear_type{0};
static const gsl_interp_type steffen_type{1};

extern "C" {
const gsl_interp_type *gsl_interp_linear = &linear_type;
const gsl_interp_type *gsl_interp_steffen = &steffen_type;

gsl_interp_accel *gsl_interp_accel_alloc(void) { return new gsl_interp_accel{0}; }
void gsl_interp_accel_free(gsl_interp_accel *a) { delete a; }

size_t gsl_interp_accel_find(gsl_interp_accel *a, const double *x, size_t n, double v) {
  size_t lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    const size_t m = (lo + hi) / 2;
    if (x[m] > v)
      hi = m;
    else
      lo = m;
  }
  if (a) a->cache = lo;
  return lo;
}

gsl_spline *gsl_spline_alloc(const gsl_interp_type *t, size_t) { return new gsl_spline{t, {}, {}}; }
void gsl_spline_free(gsl_spline *s) { delete s; }

int gsl_spline_init(gsl_spline *s, const double *x, const double *y, size_t n) {
  if (s->type != gsl_interp_linear) throw std::runtime_error("only the linear spline is provided by the stand-in");
  s->x.assign(x, x + n);
  s->y.assign(y, y + n);
  return 0;
}

double gsl_spline_eval(const gsl_spline *s, double v, gsl_interp_accel *a) {
  const size_t n = s->x.size();
  if (!(s->x[0] <= v && v <= s->x[n - 1])) return NAN;
  const size_t i = gsl_interp_accel_find(a, s->x.data(), n, v);
  const double dx = s->x[i + 1] - s->x[i];
  return dx > 0.0 ? s->y[i] + (v - s->x[i]) / dx * (s->y[i + 1] - s->y[i]) : s->y[i];
}
}
