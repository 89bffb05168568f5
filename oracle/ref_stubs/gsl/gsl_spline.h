/* Stand-in declarations for GSL (test infrastructure; never called on the hot path). */
#pragma once
#include "gsl_interp.h"
struct gsl_spline;
extern "C" {
gsl_spline *gsl_spline_alloc(const gsl_interp_type *, size_t);
void gsl_spline_free(gsl_spline *);
int gsl_spline_init(gsl_spline *, const double *, const double *, size_t);
double gsl_spline_eval(const gsl_spline *, double, gsl_interp_accel *);
}
