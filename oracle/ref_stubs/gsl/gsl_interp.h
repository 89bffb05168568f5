/* Stand-in declarations for GSL (test infrastructure; never called on the hot path). */
#pragma once
#include <cstddef>
struct gsl_interp_type;
struct gsl_interp_accel;
extern "C" {
extern const gsl_interp_type *gsl_interp_linear;
extern const gsl_interp_type *gsl_interp_steffen;
gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *);
size_t gsl_interp_accel_find(gsl_interp_accel *, const double *, size_t, double);
}
