/* Stand-in declarations for GSL (test infrastructure; never called on the hot path). */
#pragma once
#include <cstddef>
struct gsl_function {
  double (*function)(double x, void *params);
  void *params;
};
struct gsl_integration_workspace;
struct gsl_integration_qawo_table;
struct gsl_integration_qaws_table;
extern "C" {
gsl_integration_workspace *gsl_integration_workspace_alloc(size_t);
void gsl_integration_workspace_free(gsl_integration_workspace *);
int gsl_integration_qag(const gsl_function *, double, double, double, double, size_t, int,
                        gsl_integration_workspace *, double *, double *);
int gsl_integration_qags(const gsl_function *, double, double, double, double, size_t, gsl_integration_workspace *,
                         double *, double *);
int gsl_integration_qagp(const gsl_function *, double *, size_t, double, double, size_t, gsl_integration_workspace *,
                         double *, double *);
int gsl_integration_qagi(gsl_function *, double, double, size_t, gsl_integration_workspace *, double *, double *);
int gsl_integration_qagiu(gsl_function *, double, double, double, size_t, gsl_integration_workspace *, double *,
                          double *);
int gsl_integration_qagil(gsl_function *, double, double, double, size_t, gsl_integration_workspace *, double *,
                          double *);
}
