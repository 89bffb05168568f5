/* Stand-in declarations for GSL (test infrastructure; never called on the hot path). */
#pragma once
#define GSL_EROUND 18
#define GSL_EMAXITER 11
extern "C" const char *gsl_strerror(int);
typedef void gsl_error_handler_t(const char *, const char *, int, int);
extern "C" gsl_error_handler_t *gsl_set_error_handler_off(void);
extern "C" gsl_error_handler_t *gsl_set_error_handler(gsl_error_handler_t *);
