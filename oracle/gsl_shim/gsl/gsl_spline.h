/* Project-written stand-in declarations (TEST INFRASTRUCTURE ONLY).  Only the
   types and calls that the reference's orbit drivers name are declared; the
   potentials this build integrates never reach a spline, and the definitions
   in oracle/gsl_shim/gsl_shim.c abort if one is ever called. */
#ifndef ORACLE_SHIM_GSL_SPLINE_H
#define ORACLE_SHIM_GSL_SPLINE_H
#include <stddef.h>
typedef struct oracle_shim_accel gsl_interp_accel;
typedef struct oracle_shim_spline gsl_spline;
typedef struct oracle_shim_interp_type gsl_interp_type;
extern const gsl_interp_type *gsl_interp_cspline;
gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size);
void gsl_spline_free(gsl_spline *s);
int gsl_spline_init(gsl_spline *s, const double xa[], const double ya[], size_t size);
double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a);
double gsl_spline_eval_deriv(const gsl_spline *s, double x, gsl_interp_accel *a);
#endif
