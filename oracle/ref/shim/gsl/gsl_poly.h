/* shim: the GSL declaration the reference's do_tracking.c includes (its
 * cubic solver serves an element outside the tracking path and is never
 * reached here) */
#ifndef ORACLE_REF_SHIM_GSL_POLY_H
#define ORACLE_REF_SHIM_GSL_POLY_H
int gsl_poly_solve_cubic(double a, double b, double c, double *x0, double *x1, double *x2);
#endif
