/*
 * TEST INFRASTRUCTURE (oracle/ref): force-included into elegant's sources so
 * that their sin/cos/asin/tan/exp/sinh/cosh calls go through oracle/ref/shim_impl.c, which
 * can switch them to correctly rounded versions.  math.h is included first
 * so its own declarations keep the real names.
 */
#ifndef ORACLE_REF_SHIM_REFMATH_H
#define ORACLE_REF_SHIM_REFMATH_H
#include <math.h>
double ref_sin(double x);
double ref_cos(double x);
double ref_asin(double x);
double ref_tan(double x);
double ref_exp(double x);
double ref_sinh(double x);
double ref_cosh(double x);
#define sin(x) ref_sin(x)
#define cos(x) ref_cos(x)
#define asin(x) ref_asin(x)
#define tan(x) ref_tan(x)
#define exp(x) ref_exp(x)
#define sinh(x) ref_sinh(x)
#define cosh(x) ref_cosh(x)
#endif
