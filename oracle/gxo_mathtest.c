/*
 * gxo_mathtest.c -- ORACLE (test infrastructure only): batch evaluation of
 * the parity build's elementary functions (gx_math.h) and of the C library's,
 * for the tests that bound the former's error and compare it bit for bit
 * with the same header compiled for the GPU.
 * fn: 0 log, 1 exp, 2 pow(x, y), 3 sin, 4 cos, 5 expm1, 6 log1p.
 */
#include <math.h>

#include "gx_math.h"

void gxo_gxm_eval(int fn, int n, const double *x, const double *y, double *out)
{
  for (int i = 0; i < n; ++i) {
    switch (fn) {
    case 0: out[i] = gxm_log(x[i]); break;
    case 1: out[i] = gxm_exp(x[i]); break;
    case 2: out[i] = gxm_pow(x[i], y[i]); break;
    case 3: out[i] = gxm_sin(x[i]); break;
    case 4: out[i] = gxm_cos(x[i]); break;
    case 5: out[i] = gxm_expm1(x[i]); break;
    default: out[i] = gxm_log1p(x[i]); break;
    }
  }
}

void gxo_libm_eval(int fn, int n, const double *x, const double *y, double *out)
{
  for (int i = 0; i < n; ++i) {
    switch (fn) {
    case 0: out[i] = log(x[i]); break;
    case 1: out[i] = exp(x[i]); break;
    case 2: out[i] = pow(x[i], y[i]); break;
    case 3: out[i] = sin(x[i]); break;
    case 4: out[i] = cos(x[i]); break;
    case 5: out[i] = expm1(x[i]); break;
    default: out[i] = log1p(x[i]); break;
    }
  }
}
