/* Minimal CBLAS for building the reference's solver sources on a machine
 * without a BLAS package. Plain sequential loops in index order; i?amax
 * returns the 0-based index of the first maximal |x_i| (CBLAS convention).
 * Only the entry points that pcgsolver/blas_wrapper.h and RCMatrix.cpp call. */
#include <math.h>
#include "shims/gsl/gsl_blas.h"

float cblas_sdot(int n, const float *x, int incx, const float *y, int incy)
{ float s = 0.f; for (int i = 0; i < n; ++i) s += x[i*incx]*y[i*incy]; return s; }
double cblas_dsdot(int n, const float *x, int incx, const float *y, int incy)
{ double s = 0.0; for (int i = 0; i < n; ++i) s += (double)x[i*incx]*(double)y[i*incy]; return s; }
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy)
{ double s = 0.0; for (int i = 0; i < n; ++i) s += x[i*incx]*y[i*incy]; return s; }
float cblas_snrm2(int n, const float *x, int incx)
{ double s = 0.0; for (int i = 0; i < n; ++i) s += (double)x[i*incx]*x[i*incx]; return (float)sqrt(s); }
double cblas_dnrm2(int n, const double *x, int incx)
{ double s = 0.0; for (int i = 0; i < n; ++i) s += x[i*incx]*x[i*incx]; return sqrt(s); }
float cblas_sasum(int n, const float *x, int incx)
{ float s = 0.f; for (int i = 0; i < n; ++i) s += fabsf(x[i*incx]); return s; }
double cblas_dasum(int n, const double *x, int incx)
{ double s = 0.0; for (int i = 0; i < n; ++i) s += fabs(x[i*incx]); return s; }
int cblas_isamax(int n, const float *x, int incx)
{ int k = 0; float m = -1.f; for (int i = 0; i < n; ++i) { float a = fabsf(x[i*incx]); if (a > m) { m = a; k = i; } } return k; }
int cblas_idamax(int n, const double *x, int incx)
{ int k = 0; double m = -1.0; for (int i = 0; i < n; ++i) { double a = fabs(x[i*incx]); if (a > m) { m = a; k = i; } } return k; }
void cblas_scopy(int n, const float *x, int incx, float *y, int incy)
{ for (int i = 0; i < n; ++i) y[i*incy] = x[i*incx]; }
void cblas_dcopy(int n, const double *x, int incx, double *y, int incy)
{ for (int i = 0; i < n; ++i) y[i*incy] = x[i*incx]; }
void cblas_saxpy(int n, float a, const float *x, int incx, float *y, int incy)
{ for (int i = 0; i < n; ++i) y[i*incy] += a*x[i*incx]; }
void cblas_daxpy(int n, double a, const double *x, int incx, double *y, int incy)
{ for (int i = 0; i < n; ++i) y[i*incy] += a*x[i*incx]; }
void cblas_sscal(int n, float a, float *x, int incx)
{ for (int i = 0; i < n; ++i) x[i*incx] *= a; }
void cblas_dscal(int n, double a, double *x, int incx)
{ for (int i = 0; i < n; ++i) x[i*incx] *= a; }
void cblas_sswap(int n, float *x, int incx, float *y, int incy)
{ for (int i = 0; i < n; ++i) { float t = x[i*incx]; x[i*incx] = y[i*incy]; y[i*incy] = t; } }
void cblas_dswap(int n, double *x, int incx, double *y, int incy)
{ for (int i = 0; i < n; ++i) { double t = x[i*incx]; x[i*incx] = y[i*incy]; y[i*incy] = t; } }
