/* CBLAS declarations for the reference's pcgsolver/blas_wrapper.h and
 * src/math/RCMatrix.cpp (stride arguments, 0-based i?amax as in CBLAS).
 * Implemented in ../cblas_min.c with plain sequential loops. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor=101, CblasColMajor=102 };
float  cblas_sdot(int n, const float *x, int incx, const float *y, int incy);
double cblas_dsdot(int n, const float *x, int incx, const float *y, int incy);
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
float  cblas_snrm2(int n, const float *x, int incx);
double cblas_dnrm2(int n, const double *x, int incx);
float  cblas_sasum(int n, const float *x, int incx);
double cblas_dasum(int n, const double *x, int incx);
int    cblas_isamax(int n, const float *x, int incx);
int    cblas_idamax(int n, const double *x, int incx);
void   cblas_scopy(int n, const float *x, int incx, float *y, int incy);
void   cblas_dcopy(int n, const double *x, int incx, double *y, int incy);
void   cblas_saxpy(int n, float a, const float *x, int incx, float *y, int incy);
void   cblas_daxpy(int n, double a, const double *x, int incx, double *y, int incy);
void   cblas_sscal(int n, float a, float *x, int incx);
void   cblas_dscal(int n, double a, double *x, int incx);
void   cblas_sswap(int n, float *x, int incx, float *y, int incy);
void   cblas_dswap(int n, double *x, int incx, double *y, int incy);
#ifdef __cplusplus
}
#endif
