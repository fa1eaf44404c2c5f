/*
 * dfft.h -- double-precision complex FFT used by the CPU oracle and by the
 * MIP shim.  TEST INFRASTRUCTURE ONLY: the product never links it.
 *
 * dfft_c1d() transforms n complex values in place (any n >= 1; radix-2
 * iterative for powers of two, recursive mixed radix otherwise) with
 * kernel exp(sign * 2*pi*i*j*k/n) and no scaling.
 */
#ifndef ORACLE_DFFT_H
#define ORACLE_DFFT_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

void dfft_c1d(double complex *x, int n, int sign);
/* strided variant: element j lives at x[j*stride] */
void dfft_c1d_strided(double complex *x, int n, int stride, int sign);
/* full complex 3D transform of an nx*ny*nz array (x fastest), unscaled */
void dfft_c3d(double complex *x, int nx, int ny, int nz, int sign);

#ifdef __cplusplus
}
#endif
#endif
