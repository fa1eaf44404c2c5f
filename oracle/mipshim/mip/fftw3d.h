/*
 * fftw3d.h -- project-written stand-in for MIP's complex 3D FFT.
 * TEST INFRASTRUCTURE ONLY (see miputil.h).
 *
 * invfft3d(p, nx, ny, nz): in-place inverse DFT (exp(+i...) kernel, scaled
 * by 1/(nx*ny*nz)) of nx*ny*nz complex values stored as interleaved
 * (re, im) float pairs, x fastest.
 */
#ifndef MIPSHIM_FFTW3D_H
#define MIPSHIM_FFTW3D_H

#ifdef __cplusplus
extern "C" {
#endif

void invfft3d(float *p, int nx, int ny, int nz);

#ifdef __cplusplus
}
#endif
#endif
