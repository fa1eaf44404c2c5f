/*
 * realft.h -- project-written stand-in for MIP's in-place real 3D FFT.
 * TEST INFRASTRUCTURE ONLY (see miputil.h).
 *
 * realft3d(p, nx, ny, nz) replaces the nx*ny*nz real samples in p (x
 * fastest) by their forward DFT packed into the same nx*ny*nz floats;
 * realinvft3d() inverts it, including the 1/(nx*ny*nz) factor, so that
 * forward -> multrealft3d -> inverse is exactly a circular convolution.
 *
 * Packing (nx, ny even):
 *  - for 1 <= kx < nx/2 the pair (p[2kx], p[2kx+1]) of row (y, z) holds
 *    bin (kx, ky=y, kz=z) of the full spectrum;
 *  - the two real x-columns (x-frequency 0 and nx/2) are stored in floats
 *    0 and 1 of each row.  For nz == 1 this follows the layout that
 *    libirl's multrealft2d() (conv2dPsfFFT.c) multiplies element-wise:
 *    rows 0 and ny/2 hold the four purely real bins, rows 1..ny/2-1 hold
 *    the x-DC column's bins ky = row, and rows ny/2+1..ny-1 hold the
 *    x-Nyquist column's bins ky = row - ny/2.  For nz > 1 the two real
 *    (y,z) planes are combined as d + i*q and their joint 2D DFT is stored
 *    (multrealft3d separates them again before multiplying).
 */
#ifndef MIPSHIM_REALFT_H
#define MIPSHIM_REALFT_H

#ifdef __cplusplus
extern "C" {
#endif

void realft3d(float *p, int nx, int ny, int nz);
void realinvft3d(float *p, int nx, int ny, int nz);
void multrealft3d(int nx, int ny, int nz, float *a, float *b, float *out);
void realft_free(void);

#ifdef __cplusplus
}
#endif
#endif
