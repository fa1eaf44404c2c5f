/*
 * dfft.c -- double-precision complex FFT for the CPU oracle and the MIP
 * shim.  TEST INFRASTRUCTURE ONLY.
 *
 * Powers of two use an iterative radix-2 decimation-in-time transform with
 * twiddles evaluated directly by cos/sin (no recurrence), other lengths a
 * recursive Cooley-Tukey split on the smallest prime factor with a direct
 * DFT of that factor.  Accuracy is that of double arithmetic, far below the
 * float rounding of the data it is applied to.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dfft.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void fft_pow2(double complex *x, int n, int sign)
{
	int i, j, len;
	/* bit reversal permutation */
	for (i = 1, j = 0; i < n; ++i) {
		int bit = n >> 1;
		for (; j & bit; bit >>= 1)
			j ^= bit;
		j ^= bit;
		if (i < j) {
			double complex t = x[i];
			x[i] = x[j];
			x[j] = t;
		}
	}
	for (len = 2; len <= n; len <<= 1) {
		int half = len >> 1;
		for (j = 0; j < half; ++j) {
			double ang = sign * 2.0 * M_PI * (double)j / (double)len;
			double complex w = cos(ang) + I * sin(ang);
			for (i = j; i < n; i += len) {
				double complex u = x[i];
				double complex v = x[i + half] * w;
				x[i] = u + v;
				x[i + half] = u - v;
			}
		}
	}
}

static int smallest_factor(int n)
{
	int p;
	if (n % 2 == 0)
		return 2;
	for (p = 3; p * p <= n; p += 2)
		if (n % p == 0)
			return p;
	return n;
}

/* out[k*os] = sum_j in[j*is] exp(sign 2 pi i j k / n) */
static void fft_rec(const double complex *in, int is, double complex *out, int n, int sign)
{
	int p, m, r, k, q;
	double complex *tmp;
	if (n == 1) {
		out[0] = in[0];
		return;
	}
	p = smallest_factor(n);
	m = n / p;
	/* sub-transforms of the p decimated sequences, stored contiguously */
	tmp = (double complex *)malloc(sizeof(double complex) * n);
	for (r = 0; r < p; ++r)
		fft_rec(in + r * is, is * p, tmp + r * m, m, sign);
	for (k = 0; k < m; ++k) {
		double complex t[64];
		double complex *tt = p <= 64 ? t : (double complex *)malloc(sizeof(double complex) * p);
		for (r = 0; r < p; ++r) {
			double ang = sign * 2.0 * M_PI * (double)r * (double)k / (double)n;
			tt[r] = tmp[r * m + k] * (cos(ang) + I * sin(ang));
		}
		for (q = 0; q < p; ++q) {
			double complex s = 0;
			for (r = 0; r < p; ++r) {
				double ang = sign * 2.0 * M_PI * (double)((long)r * q % p) / (double)p;
				s += tt[r] * (cos(ang) + I * sin(ang));
			}
			out[k + q * m] = s;
		}
		if (tt != t)
			free(tt);
	}
	free(tmp);
}

void dfft_c1d(double complex *x, int n, int sign)
{
	double complex *out;
	if (n <= 1)
		return;
	if (is_pow2(n)) {
		fft_pow2(x, n, sign);
		return;
	}
	out = (double complex *)malloc(sizeof(double complex) * n);
	fft_rec(x, 1, out, n, sign);
	memcpy(x, out, sizeof(double complex) * n);
	free(out);
}

void dfft_c1d_strided(double complex *x, int n, int stride, int sign)
{
	int j;
	double complex *buf;
	if (stride == 1) {
		dfft_c1d(x, n, sign);
		return;
	}
	buf = (double complex *)malloc(sizeof(double complex) * n);
	for (j = 0; j < n; ++j)
		buf[j] = x[(long)j * stride];
	dfft_c1d(buf, n, sign);
	for (j = 0; j < n; ++j)
		x[(long)j * stride] = buf[j];
	free(buf);
}

void dfft_c3d(double complex *x, int nx, int ny, int nz, int sign)
{
	int i, j, k;
	for (k = 0; k < nz; ++k)
		for (j = 0; j < ny; ++j)
			dfft_c1d(x + ((long)k * ny + j) * nx, nx, sign);
	if (ny > 1)
		for (k = 0; k < nz; ++k)
			for (i = 0; i < nx; ++i)
				dfft_c1d_strided(x + (long)k * ny * nx + i, ny, nx, sign);
	if (nz > 1)
		for (j = 0; j < ny; ++j)
			for (i = 0; i < nx; ++i)
				dfft_c1d_strided(x + (long)j * nx + i, nz, nx * ny, sign);
}
