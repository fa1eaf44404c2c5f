/*
 * mipshim.c -- project-written implementation of the MIP library routines
 * that libirl calls (utility, error, message and FFT routines).
 *
 * TEST INFRASTRUCTURE ONLY.  It is linked with the unmodified reference C
 * sources to form the CPU oracle oracle/_ref/libirl_ref.so.  The contract
 * of each routine is inferred from its libirl call sites; see the headers
 * in mip/ for the details, in particular the real-FFT packing.
 */
#include <complex.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <setjmp.h>

#include "mip/miputil.h"
#include "mip/errdefs.h"
#include "mip/printmsg.h"
#include "mip/realft.h"
#include "mip/fftw3d.h"
#include "../src/dfft.h"

/* ---------------------------------------------------------------- errors */

static jmp_buf *g_psTrap = NULL;
static FILE *g_fpErrLog = NULL;
static char g_pchErrMsg[1024] = "";

void vTrapFatalErrs(jmp_buf *psEnv) { g_psTrap = psEnv; }
char *pchErrorMsg(void) { return g_pchErrMsg; }
void vSetErrLog(FILE *fp) { g_fpErrLog = fp; }

void vErrorHandler(int iClass, int iType, char *pchRoutine, char *pchFmt, ...)
{
	va_list ap;
	char body[900];
	va_start(ap, pchFmt);
	vsnprintf(body, sizeof(body), pchFmt, ap);
	va_end(ap);
	if (iClass == ECLASS_FATAL) {
		snprintf(g_pchErrMsg, sizeof(g_pchErrMsg), "%s: %s", pchRoutine, body);
		if (g_fpErrLog != NULL)
			fprintf(g_fpErrLog, "FATAL %s\n", g_pchErrMsg);
		if (g_psTrap != NULL)
			longjmp(*g_psTrap, iType > 0 ? iType : 1);
		fprintf(stderr, "untrapped fatal error: %s\n", g_pchErrMsg);
		abort();
	}
	if (g_fpErrLog != NULL)
		fprintf(g_fpErrLog, "%s %s: %s\n", iClass == ECLASS_WARN ? "WARNING" : "INFO",
			pchRoutine, body);
}

/* -------------------------------------------------------------- messages */

static int g_iMsgLevel = 0;
static FILE *g_fpMsg = NULL;

void vSetMsgLevel(int iLevel) { g_iMsgLevel = iLevel; }
void vSetAllMsgFilePtr(FILE *fp) { g_fpMsg = fp; }

void vPrintMsg(int iLevel, char *pchFmt, ...)
{
	va_list ap;
	if (g_fpMsg == NULL || iLevel > g_iMsgLevel)
		return;
	va_start(ap, pchFmt);
	vfprintf(g_fpMsg, pchFmt, ap);
	va_end(ap);
}

void PrintTimes(char *label) { vPrintMsg(5, "%s\n", label); }

/* ---------------------------------------------------------------- memory */

void *pvIrlMalloc(size_t n, char *name)
{
	void *p = malloc(n > 0 ? n : 1);
	if (p == NULL)
		vErrorHandler(ECLASS_FATAL, ETYPE_MALLOC, "pvIrlMalloc", "out of memory for %s", name);
	return p;
}

void *pvIrlRealloc(void *p, size_t n, char *name)
{
	void *q = realloc(p, n > 0 ? n : 1);
	if (q == NULL)
		vErrorHandler(ECLASS_FATAL, ETYPE_MALLOC, "pvIrlRealloc", "out of memory for %s", name);
	return q;
}

void IrlFree(void *p) { free(p); }
void vFreeAllMem(void) {}

char *pchIrlStrdup(char *s)
{
	size_t n = strlen(s) + 1;
	char *p = (char *)pvIrlMalloc(n, "strdup");
	memcpy(p, s, n);
	return p;
}

float *vector(int n, char *name) { return (float *)pvIrlMalloc(sizeof(float) * (size_t)(n > 0 ? n : 1), name); }
int *ivector(int n, char *name) { return (int *)pvIrlMalloc(sizeof(int) * (size_t)(n > 0 ? n : 1), name); }
void free_vector(void *p) { free(p); }

/* ---------------------------------------------------------- array helpers */

void set_float(float *p, int n, float v)
{
	int i;
	for (i = 0; i < n; ++i)
		p[i] = v;
}

float sum_float(float *p, int n)
{
	int i;
	float s = 0.0f;
	for (i = 0; i < n; ++i)
		s += p[i];
	return s;
}

void scale_float(float *p, int n, float s)
{
	int i;
	for (i = 0; i < n; ++i)
		p[i] *= s;
}

void vZeroNeg(float *p, int n)
{
	int i;
	for (i = 0; i < n; ++i)
		if (p[i] < 0.0f)
			p[i] = 0.0f;
}

float *reorder(int d0, int d1, int d2, float *in, float *out)
{
	int i, j, k;
	if (out == NULL)
		out = vector(d0 * d1 * d2, "reorder");
	for (j = 0; j < d1; ++j)
		for (k = 0; k < d0; ++k)
			for (i = 0; i < d2; ++i)
				out[((long)j * d0 + k) * d2 + i] = in[((long)k * d1 + j) * d2 + i];
	return out;
}

void vSwapWords(void *p, int n)
{
	unsigned char *b = (unsigned char *)p;
	int i;
	for (i = 0; i < n; ++i, b += 4) {
		unsigned char t0 = b[0], t1 = b[1];
		b[0] = b[3];
		b[1] = b[2];
		b[2] = t1;
		b[3] = t0;
	}
}

/* ------------------------------------------------------------------- FFT */

/* x-direction half spectrum of every row: H[row][kx], kx = 0..nx/2 */
static double complex *rows_forward(const float *p, int nx, int nrows)
{
	int h = nx / 2 + 1, r, i;
	double complex *H = (double complex *)malloc(sizeof(double complex) * (size_t)h * nrows);
	double complex *buf = (double complex *)malloc(sizeof(double complex) * nx);
	for (r = 0; r < nrows; ++r) {
		for (i = 0; i < nx; ++i)
			buf[i] = p[(long)r * nx + i];
		dfft_c1d(buf, nx, -1);
		for (i = 0; i < h; ++i)
			H[(long)r * h + i] = buf[i];
	}
	free(buf);
	return H;
}

/* inverse of rows_forward (unscaled), writing real rows into p */
static void rows_inverse(double complex *H, float *p, int nx, int nrows, double scale)
{
	int h = nx / 2 + 1, r, i;
	double complex *buf = (double complex *)malloc(sizeof(double complex) * nx);
	for (r = 0; r < nrows; ++r) {
		for (i = 0; i < h; ++i)
			buf[i] = H[(long)r * h + i];
		for (i = h; i < nx; ++i)
			buf[i] = conj(H[(long)r * h + (nx - i)]);
		dfft_c1d(buf, nx, +1);
		for (i = 0; i < nx; ++i)
			p[(long)r * nx + i] = (float)(creal(buf[i]) * scale);
	}
	free(buf);
}

/* transform along y and z of the half spectrum H[z][y][kx] for kx in [k0,k1) */
static void yz_transform(double complex *H, int h, int ny, int nz, int k0, int k1, int sign)
{
	int kx, y, z;
	for (kx = k0; kx < k1; ++kx) {
		if (ny > 1)
			for (z = 0; z < nz; ++z)
				dfft_c1d_strided(H + (long)z * ny * h + kx, ny, h, sign);
		if (nz > 1)
			for (y = 0; y < ny; ++y)
				dfft_c1d_strided(H + (long)y * h + kx, nz, h * ny, sign);
	}
}

void realft3d(float *p, int nx, int ny, int nz)
{
	int h = nx / 2 + 1, nrows = ny * nz, y, z, kx;
	double complex *H = rows_forward(p, nx, nrows);
	double complex *Z = (double complex *)malloc(sizeof(double complex) * nrows);
	yz_transform(H, h, ny, nz, 1, nx / 2, -1);
	/* joint transform of the two real columns d + i q */
	for (z = 0; z < nz; ++z)
		for (y = 0; y < ny; ++y) {
			long r = (long)z * ny + y;
			Z[r] = creal(H[r * h]) + I * creal(H[r * h + nx / 2]);
		}
	dfft_c3d(Z, ny, nz, 1, -1);
	for (z = 0; z < nz; ++z)
		for (y = 0; y < ny; ++y) {
			long r = (long)z * ny + y;
			for (kx = 1; kx < nx / 2; ++kx) {
				p[r * nx + 2 * kx] = (float)creal(H[r * h + kx]);
				p[r * nx + 2 * kx + 1] = (float)cimag(H[r * h + kx]);
			}
		}
	if (nz > 1) {
		for (z = 0; z < nz; ++z)
			for (y = 0; y < ny; ++y) {
				long r = (long)z * ny + y;
				p[r * nx] = (float)creal(Z[r]);
				p[r * nx + 1] = (float)cimag(Z[r]);
			}
	} else {
		/* separate D (x-DC column) and Q (x-Nyquist column) spectra along y */
		for (y = 0; y <= ny / 2; ++y) {
			double complex zk = Z[y], zm = conj(Z[(ny - y) % ny]);
			double complex D = 0.5 * (zk + zm), Q = -0.5 * I * (zk - zm);
			if (y == 0 || y == ny / 2) {
				p[(long)y * nx] = (float)creal(D);
				p[(long)y * nx + 1] = (float)creal(Q);
			} else {
				p[(long)y * nx] = (float)creal(D);
				p[(long)y * nx + 1] = (float)cimag(D);
				p[(long)(y + ny / 2) * nx] = (float)creal(Q);
				p[(long)(y + ny / 2) * nx + 1] = (float)cimag(Q);
			}
		}
	}
	free(Z);
	free(H);
}

void realinvft3d(float *p, int nx, int ny, int nz)
{
	int h = nx / 2 + 1, nrows = ny * nz, y, z, kx;
	double complex *H = (double complex *)malloc(sizeof(double complex) * (size_t)h * nrows);
	double complex *Z = (double complex *)malloc(sizeof(double complex) * nrows);
	for (z = 0; z < nz; ++z)
		for (y = 0; y < ny; ++y) {
			long r = (long)z * ny + y;
			for (kx = 1; kx < nx / 2; ++kx)
				H[r * h + kx] = p[r * nx + 2 * kx] + I * p[r * nx + 2 * kx + 1];
		}
	if (nz > 1) {
		for (z = 0; z < nz; ++z)
			for (y = 0; y < ny; ++y) {
				long r = (long)z * ny + y;
				Z[r] = p[r * nx] + I * p[r * nx + 1];
			}
	} else {
		for (y = 0; y < ny; ++y) {
			double complex D, Q;
			int yy = y <= ny / 2 ? y : ny - y; /* conjugate partner row */
			if (yy == 0 || yy == ny / 2) {
				D = p[(long)yy * nx];
				Q = p[(long)yy * nx + 1];
			} else {
				D = p[(long)yy * nx] + I * p[(long)yy * nx + 1];
				Q = p[(long)(yy + ny / 2) * nx] + I * p[(long)(yy + ny / 2) * nx + 1];
				if (yy != y) {
					D = conj(D);
					Q = conj(Q);
				}
			}
			Z[y] = D + I * Q;
		}
	}
	dfft_c3d(Z, ny, nz, 1, +1);
	yz_transform(H, h, ny, nz, 1, nx / 2, +1);
	for (z = 0; z < nz; ++z)
		for (y = 0; y < ny; ++y) {
			long r = (long)z * ny + y;
			H[r * h] = creal(Z[r]);
			H[r * h + nx / 2] = cimag(Z[r]);
		}
	rows_inverse(H, p, nx, nrows, 1.0 / ((double)nx * ny * nz));
	free(Z);
	free(H);
}

void multrealft3d(int nx, int ny, int nz, float *a, float *b, float *out)
{
	long n = (long)nx * ny * nz, r;
	int y, z;
	if (nz == 1) {
		/* identical to the 2D element-wise layout product */
		float f1 = a[(ny / 2) * nx] * b[(ny / 2) * nx];
		float f2 = a[(ny / 2) * nx + 1] * b[(ny / 2) * nx + 1];
		float o0 = a[0] * b[0], o1 = a[1] * b[1];
		long i;
		for (i = 2; i < n; i += 2) {
			float re = a[i] * b[i] - a[i + 1] * b[i + 1];
			float im = a[i] * b[i + 1] + a[i + 1] * b[i];
			out[i] = re;
			out[i + 1] = im;
		}
		out[0] = o0;
		out[1] = o1;
		out[(ny / 2) * nx] = f1;
		out[(ny / 2) * nx + 1] = f2;
		return;
	}
	{
		long nrows = (long)ny * nz;
		double complex *za = (double complex *)malloc(sizeof(double complex) * nrows);
		double complex *zb = (double complex *)malloc(sizeof(double complex) * nrows);
		for (r = 0; r < nrows; ++r) {
			za[r] = a[r * nx] + I * a[r * nx + 1];
			zb[r] = b[r * nx] + I * b[r * nx + 1];
		}
		for (r = 0; r < nrows; ++r) {
			int kx;
			for (kx = 1; kx < nx / 2; ++kx) {
				long i = r * nx + 2 * kx;
				double ar = a[i], ai = a[i + 1], br = b[i], bi = b[i + 1];
				out[i] = (float)(ar * br - ai * bi);
				out[i + 1] = (float)(ar * bi + ai * br);
			}
		}
		for (z = 0; z < nz; ++z)
			for (y = 0; y < ny; ++y) {
				long k = (long)z * ny + y;
				long m = (long)((nz - z) % nz) * ny + (ny - y) % ny;
				double complex Da = 0.5 * (za[k] + conj(za[m]));
				double complex Qa = -0.5 * I * (za[k] - conj(za[m]));
				double complex Db = 0.5 * (zb[k] + conj(zb[m]));
				double complex Qb = -0.5 * I * (zb[k] - conj(zb[m]));
				double complex zo = Da * Db + I * (Qa * Qb);
				out[k * nx] = (float)creal(zo);
				out[k * nx + 1] = (float)cimag(zo);
			}
		free(za);
		free(zb);
	}
}

void realft_free(void) {}

void invfft3d(float *p, int nx, int ny, int nz)
{
	long n = (long)nx * ny * nz, i;
	double complex *x = (double complex *)malloc(sizeof(double complex) * n);
	for (i = 0; i < n; ++i)
		x[i] = p[2 * i] + I * p[2 * i + 1];
	dfft_c3d(x, nx, ny, nz, +1);
	for (i = 0; i < n; ++i) {
		p[2 * i] = (float)(creal(x[i]) / (double)n);
		p[2 * i + 1] = (float)(cimag(x[i]) / (double)n);
	}
	free(x);
}
