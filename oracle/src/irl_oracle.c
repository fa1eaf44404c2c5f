/*
 * irl_oracle.c -- CPU restatement of libirl's OSEM projector/backprojector
 * path.  TEST INFRASTRUCTURE ONLY (see irl_oracle.h).
 *
 * Each function restates the libirl routine cited beside it.  Arithmetic
 * keeps libirl's operand types (float data, double literals and libm
 * calls) so that, compiled with gcc on x86-64, every non-FFT step rounds
 * exactly like the reference.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "dfft.h"
#include "irl_oracle.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define MAXF(a, b) ((a) > (b) ? (a) : (b))
#define MINF(a, b) ((a) < (b) ? (a) : (b))

/* ------------------------------------------------------------- threads */

/* Views of a subset (and of IrlGenprj) are independent until their
   backprojections are summed, so the restatement runs them on a pool of
   host threads; everything order-dependent (the clamped accumulation of
   prjbck.c:418-426, the EM update) stays serial, so the results do not
   depend on the thread count. */
static int g_threads = 1;

void or_set_threads(int n)
{
	g_threads = n < 1 ? 1 : n;
}

typedef struct {
	void (*fn)(void *ctx, int i);
	void *ctx;
	int count, next;
	pthread_mutex_t mu;
} par_job;

static void *par_worker(void *arg)
{
	par_job *j = (par_job *)arg;
	for (;;) {
		int i;
		pthread_mutex_lock(&j->mu);
		i = j->next++;
		pthread_mutex_unlock(&j->mu);
		if (i >= j->count)
			break;
		j->fn(j->ctx, i);
	}
	return NULL;
}

static void par_for(int count, void (*fn)(void *ctx, int i), void *ctx)
{
	int nt = MINF(g_threads, count), t, started = 0;
	pthread_t th[256];
	par_job j;
	if (nt > 256)
		nt = 256;
	if (nt <= 1) {
		for (t = 0; t < count; ++t)
			fn(ctx, t);
		return;
	}
	j.fn = fn;
	j.ctx = ctx;
	j.count = count;
	j.next = 0;
	pthread_mutex_init(&j.mu, NULL);
	for (t = 0; t < nt - 1; ++t)
		if (pthread_create(&th[started], NULL, par_worker, &j) == 0)
			++started;
	par_worker(&j);
	for (t = 0; t < started; ++t)
		pthread_join(th[t], NULL);
	pthread_mutex_destroy(&j.mu);
}

/* ------------------------------------------------------------ rotation */

/* circular support rows (fastrotate.c:573-589) */
static void support(int n, int *st, int *en)
{
	int j, len;
	float t, c = (n - 1) * 0.5;
	for (j = 0; j < n; j++) {
		t = ((float)j - c);
		len = 2 * floor(sqrt(c * c - t * t)) + 2;
		st[j] = (n - len) / 2;
		en[j] = st[j] + len;
	}
}

/* vShearsRotate (fastrotate.c:330-563): three 1D linear-interpolation
   shears per z-slice after reducing the angle to (-45, 45] degrees */
void or_shears_rotate(float fAngle, const float *in, float *out, int n, int nz)
{
	int b90 = 0, b180 = 0, i, j, k, iAdd, mDim, iT, jT, *st, *en;
	float c, tc, yd, xd, fd, f1, f2, *X, *Y;
#define IN(x, y, s) in[(size_t)(y) * nz * n + (size_t)(s) * n + (x)]
	/* a pass-1 tap outside the slice (x or y outside [0, n)) reads 0: for odd
	   n the middle row's last second tap lies one past the row
	   (fastrotate.c:400-488 reads that memory, and for the last row of the
	   last slice memory past the volume) with weight f2 = 0 exactly, so the
	   reference's result equals this one whenever that memory is finite */
#define TAP(x, y, s) (((x) < 0 || (x) >= n || (y) < 0 || (y) >= n) ? 0.f : IN(x, y, s))
	while (fAngle > 0.75 * M_PI) {
		fAngle -= M_PI;
		b180 = !b180;
	}
	while (fAngle <= -M_PI / 4.0) {
		fAngle += M_PI;
		b180 = !b180;
	}
	if (fAngle > M_PI / 4.0) {
		b90 = 1;
		fAngle -= M_PI / 2.0;
	}
	c = ((float)n - 1.0) * 0.5;
	iAdd = 0;
	for (j = n / 4; j < n / 2; j++) {
		yd = (float)j - c;
		fd = fabs(yd * tan((double)(fAngle * 0.5)));
		fd -= c - sqrt(c * c - yd * yd);
		iT = ceil(fd);
		if (iT > iAdd)
			iAdd = iT;
	}
	mDim = n + 2 * iAdd;
	tc = ((float)mDim - 1.0) * 0.5;
	st = (int *)malloc(sizeof(int) * n);
	en = (int *)malloc(sizeof(int) * n);
	support(n, st, en);
	X = (float *)calloc((size_t)mDim * mDim, sizeof(float));
	Y = (float *)calloc((size_t)mDim * mDim, sizeof(float));
	memset(out, 0, sizeof(float) * (size_t)n * nz * n);
	for (k = 0; k < nz; k++) {
		/* pass 1: x shear of every source row into X (fastrotate.c:400-488) */
		for (j = 0; j < n; j++) {
			int s0, s1, jj = n - j - 1;
			yd = (float)j - c;
			fd = -1.0 * yd * tan((double)(fAngle * 0.5));
			iT = floorf(fd);
			f2 = fd - (float)iT;
			f1 = 1.0 - f2;
			s0 = st[j] - iT + iAdd;
			s1 = en[j] - iT - 1 + iAdd;
			for (i = s0; i < s1; i++) {
				float a, b;
				if (!b180) {
					int t = i + iT - iAdd;
					if (!b90) {
						a = TAP(t, j, k);
						b = TAP(t + 1, j, k);
					} else {
						a = TAP(jj, t, k);
						b = TAP(jj, t + 1, k);
					}
				} else {
					int t = n - i - (iT - iAdd + 1);
					if (!b90) {
						a = TAP(t, jj, k);
						b = TAP(t - 1, jj, k);
					} else {
						a = TAP(j, t, k);
						b = TAP(j, t - 1, k);
					}
				}
				X[i + (size_t)mDim * (j + iAdd)] = f1 * a + f2 * b;
			}
		}
		/* pass 2: y shear (fastrotate.c:498-516) */
		for (i = 0; i < mDim; i++) {
			int js, je;
			xd = (float)i - tc;
			fd = xd * sin((double)(fAngle));
			jT = floorf(fd);
			f2 = fd - (float)jT;
			f1 = 1.0 - f2;
			js = MAXF(0, -jT);
			je = MINF(mDim, mDim - jT - 1);
			for (j = js; j < je; j++)
				Y[i + (size_t)mDim * j] = f1 * X[i + (size_t)mDim * (j + jT)] + f2 * X[i + (size_t)mDim * (j + jT + 1)];
		}
		/* pass 3: second x shear, one pixel inside the support (fastrotate.c:526-547) */
		for (j = 0; j < n; j++) {
			yd = (float)j - c;
			fd = -1.0 * yd * tan((double)(fAngle * 0.5));
			iT = floorf(fd);
			f2 = fd - (float)iT;
			f1 = 1.0 - f2;
			iT += iAdd;
			for (i = st[j] + 1; i < en[j] - 1; i++)
				out[(size_t)j * nz * n + (size_t)k * n + i] =
					f1 * Y[i + iT + (size_t)mDim * (j + iAdd)] + f2 * Y[i + iT + 1 + (size_t)mDim * (j + iAdd)];
		}
	}
#undef TAP
#undef IN
	free(X);
	free(Y);
	free(st);
	free(en);
}

/* rot3dpar (rot3dpar.c:19-198), NumPixels == NumRotPixs */
void or_rot3dpar(float fAngle, const float *in, float *out, int n, int nz)
{
	int s, X0, Y0, ox, oy, head, tail, np;
	float fx, fy, X, Y, z0, z1, z2, z3, z01, z23, z0123, ax, rad, sn, cs;
	int o0, o1, o2, o3;
	sn = (float)sin(fAngle);
	cs = (float)cos(fAngle);
	memset(out, 0, sizeof(float) * (size_t)n * nz * n);
	ax = 0.5 * (n - 1);
	rad = 0.5 * n;
	for (Y0 = 0; Y0 < n; Y0++) {
		Y = Y0 - ax;
		np = (int)(sqrt(rad * rad - (rad - Y0 - .5) * (rad - Y0 - .5)) + .5);
		np *= 2;
		head = (int)(0.5 * (n - np));
		tail = head + np - 1;
		for (X0 = head; X0 <= tail; X0++) {
			X = X0 - ax;
			fx = X * cs - Y * sn + ax;
			fy = X * sn + Y * cs + ax;
			ox = (int)fx;
			oy = (int)fy;
			o0 = o1 = o2 = o3 = 0;
			if (ox < 0 || ox >= n)
				o0 = o1 = 1;
			if (oy < 0 || oy >= n)
				o0 = o2 = 1;
			if (ox + 1 < 0 || ox + 1 >= n)
				o2 = o3 = 1;
			if (oy + 1 < 0 || oy + 1 >= n)
				o1 = o3 = 1;
			for (s = 0; s < nz; s++) {
				z0 = o0 ? 0.0f : in[(size_t)oy * nz * n + (size_t)s * n + ox];
				z1 = o1 ? 0.0f : in[(size_t)(oy + 1) * nz * n + (size_t)s * n + ox];
				z2 = o2 ? 0.0f : in[(size_t)oy * nz * n + (size_t)s * n + ox + 1];
				z3 = o3 ? 0.0f : in[(size_t)(oy + 1) * nz * n + (size_t)s * n + ox + 1];
				z01 = z0 + (fy - oy) * (z1 - z0);
				z23 = z2 + (fy - oy) * (z3 - z2);
				if (fy < 0) {
					z01 = z0;
					z23 = z2;
				}
				z0123 = z01 + (fx - ox) * (z23 - z01);
				if (fx < 0)
					z0123 = z01;
				out[(size_t)Y0 * nz * n + (size_t)s * n + X0] = z0123;
			}
		}
	}
}

static void rotate(const or_problem *P, float angle, const float *in, float *out)
{
	if (P->fast_rotate)
		or_shears_rotate(angle, in, out, P->n, P->nz);
	else
		or_rot3dpar(angle, in, out, P->n, P->nz);
}

/* ----------------------------------------------------------- DRF conv */

/* conv2d_ypad (conv2d_ypad.c:39-108) with pfPad2d, pfAvgRows, pfCopyRows
   (pad2d.c:21-141): x zero padding, y padding by averaged end rows */
void or_conv2d_ypad(const float *a, int nx, int ny, const float *b, int cx, int cy, int pady, int avgy, float *out)
{
	int W, H, x, y, bx, by, r;
	float *t;
	pady = MAXF(pady, 0);
	pady = MINF(pady, cy);
	avgy = MAXF(avgy, 0);
	avgy = MINF(avgy, ny);
	W = nx + 2 * cx;
	H = ny + 2 * pady;
	t = (float *)calloc((size_t)W * H, sizeof(float));
	for (y = 0; y < ny; y++)
		for (x = 0; x < nx; x++)
			t[(size_t)(y + pady) * W + x + cx] = a[(size_t)y * nx + x];
	if (avgy > 0 && pady > 0) {
		float *top = t, *bot = t + (size_t)(H - 1) * W;
		for (r = 0; r < avgy; r++)
			for (x = 0; x < W; x++)
				top[x] += t[(size_t)(pady + r) * W + x];
		if (avgy > 1)
			for (x = 0; x < W; x++)
				top[x] /= (float)avgy;
		for (r = 1; r < pady; r++)
			for (x = 0; x < W; x++)
				t[(size_t)r * W + x] += top[x];
		for (r = 0; r < avgy; r++)
			for (x = 0; x < W; x++)
				bot[x] += t[(size_t)(pady + ny - avgy + r) * W + x];
		if (avgy > 1)
			for (x = 0; x < W; x++)
				bot[x] /= (float)avgy;
		for (r = 0; r < pady - 1; r++)
			for (x = 0; x < W; x++)
				t[(size_t)(pady + ny + r) * W + x] += bot[x];
	}
	memset(out, 0, sizeof(float) * (size_t)nx * ny);
	for (by = -cy; by <= cy; by++)
		for (y = 0; y < ny; y++) {
			if (y - by + pady < 0 || y - by > ny + pady - 1)
				continue;
			for (bx = -cx; bx <= cx; bx++) {
				const float w = b[(size_t)(by + cy) * (2 * cx + 1) + bx + cx];
				const float *src = t + (size_t)(pady + y - by) * W + cx - bx;
				float *o = out + (size_t)y * nx;
				for (x = 0; x < nx; x++)
					o[x] += w * src[x];
			}
		}
	free(t);
}

/* DRF table index of a rotated row, or -1 (prjbck.c:187-203, 233) */
static int drf_index(float cfcr, float pix, int n, int row, float start, float spacing, int ndist)
{
	float fs = cfcr - pix * n / 2 + 0.5 * pix;
	float fd = fs + row * pix;
	int id = (int)floor((fd - start) / spacing + 0.5);
	id = MAXF(0, id);
	id = MINF(id, ndist - 1);
	return fd > 0.0 ? id : -1;
}

/* ---------------------------------------------------------------- ESSE */

/* pfReorder3dKrnl (krnlprj3d.c:43-128) and the weighted mean mu plus
   K*(mu - mu_avg) of pvInitScatterPrj (krnlprj3d.c:495-525) */
void or_esse_prepare(const float *krnl, const float *kmu, int noffs, int nd, int n, int nz, int c,
	float *gk, float *gkmu, float *mu_avg)
{
	int kx = (int)ceil(2.0f * (float)(n / c)), ky = kx, kz = (int)ceil(2.0f * (float)(nz / c));
	int xm = MINF(noffs, kx / 2), ym = MINF(noffs, kz / 2), iz, iy, ix, q;
	size_t cnt = (size_t)kx * ky * kz, i;
	float *mu = (float *)calloc(cnt, sizeof(float)), sk = 0.0f, skm = 0.0f;
	const float *src[2] = {krnl, kmu};
	float *dst[2] = {gk, mu};
	memset(gk, 0, sizeof(float) * cnt);
	for (q = 0; q < 2; ++q)
		for (iz = 0; iz < nd; ++iz) {
			int zo = ky / 2 - iz + nd / 2 - 1;
			if (zo < 0 || zo >= ky)
				continue;
			zo += zo < ky / 2 ? ky / 2 : -ky / 2;
			for (iy = 0; iy < ym; ++iy)
				for (ix = 0; ix < xm; ++ix) {
					float v = src[q][ix + noffs * (iy + noffs * iz)];
					int a, b;
					for (a = 0; a < (iy ? 2 : 1); ++a)
						for (b = 0; b < (ix ? 2 : 1); ++b)
							dst[q][(b ? kx - ix : ix) + (size_t)kx * ((a ? kz - iy : iy) + (size_t)kz * zo)] = v;
				}
		}
	for (i = 0; i < cnt; ++i) {
		sk += gk[i];
		skm += gk[i] * mu[i];
	}
	*mu_avg = sk == 0.0f ? 0.0f : skm / sk;
	for (i = 0; i < cnt; ++i) {
		mu[i] -= *mu_avg;
		gkmu[i] = mu[i] * gk[i];
	}
	free(mu);
}

/* exact circular convolution of a real [ky][kz][kx] grid with a real
   kernel grid (the realft3d / multrealft3d / realinvft3d chain) */
/* The kernel grids are the same for every view, so their spectra are
   computed once and kept (keyed by content, not only by address, since a
   later problem may reuse a freed address); the spectrum is the same
   deterministic transform either way. */
#define SPEC_CACHE 4
static struct {
	float *key;
	int kx, ky, kz;
	double complex *spec;
} g_spec[SPEC_CACHE];
static int g_spec_next;
static pthread_mutex_t g_spec_mu = PTHREAD_MUTEX_INITIALIZER;

static const double complex *kernel_spectrum(const float *k, int kx, int ky, int kz)
{
	size_t cnt = (size_t)kx * ky * kz, i;
	double complex *K;
	int e;
	pthread_mutex_lock(&g_spec_mu);
	for (e = 0; e < SPEC_CACHE; ++e)
		if (g_spec[e].key != NULL && g_spec[e].kx == kx && g_spec[e].ky == ky && g_spec[e].kz == kz &&
			memcmp(g_spec[e].key, k, sizeof(float) * cnt) == 0) {
			K = g_spec[e].spec;
			pthread_mutex_unlock(&g_spec_mu);
			return K;
		}
	K = (double complex *)malloc(sizeof(double complex) * cnt);
	for (i = 0; i < cnt; ++i)
		K[i] = k[i];
	dfft_c3d(K, kx, kz, ky, -1);
	e = g_spec_next;
	g_spec_next = (g_spec_next + 1) % SPEC_CACHE;
	/* an evicted entry may still be in use by another thread's convolution
	   only if more than SPEC_CACHE kernels are live at once; the oracle
	   never has more than two per problem and one problem at a time */
	free(g_spec[e].key);
	free(g_spec[e].spec);
	g_spec[e].key = (float *)malloc(sizeof(float) * cnt);
	memcpy(g_spec[e].key, k, sizeof(float) * cnt);
	g_spec[e].kx = kx;
	g_spec[e].ky = ky;
	g_spec[e].kz = kz;
	g_spec[e].spec = K;
	pthread_mutex_unlock(&g_spec_mu);
	return K;
}

static void circ_conv3(const float *a, const float *k, float *out, int kx, int ky, int kz)
{
	size_t cnt = (size_t)kx * ky * kz, i;
	double complex *A = (double complex *)malloc(sizeof(double complex) * cnt);
	const double complex *K = kernel_spectrum(k, kx, ky, kz);
	for (i = 0; i < cnt; ++i)
		A[i] = a[i];
	dfft_c3d(A, kx, kz, ky, -1);
	for (i = 0; i < cnt; ++i)
		A[i] *= K[i];
	dfft_c3d(A, kx, kz, ky, +1);
	for (i = 0; i < cnt; ++i)
		out[i] = (float)(creal(A[i]) / (double)cnt);
	free(A);
}

/* ExpandByFac (krnlprj3d.c:595-673): nearest expansion divided by c^3 and
   in-place (recursive) (2*(c/2)+1)-point smoothing along y, z, x */
static void expand(const float *g, int c, int n, int nz, float *img)
{
	int nx1 = n / c, nz1 = nz / c, h = c / 2, x, y, z, q;
#define IMG(x, y, z) img[(size_t)(y) * nz * n + (size_t)(z) * n + (x)]
	for (y = 0; y < n; ++y)
		for (z = 0; z < nz; ++z)
			for (x = 0; x < n; ++x)
				IMG(x, y, z) = g[(size_t)(y / c) * nz1 * nx1 + (size_t)(z / c) * nx1 + x / c] / c / c / c;
	for (y = h; y < n - h; ++y)
		for (z = 0; z < nz; ++z)
			for (x = 0; x < n; ++x) {
				float t = 0.0;
				for (q = y - h; q <= y + h; ++q)
					t += IMG(x, q, z);
				IMG(x, y, z) = t / (2 * h + 1);
			}
	for (z = h; z < nz - h; ++z)
		for (y = 0; y < n; ++y)
			for (x = 0; x < n; ++x) {
				float t = 0.0;
				for (q = z - h; q <= z + h; ++q)
					t += IMG(x, y, q);
				IMG(x, y, z) = t / (2 * h + 1);
			}
	for (x = h; x < n - h; ++x)
		for (y = 0; y < n; ++y)
			for (z = 0; z < nz; ++z) {
				float t = 0.0;
				for (q = x - h; q <= x + h; ++q)
					t += IMG(q, y, z);
				IMG(x, y, z) = t / (2 * h + 1);
			}
#undef IMG
}

/* CalcEffScatterSource (krnlprj3d.c:676-954) with two Taylor terms */
void or_esse_source(const or_problem *P, const float *act, const float *map, float *eff)
{
	int n = P->n, nz = P->nz, c = P->collapse, kx = P->kx, ky = P->ky, kz = P->kz;
	int n1 = n / c, nz1 = nz / c, x, y, z, t, k, j, i;
	size_t vox = (size_t)n * nz * n, cnt = (size_t)kx * ky * kz, e;
	float *grid = (float *)calloc(cnt, sizeof(float)), *res = (float *)malloc(sizeof(float) * cnt);
	float *g = (float *)malloc(sizeof(float) * (size_t)n1 * nz1 * n1);
	float *T[2];
	float *sum = (float *)calloc((size_t)nz * n, sizeof(float));
	float cnv = 1.0 / (P->mu0), fmu;
	T[0] = (float *)malloc(sizeof(float) * vox);
	T[1] = (float *)malloc(sizeof(float) * vox);
	/* CollapseByFac (sum pooling: y, then z, then x offsets), zero padded */
	for (y = 0; y < n1; ++y)
		for (z = 0; z < nz1; ++z)
			for (x = 0; x < n1; ++x) {
				float s = 0.0;
				for (k = 0; k < c; ++k)
					for (j = 0; j < c; ++j)
						for (i = 0; i < c; ++i)
							s += act[(size_t)(y * c + k) * nz * n + (size_t)(z * c + j) * n + x * c + i];
				grid[((size_t)y * kz + z) * kx + x] = s;
			}
	for (t = 0; t < P->nterms && t < 2; ++t) {
		circ_conv3(grid, t == 0 ? P->krnl : P->kmu, res, kx, ky, kz);
		for (y = 0; y < n1; ++y)
			for (z = 0; z < nz1; ++z)
				for (x = 0; x < n1; ++x)
					g[((size_t)y * nz1 + z) * n1 + x] = res[((size_t)y * kz + z) * kx + x];
		if (c != 1)
			expand(g, c, n, nz, T[t]);
		else
			memcpy(T[t], g, sizeof(float) * vox);
	}
	memcpy(eff, T[0], sizeof(float) * vox);
	if (P->nterms > 1) {
		for (y = 0; y < n; ++y) {
			for (e = 0; e < (size_t)nz * n; ++e)
				sum[e] += 0.5 * map[(size_t)y * nz * n + e];
			for (e = 0; e < (size_t)nz * n; ++e) {
				float d = sum[e] * cnv;
				eff[(size_t)y * nz * n + e] -= d * T[1][(size_t)y * nz * n + e];
			}
			for (e = 0; e < (size_t)nz * n; ++e)
				sum[e] += 0.5 * map[(size_t)y * nz * n + e];
		}
	}
	fmu = P->mu0 - P->mu_avg;
	memset(sum, 0, sizeof(float) * (size_t)nz * n);
	for (y = 0; y < n; ++y) {
		for (e = 0; e < (size_t)nz * n; ++e)
			sum[e] += 0.5 * map[(size_t)y * nz * n + e];
		for (e = 0; e < (size_t)nz * n; ++e) {
			float d = sum[e] * cnv;
			eff[(size_t)y * nz * n + e] *= exp(d * fmu);
		}
		for (e = 0; e < (size_t)nz * n; ++e)
			sum[e] += 0.5 * map[(size_t)y * nz * n + e];
	}
	if (P->cntr > 0)
		for (e = 0; e < vox; ++e)
			eff[e] += act[e] * P->cntr;
	cnv /= P->esse_pix;
	for (e = 0; e < vox; ++e) {
		eff[e] *= map[e] * cnv;
		if (eff[e] < 0)
			eff[e] = 0.0;
	}
	free(grid);
	free(res);
	free(g);
	free(T[0]);
	free(T[1]);
	free(sum);
}

/* ----------------------------------------------------- project / back */

static const float *psf_of(const or_problem *P, int bck, int id, int *mx, int *my)
{
	if (bck && P->bck_psf != NULL) {
		*mx = P->bck_mx[id];
		*my = P->bck_my[id];
		return P->bck_psf + P->bck_off[id];
	}
	*mx = P->mx[id];
	*my = P->my[id];
	return P->psf + P->psf_off[id];
}

/* Project (prjbck.c:68-252) with fAtnFac = 1 */
void or_project(const or_problem *P, int model, int view, const float *est, const float *atn, float primary,
	float *calc)
{
	int n = P->n, nz = P->nz, r, atnm = model & 1, drfm = model & 2, srfm = model & 4;
	size_t pl = (size_t)nz * n, vox = pl * n, i;
	float *rot = (float *)malloc(sizeof(float) * vox), *ratn = NULL, *src = rot;
	float *sumatn = (float *)calloc(pl, sizeof(float)), *plane = (float *)malloc(sizeof(float) * pl);
	float *conv = (float *)malloc(sizeof(float) * pl);
	float ang = 0.5 * M_PI + P->angle[view], scale = srfm ? 1.0 : primary;
	rotate(P, ang, est, rot);
	if (atnm || srfm) {
		ratn = (float *)malloc(sizeof(float) * vox);
		rotate(P, ang, atn, ratn);
	}
	if (srfm) {
		float *eff = (float *)malloc(sizeof(float) * vox);
		or_esse_source(P, rot, ratn, eff);
		for (i = 0; i < vox; ++i)
			eff[i] = rot[i] * primary + eff[i];
		src = eff;
	}
	memset(calc, 0, sizeof(float) * pl);
	for (r = 0; r < n; r++) {
		const float *pp = src + (size_t)r * pl;
		if (atnm || srfm)
			for (i = 0; i < pl; i++)
				sumatn[i] += (0.5 * ratn[(size_t)r * pl + i]);
		if (atnm) {
			for (i = 0; i < pl; i++)
				plane[i] = pp[i] * exp(-sumatn[i] * 1.0f);
			pp = plane;
		}
		if (drfm) {
			int id = drf_index(P->cfcr[view], P->pix, n, r, P->drf_start, P->drf_spacing, P->ndist), mx, my;
			if (id >= 0) {
				const float *b = psf_of(P, 0, id, &mx, &my);
				or_conv2d_ypad(pp, n, nz, b, mx - 1, my - 1, P->pad_len, P->avg_len, conv);
				pp = conv;
			}
		}
		for (i = 0; i < pl; i++)
			calc[i] += pp[i] * scale;
		if (atnm || srfm)
			for (i = 0; i < pl; i++)
				sumatn[i] += 0.5 * ratn[(size_t)r * pl + i];
	}
	if (src != rot)
		free(src);
	free(rot);
	free(ratn);
	free(sumatn);
	free(plane);
	free(conv);
}

/* BackProject (prjbck.c:254-427), fPrimaryFac = fAtnFac = 1, up to the
   unrotated volume un (the caller adds it to the image and clamps) */
static void backproject_view(const or_problem *P, int model, int view, const float *atn, const float *ratio,
	float *un)
{
	int n = P->n, nz = P->nz, r, atnm = model & 1, drfm = model & 2;
	size_t pl = (size_t)nz * n, vox = pl * n, i;
	float *ratn = NULL, *rot = (float *)malloc(sizeof(float) * vox);
	float *sumatn = (float *)calloc(pl, sizeof(float)), *plane = (float *)malloc(sizeof(float) * pl);
	float *conv = (float *)malloc(sizeof(float) * pl);
	const int bck = P->bck_psf != NULL;
	const int ndist = bck ? P->bck_ndist : P->ndist;
	const float start = bck ? P->bck_start : P->drf_start, spacing = bck ? P->bck_spacing : P->drf_spacing;
	if (atnm) {
		ratn = (float *)malloc(sizeof(float) * vox);
		rotate(P, 0.5 * M_PI + P->angle[view], atn, ratn);
	}
	for (r = 0; r < n; r++) {
		const float *pp = ratio;
		if (atnm) {
			for (i = 0; i < pl; i++)
				sumatn[i] += (0.5 * ratn[(size_t)r * pl + i]);
			for (i = 0; i < pl; i++)
				plane[i] = pp[i] * exp(-sumatn[i] * 1.0f);
			pp = plane;
		}
		if (drfm) {
			int id = drf_index(P->cfcr[view], P->pix, n, r, start, spacing, ndist), mx, my;
			if (id >= 0) {
				const float *b = psf_of(P, 1, id, &mx, &my);
				or_conv2d_ypad(pp, n, nz, b, mx - 1, my - 1, P->pad_len, P->avg_len, conv);
				pp = conv;
			}
		}
		for (i = 0; i < pl; i++)
			rot[(size_t)r * pl + i] = pp[i] * 1.0f;
		if (atnm)
			for (i = 0; i < pl; i++)
				sumatn[i] += (0.5 * ratn[(size_t)r * pl + i]);
	}
	rotate(P, -0.5 * M_PI - P->angle[view], rot, un);
	free(ratn);
	free(rot);
	free(sumatn);
	free(plane);
	free(conv);
}

/* image += un, then the clamp of prjbck.c:418-426 */
static void add_clamped(float *image, const float *un, size_t vox)
{
	size_t i;
	for (i = 0; i < vox; i++)
		image[i] += un[i];
	for (i = 0; i < vox; i++)
		if (image[i] < 1.0e-5)
			image[i] = 0.0;
}

void or_backproject(const or_problem *P, int model, int view, const float *atn, const float *ratio, float *image)
{
	size_t vox = (size_t)P->nz * P->n * P->n;
	float *un = (float *)malloc(sizeof(float) * vox);
	backproject_view(P, model, view, atn, ratio, un);
	add_clamped(image, un, vox);
	free(un);
}

/* IrlGenprj view loop (irlgenprj.c:225-264), the views on the thread pool */
typedef struct {
	const or_problem *P;
	int model;
	const float *act, *atn, *scatest;
	float primary, *prj;
} genprj_job;

static void genprj_view(void *ctx, int a)
{
	const genprj_job *g = (const genprj_job *)ctx;
	size_t pl = (size_t)g->P->nz * g->P->n, i;
	float *calc = g->prj + pl * a;
	or_project(g->P, g->model, a, g->act, g->atn, g->primary, calc);
	if (g->scatest != NULL)
		for (i = 0; i < pl; ++i)
			calc[i] += g->scatest[pl * a + i];
	for (i = 0; i < pl; ++i)
		calc[i] = calc[i] * g->P->view_time[a] * g->P->sens[a];
}

void or_genprj(const or_problem *P, int model, const float *act, const float *atn, const float *scatest,
	float primary, float *prj)
{
	size_t pl = (size_t)P->nz * P->n, i;
	genprj_job g = {P, model, act, atn, scatest, primary, prj};
	float s;
	par_for(P->nviews, genprj_view, &g);
	s = 1.0 / (float)P->nviews;
	for (i = 0; i < pl * P->nviews; ++i)
		prj[i] *= s;
}

/* measured-bin mask helpers (osemrecon.c:92-184) with PixelWidth = BinWidth */
static void set_measured_to_one(const or_problem *P, int v, const float *meas, float *out)
{
	int nb = P->n, nz = P->nz, ip, s, bl, br;
	float pl = P->left[v], pr;
	memset(out, 0, sizeof(float) * (size_t)nz * nb);
	for (ip = 0; ip < nb; ip++) {
		pr = pl + 1.0f;
		bl = floor((double)pl);
		br = floor((double)pr);
		if (bl > P->right[v])
			break;
		if (br > 0 && bl < nb)
			for (s = 0; s < nz; s++)
				if (meas[(size_t)s * nb + ip] >= 0.0)
					out[(size_t)s * nb + ip] = 1.0;
		pl = pr;
	}
}

static void zero_nonmeasured(const or_problem *P, int v, const float *meas0, float *calc)
{
	int nb = P->n, nz = P->nz, ip, s, bl, br;
	float pl = P->left[v], pr;
	for (ip = 0; ip < nb; ip++) {
		pr = pl + 1.0f;
		bl = floor((double)pl);
		br = floor((double)pr);
		for (s = 0; s < nz; s++)
			if (br <= 0 || bl >= nb || meas0[(size_t)s * nb + ip] < 0.0)
				calc[(size_t)s * nb + ip] = 0.0;
		pl = pr;
	}
}

/* one view of a subset: its backprojection un (not yet accumulated) */
typedef struct {
	const or_problem *P;
	int prj_model, bck_model, model, this_s, next_s, srf, s, ns, per;
	const float *meas, *atn, *scatest, *est;
	float *scat, *calc, *c2, *un;   /* calc, c2: per member planes; un: per member volumes */
	int norm_pass;
} subset_job;

static int subset_view(int s, int m, int ns)
{
	return s / 2 + (s % 2) * ns / 2 + m * ns;
}

static void subset_member(void *ctx, int m)
{
	const subset_job *j = (const subset_job *)ctx;
	const or_problem *P = j->P;
	size_t pl = (size_t)P->nz * P->n, vox = pl * P->n, i;
	int a = subset_view(j->s, m, j->ns);
	float *calc = j->calc + pl * m, *c2 = j->c2 + pl * m, *un = j->un + vox * m;
	if (j->norm_pass) {
		set_measured_to_one(P, a, j->meas + pl * a, calc);
		for (i = 0; i < pl; ++i)
			calc[i] *= P->view_time[a];
		backproject_view(P, j->bck_model, a, j->atn, calc, un);
		return;
	}
	or_project(P, j->model, a, j->est, j->atn, 1.0, calc);
	for (i = 0; i < pl; ++i)
		calc[i] *= P->view_time[a] * P->sens[a];
	if (j->srf) {
		if (!j->this_s) {
			for (i = 0; i < pl; ++i)
				calc[i] += j->scat[pl * a + i];
		} else if (!j->next_s) {
			or_project(P, j->prj_model & ~4, a, j->est, j->atn, 1.0, c2);
			for (i = 0; i < pl; ++i)
				c2[i] *= P->view_time[a];
			for (i = 0; i < pl; ++i)
				j->scat[pl * a + i] = calc[i] - c2[i];
		}
	}
	if (j->scatest != NULL)
		for (i = 0; i < pl; ++i)
			calc[i] += j->scatest[pl * a + i];
	zero_nonmeasured(P, a, j->meas, calc);
	for (i = 0; i < pl; ++i)
		calc[i] = calc[i] > 1e-20 ? j->meas[pl * a + i] / calc[i] : 0.0;
	for (i = 0; i < pl; ++i)
		calc[i] *= P->view_time[a];
	backproject_view(P, j->bck_model, a, j->atn, calc, un);
}

/* vOsemRecon (osemrecon.c:557-897) without hooks, norm images in memory.
   The members of a subset run on the thread pool; their backprojections
   are then added to the update image in member order with the clamp of
   prjbck.c:418-426, exactly as the serial loop does. */
int or_osem(const or_problem *P, int prj_model, int bck_model, int srf_iters, int iterations, int per,
	const float *meas, const float *atn, const float *scatest, float *est)
{
	int n = P->n, nz = P->nz, na = P->nviews, ns, s, m, it, srf = prj_model & 4, this_s = 0, next_s = 0;
	size_t pl = (size_t)nz * n, vox = pl * n, i;
	float *norm, *tmp, *scat = NULL;
	subset_job j;
	if (per <= 0 || na % per)
		return 1;
	ns = na / per;
	if (ns != 1 && ns % 2)
		return 2;
	norm = (float *)calloc(vox * ns, sizeof(float));
	tmp = (float *)malloc(sizeof(float) * vox);
	memset(&j, 0, sizeof(j));
	j.P = P;
	j.prj_model = prj_model;
	j.bck_model = bck_model;
	j.srf = srf;
	j.ns = ns;
	j.per = per;
	j.meas = meas;
	j.atn = atn;
	j.scatest = scatest;
	j.est = est;
	j.calc = (float *)malloc(sizeof(float) * pl * per);
	j.c2 = (float *)malloc(sizeof(float) * pl * per);
	j.un = (float *)malloc(sizeof(float) * vox * per);
	/* libirl allocates the stored scatter projections only when
	   iNumSrfIterations > 0 (osemrecon.c:610-615) but adds them whenever
	   scatter is not modelled in an iteration (osemrecon.c:743-745), a NULL
	   dereference for iNumSrfIterations = 0; here they start at zero */
	if (srf)
		scat = (float *)calloc(pl * na, sizeof(float));
	j.scat = scat;
	j.norm_pass = 1;
	for (s = 0; s < ns; ++s) {
		float *nm = norm + vox * s;
		j.s = s;
		par_for(per, subset_member, &j);
		for (m = 0; m < per; ++m)
			add_clamped(nm, j.un + vox * m, vox);
		for (i = 0; i < vox; ++i)
			nm[i] = nm[i] < 1e-6 ? 0.0 : 1.0 / nm[i];
	}
	j.norm_pass = 0;
	if (srf)
		next_s = 0 + 1 <= srf_iters;
	for (it = 1; it <= iterations; ++it) {
		int model = prj_model;
		if (srf) {
			this_s = next_s;
			next_s = (it == iterations) ? this_s : (it + 1 <= srf_iters);
			model = this_s ? prj_model : (prj_model & ~4);
		}
		j.model = model;
		j.this_s = this_s;
		j.next_s = next_s;
		for (s = 0; s < ns; ++s) {
			j.s = s;
			par_for(per, subset_member, &j);
			memset(tmp, 0, sizeof(float) * vox);
			for (m = 0; m < per; ++m)
				add_clamped(tmp, j.un + vox * m, vox);
			for (i = 0; i < vox; ++i)
				est[i] *= tmp[i] * norm[vox * s + i];
		}
	}
	free(norm);
	free(tmp);
	free(j.calc);
	free(j.c2);
	free(j.un);
	free(scat);
	return 0;
}

/* uniform initial estimate in the inscribed cylinder (initial_est.c:29-153,
   no contour or attenuation-map support) */
void or_initial_estimate(int n, int nz, int na, const float *prj, float *est)
{
	float fn = (float)(n * n * nz), sum = 0.0f, avg, rad = (float)n * 0.5, fx, fy;
	size_t i, tot = (size_t)n * nz * na;
	int r, c, s;
	fn *= M_PI / 4.0;
	for (i = 0; i < tot; ++i)
		sum += prj[i];
	avg = sum / (fn * na);
	for (i = 0; i < (size_t)n * nz * n; ++i)
		est[i] = avg;
	for (r = 0; r < n; ++r) {
		fy = (float)r - rad;
		if (fy > 0)
			fy += 1;
		for (c = 0; c < n; ++c) {
			fx = (float)c - rad;
			if (fx > 0)
				fx += 1;
			if (hypot(fx, fy) > rad)
				for (s = 0; s < nz; ++s)
					est[(size_t)r * nz * n + (size_t)s * n + c] = 0.0;
		}
	}
}
