/*
 * irl_grf.c -- geometric response (GRF) tables of a parallel-hole
 * collimator: libirl's gendrf (gendrf.c:44-427), which IrlSetup uses when
 * no DRF table file is given, or for the backprojector when bUseGrfInBck
 * is set (IrlSetup.c:243-334, 514-588).
 *
 * The response model is the published one that gendrf evaluates.  At
 * source distance d, with hole diameter D, hole length L and a gap g
 * behind the collimator, the transfer function at spatial frequency f is
 *
 *   H(f) = [2 J1(b f) / (b f)]^2  exp(-(pi F f)^2 / (4 ln 2))  sinc(pi w f)
 *
 * where b = pi D (d + g + L) / L, F is the intrinsic FWHM and w the bin
 * width (the sinc is the bin's own blur).  The point-spread function is H's
 * inverse 2D Fourier transform.  This file computes it as follows:
 *
 *   1. H is sampled on a square frequency grid of side S (a power of two,
 *      enough for 4 x the response's radius D (d + g + L) / L, at most
 *      1024) over a fine spatial bin w / r.  The oversampling r keeps b f
 *      near 10 at the fine Nyquist frequency.  The samples are stored as
 *      float, as gendrf stores them.
 *   2. Because H is even in both axes, its inverse transform is a real,
 *      separable cosine sum.  Each sum over S frequencies folds to S/2 + 1
 *      terms.  Only the first quadrant at the decimated points (every r-th
 *      fine sample) is needed, so it is evaluated there directly in double,
 *      with the angles reduced exactly (k = u x mod S).  The results are
 *      rounded to float, as gendrf's transform output is.
 *   3. Negative samples are set to 0.  The decimated quadrant is normalised
 *      by the sum of the mirrored decimated grid.  A square of
 *      half-width m is then kept: the smallest m whose enclosed sum exceeds
 *      1 - max_err, found from ring sums.  That square is renormalised and
 *      mirrored into the (2m-1)^2 PSF.
 *
 * gendrf does step 2 with a complex 2D FFT over the whole S x S grid and
 * step 3 with incremental sums.  Both give the same values up to the last
 * bits of double rounding, well below the float storage.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "irl_err.h"
#include "irl_host.h"

/* sampling of one distance's transfer function */
typedef struct {
	int ratio;      /* fine bins per output bin */
	int side;       /* frequency grid side (power of two) */
	int lim;        /* fine samples kept per axis: min(side/2, ratio * noffs) */
	int aliased;    /* the grid is wider than twice the table */
	double b;       /* Bessel argument per unit frequency */
	double gauss;   /* Gaussian exponent per unit frequency squared */
	double sinc;    /* sinc argument per unit frequency */
	double df;      /* frequency step */
} grf_grid;

static grf_grid grf_plan(double dist, double thick, double gap, double hole, double bin, double fwhm, int noffs)
{
	grf_grid g;
	const double spread = (dist + gap + thick) / thick;   /* magnification of the hole aperture */
	const double radius = hole * (dist + gap + thick) / thick;  /* where the geometric response ends */
	int need;
	g.b = M_PI * spread * hole;
	g.gauss = M_PI * M_PI * fwhm * fwhm / (4.0 * log(2.0));
	g.sinc = M_PI * bin;
	g.ratio = (int)(20.0 * bin / g.b + 0.5);
	if (g.ratio < 1)
		g.ratio = 1;
	need = (int)(4.0 * radius / (bin / g.ratio));
	for (g.side = 2; g.side < need && g.side < 1024; g.side <<= 1)
		;
	g.df = 1.0 / ((double)g.side * (bin / g.ratio));
	g.lim = g.side / 2 < g.ratio * noffs ? g.side / 2 : g.ratio * noffs;
	g.aliased = g.side > 2 * noffs;
	return g;
}

/* H at the frequency of grid point (u, v), 0 <= u, v <= side/2, as float */
static float grf_mtf(const grf_grid *g, int u, int v)
{
	double f, a, h;
	if (u == 0 && v == 0)
		return 1.0f;
	f = hypot((double)v * g->df, (double)u * g->df);
	a = g->b * f;
	h = 2.0 * j1(a) / a;
	h = h * h * exp(-f * f * g->gauss);
	if (g->sinc > 0.0)
		h *= sin(g->sinc * f) / (f * g->sinc);
	return (float)h;
}

/* decimated first quadrant of the PSF, q[j * noffs + i] = psf(i r, j r),
   normalised over the mirrored decimated grid; entries past lim are 0 */
static void grf_quadrant(const grf_grid *g, int noffs, float *q)
{
	const int S = g->side, H2 = S / 2, r = g->ratio;
	const int nd = (g->lim + r - 1) / r;   /* decimated samples per axis */
	double *cs = (double *)irl_malloc(sizeof(double) * S, "GRF cosines");
	float *mtf = (float *)irl_malloc(sizeof(float) * (size_t)(H2 + 1) * (H2 + 1), "GRF spectrum");
	double *half = (double *)irl_malloc(sizeof(double) * (size_t)(H2 + 1) * nd, "GRF half transform");
	float *p = (float *)irl_malloc(sizeof(float) * (size_t)nd * nd, "GRF quadrant");
	double norm;
	int i, j, u, v;
	for (u = 0; u < S; ++u)
		cs[u] = cos(2.0 * M_PI * (double)u / (double)S);
	for (v = 0; v <= H2; ++v)
		for (u = 0; u <= H2; ++u)
			mtf[(size_t)v * (H2 + 1) + u] = grf_mtf(g, u, v);
	/* x transform: half[v][i] = sum over all S frequencies u of H(u, v)
	   cos(2 pi u x / S) at x = i r, folded over u <-> S - u */
	for (v = 0; v <= H2; ++v)
		for (i = 0; i < nd; ++i) {
			const float *row = mtf + (size_t)v * (H2 + 1);
			const long x = (long)i * r;
			double s = row[0] + ((x & 1) ? -1.0 : 1.0) * row[H2];
			for (u = 1; u < H2; ++u)
				s += 2.0 * row[u] * cs[(x * u) % S];
			half[(size_t)v * nd + i] = s;
		}
	/* y transform at y = j r, then float rounding and the clip at 0 */
	for (j = 0; j < nd; ++j) {
		const long y = (long)j * r;
		for (i = 0; i < nd; ++i) {
			double s = half[i] + ((y & 1) ? -1.0 : 1.0) * half[(size_t)H2 * nd + i];
			float t;
			for (v = 1; v < H2; ++v)
				s += 2.0 * half[(size_t)v * nd + i] * cs[(y * v) % S];
			t = (float)(s / ((double)S * S));
			p[(size_t)j * nd + i] = t < 0.0f ? 0.0f : t;
		}
	}
	/* unit sum over the mirrored decimated grid: the centre once, the axes
	   twice, the rest four times */
	norm = p[0];
	for (i = 1; i < nd; ++i)
		norm += 2.0 * ((double)p[i] + (double)p[(size_t)i * nd]);
	for (j = 1; j < nd; ++j)
		for (i = 1; i < nd; ++i)
			norm += 4.0 * p[(size_t)j * nd + i];
	norm = 1.0 / norm;
	memset(q, 0, sizeof(float) * (size_t)noffs * noffs);
	for (j = 0; j < nd && j < noffs; ++j)
		for (i = 0; i < nd && i < noffs; ++i)
			q[(size_t)j * noffs + i] = (float)(p[(size_t)j * nd + i] * norm);
	free(cs);
	free(mtf);
	free(half);
	free(p);
}

/* sum of the mirrored quadrant over the square ring at half-width m
   (the points with max(|x|, |y|) = m) */
static double grf_ring(const float *q, int noffs, int m)
{
	double s = 2.0 * ((double)q[m] + (double)q[(size_t)m * noffs]);
	int t;
	for (t = 1; t < m; ++t)
		s += 4.0 * ((double)q[(size_t)t * noffs + m] + (double)q[(size_t)m * noffs + t]);
	return s + 4.0 * (double)q[(size_t)m * noffs + m];
}

void irl_gendrf(float col_thick, float hole_diam, float gap, float intrinsic, float max_err, float bin_size,
	float drf_spacing, float min_dist, int ndist, int noffs, Drf_t *tab)
{
	float *q = (float *)irl_malloc(sizeof(float) * (size_t)noffs * noffs, "GRF quadrant");
	float dist = min_dist;
	int k;
	for (k = 0; k < ndist; ++k, dist += drf_spacing) {
		int m = noffs, w, h, x, y;
		double inside, norm = 1.0;
		float *psf;
		if (dist <= 0.0f) {
			/* at or behind the collimator face: a delta */
			memset(q, 0, sizeof(float) * (size_t)noffs * noffs);
			q[0] = 1.0f;
		} else {
			grf_grid g = grf_plan(dist, col_thick, gap, hole_diam, bin_size, intrinsic, noffs);
			grf_quadrant(&g, noffs, q);
			if (g.aliased)
				irl_warn("gendrf", "Possible aliasing in DRF table computation at distance %.2f", dist);
		}
		if (max_err > 0.0f) {
			/* smallest half-width whose square holds more than 1 - max_err */
			inside = q[0];
			for (m = 1; m < noffs && !(inside > 1.0 - max_err); ++m)
				inside += grf_ring(q, noffs, m);
			norm = 1.0 / inside;
		}
		w = 2 * m - 1;
		h = 2 * m - 1;
		psf = (float *)irl_malloc(sizeof(float) * (size_t)w * h, "PSF");
		for (y = 0; y < h; ++y)
			for (x = 0; x < w; ++x) {
				const int ay = abs(y - (m - 1)), ax = abs(x - (m - 1));
				psf[(size_t)y * w + x] = (float)(q[(size_t)ay * noffs + ax] * norm);
			}
		tab[k].MaxOffsX = m;
		tab[k].MaxOffsY = m;
		tab[k].bFFTdone = 0;
		tab[k].Psf = psf;
	}
	free(q);
}
