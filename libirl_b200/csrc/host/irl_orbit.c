/*
 * irl_orbit.c -- ComputeOrbit (irl.h; libirl computeorbit.c:21-150): the
 * camera's centre-of-rotation distance (CFCR) per view.
 *
 *   type 0: circular; every view gets fMargin.
 *   type 1: body contour; each view's camera sits fMargin (or
 *           pfMargins[view]) outside the body, whose outline is the part
 *           of the 2D image above the threshold.
 *   type 2: as 1, in L-mode: views i and i + NumViews/2 come from one
 *           camera configuration, so both get the larger of their two
 *           distances.
 *
 * For type 1/2 the body's extent towards each view's detector is the
 * device kernel irlcu_orbit_edges (k_orbit.cu).  It scans, for all views
 * at once, the image rotated onto a sqrt(2)-larger grid for the first row
 * that holds body.  This file does the rest on the host:
 *   - the threshold, applied in place to the caller's image as libirl
 *     does;
 *   - the grid side (ceil(sqrt 2 n), with n's parity);
 *   - each view's rotation sine and cosine from libm;
 *   - the radius arithmetic in libirl's operand types.
 * Any failure is trapped and returned as 1, with the message in
 * pchIrlErrorString.
 */
#include <math.h>
#include <setjmp.h>
#include <stdlib.h>

#include "irl_err.h"
#include "irl_host.h"
#include "irlcu.h"

#define ORBIT_E_MEMORY 1
#define ORBIT_E_TYPE 2

/* pixels at or below the threshold become 0: fThresh > 0 is a fraction of
   the maximum, fThresh <= 0 minus an absolute level */
static void orbit_threshold(float *img, int count, float fThresh)
{
	float level, top;
	int i;
	if (fThresh <= 0.0f) {
		level = -fThresh;
	} else {
		top = img[0];
		for (i = 1; i < count; ++i)
			if (img[i] > top)
				top = img[i];
		level = top * fThresh;
	}
	for (i = 0; i < count; ++i)
		if (img[i] <= level)
			img[i] = 0.0f;
}

int ComputeOrbit(float *pfPixels, IrlParms_t *psParms, float fMargin, float *pfMargins, float fThresh,
	int OrbitType, PrjView_t *psViews)
{
	const int nviews = psParms->NumViews, n = psParms->NumPixels;
	const float pix = psParms->BinWidth;
	/* volatile: read after a longjmp back to the trap */
	float *volatile sc = NULL;
	int *volatile rows = NULL;
	int side, v;
	jmp_buf env;
	if (OrbitType == 0) {
		for (v = 0; v < nviews; ++v)
			psViews[v].CFCR = fMargin;
		return 0;
	}
	/* libirl rejects only types above 2 (computeorbit.c:81-84); a negative
	   type runs the contour search as type 1 does */
	if (OrbitType > 2)
		return ORBIT_E_TYPE;
	if (setjmp(env)) {
		irl_untrap();
		free(sc);
		free(rows);
		return ORBIT_E_MEMORY;
	}
	irl_trap(&env);
	orbit_threshold(pfPixels, n * n, fThresh);
	side = (int)ceil(sqrt(2.0) * (double)n);
	side += (side & 1) != (n & 1);
	sc = (float *)irl_malloc(sizeof(float) * 2 * nviews, "orbit rotations");
	rows = (int *)irl_malloc(sizeof(int) * nviews, "orbit edges");
	for (v = 0; v < nviews; ++v) {
		/* rows parallel to the detector, row 0 the farthest from the centre
		   towards it: the rotation libirl applies, at float angle */
		const float a = (float)(0.5 * M_PI + psViews[v].Angle);
		sc[v] = (float)sin(a);
		sc[nviews + v] = (float)cos(a);
	}
	irl_cu(irlcu_orbit_edges(pfPixels, n, side, sc, sc + nviews, nviews, rows), "ComputeOrbit");
	for (v = 0; v < nviews; ++v) {
		/* half the grid minus the rows outside the body, in cm */
		float r = (float)(((double)(float)side / 2.0 - (double)(float)rows[v]) * (double)pix);
		r += pfMargins != NULL ? pfMargins[v] : fMargin;
		psViews[v].CFCR = r;
	}
	if (OrbitType == 2)
		for (v = 0; v < nviews / 2; ++v) {
			float *a = &psViews[v].CFCR, *b = &psViews[v + nviews / 2].CFCR;
			const float far = *a > *b ? *a : *b;
			*a = *b = far;
		}
	irl_untrap();
	free(sc);
	free(rows);
	return 0;
}
