/*
 * irl_geom.h -- exact host-side geometry tables for the device kernels.
 *
 * These are computed in C (gcc, x86-64 SSE arithmetic, no contraction) with
 * the same float/double expression types as libirl so that the integer
 * shifts and interpolation weights the kernels use are bit-identical to
 * the ones libirl computes inline.
 */
#ifndef IRL_GEOM_H
#define IRL_GEOM_H

#ifdef __cplusplus
extern "C" {
#endif

/* Three-shear rotation of an n x n slice (fastrotate.c:330-563). */
typedef struct {
	int b90, b180;   /* 90 degree and 180 degree index flips */
	int iadd, mdim;  /* margin and side of the intermediate images */
	/* x shifts of passes 1 and 3 for row j: floor, weights f1, f2 */
	int *row_sh;
	float *row_f1, *row_f2;
	/* y shift of pass 2 for column i < mdim */
	int *col_sh;
	float *col_f1, *col_f2;
} irl_shear_tab;

/* Fills t for rotation by `angle` (already reduced to float as libirl's
   float parameter); row arrays need n entries, column arrays 2*n. */
void irl_shear_table(float angle, int n, irl_shear_tab *t);

/* Circular support of the fast rotator (fastrotate.c:573-589). */
void irl_shear_support(int n, int *start, int *end);

/* Bilinear rotator constants (rot3dpar.c:51-52). */
void irl_rot3dpar_sincos(float angle, float *s, float *c);

/* DRF table index of every rotated row of one view (prjbck.c:187-203), or
   -1 where the distance is <= 0 and libirl skips the convolution. */
void irl_drf_rows(float cfcr, float pix, int n, float start, float spacing, int ndist,
	int *row_idist);

/* Columns of a view treated as measured (osemrecon.c:140-184): 1 where
   the bin is inside [0, nbins), 0 where SetNonMeasuredBinsToZero zeroes
   the whole column. */
void irl_measured_columns(float left, float pix_over_bin, int n, int nbins,
	unsigned char *mask);

/* Columns that SetMeasuredPrjBinsToOne sets (osemrecon.c:92-138); it stops
   once the bin passes view->Right. */
void irl_norm_columns(float left, float right, float pix_over_bin, int n, int nbins,
	unsigned char *mask);

#ifdef __cplusplus
}
#endif
#endif
