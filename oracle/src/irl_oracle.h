/*
 * irl_oracle.h -- CPU restatement of libirl's OSEM projector/backprojector
 * path.  TEST INFRASTRUCTURE ONLY: it is the checker for the CUDA product,
 * never part of it.
 *
 * All arrays use libirl's internal layout: volumes [y][z][x] (n*nz*n),
 * projections [view][z][x].  The restatement is written from the libirl
 * sources it cites; its ESSE convolution is an exact (double precision)
 * circular convolution, which is also what the MIP shim gives the compiled
 * reference.
 */
#ifndef IRL_ORACLE_H
#define IRL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
	int n, nz, nviews;
	float pix;
	int fast_rotate;
	const float *angle, *cfcr, *left, *right, *view_time, *sens;  /* per view */
	/* DRF table (projector); bck_* may point to a second table */
	int ndist;
	float drf_start, drf_spacing;
	const int *mx, *my;          /* MaxOffsX / MaxOffsY per distance */
	const float *psf;            /* concatenated PSFs */
	const long *psf_off;         /* offset of each PSF in psf */
	int bck_ndist;
	float bck_start, bck_spacing;
	const int *bck_mx, *bck_my;
	const float *bck_psf;
	const long *bck_off;
	int pad_len, avg_len;
	/* ESSE */
	int esse_on;
	int kx, ky, kz, collapse, nterms;
	float mu0, mu_avg, esse_pix, cntr;
	const float *krnl, *kmu;     /* reordered kernel grids [ky][kz][kx] */
} or_problem;

void or_shears_rotate(float angle, const float *in, float *out, int n, int nz);
void or_rot3dpar(float angle, const float *in, float *out, int n, int nz);
void or_conv2d_ypad(const float *a, int nx, int ny, const float *b, int cx, int cy, int pady, int avgy,
	float *out);
void or_esse_prepare(const float *krnl, const float *kmu, int noffs, int ndists, int n, int nz, int c,
	float *grid_k, float *grid_kmu, float *mu_avg);
void or_esse_source(const or_problem *P, const float *act, const float *map, float *eff);
/* libirl Project: calcprj (nz*n) of one view; model bits 1 atn, 2 drf, 4 srf */
void or_project(const or_problem *P, int model, int view, const float *est, const float *atn,
	float primary, float *calcprj);
/* libirl BackProject: image += unrotated backprojection of ratio, clamp */
void or_backproject(const or_problem *P, int model, int view, const float *atn, const float *ratio,
	float *image);
/* libirl IrlGenprj core (irlgenprj.c:225-264) on internal-layout inputs */
void or_genprj(const or_problem *P, int model, const float *act, const float *atn, const float *scatest,
	float primary, float *prj);
/* libirl vOsemRecon (osemrecon.c:557-897) on internal-layout inputs;
   est is the initial estimate on entry and the result on return */
int or_osem(const or_problem *P, int prj_model, int bck_model, int srf_iters, int iterations, int per_subset,
	const float *meas, const float *atn, const float *scatest, float *est);
void or_initial_estimate(int n, int nz, int nviews, const float *prj, float *est);
/* host threads for the independent views of or_genprj and of each or_osem
   subset (default 1); results do not depend on it */
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
