/*
 * irl_host.h -- internal declarations of the libirl_b200 host library.
 */
#ifndef IRL_HOST_H
#define IRL_HOST_H

#include "irl.h"
#include "osemhooks.h"
#include "drftabio.h"
#include "krnlio.h"

#ifdef __cplusplus
extern "C" {
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* derived run parameters (libirl Parms_t, irlprivate.h:46-107, as set by
   vSetupParms, IrlSetup.c:51-91) */
typedef struct {
	int n, nz, nviews, nbins;
	float pix;
	float atn_scale, scatest_fac;
	int srf_iters;
	int prj_model, bck_model, model;
	char *norm_base;
	int ang_per_subset, iterations, start_iteration;
	int pad_len, avg_len;
	float hole_diam, hole_len, back_to_det, intrinsic_fwhm, max_frac_err;
} irl_parms;

/* per-view data (libirl View_t, irlprivate.h:134-154) */
typedef struct {
	float angle, cfcr, left, right;
	float view_time, sensitivity;
	DrfTab_t *drf;       /* table for this view's detector (not owned) */
	int det;
} irl_view;

/* detector (libirl Detector_t, irlprivate.h:117-127) */
typedef struct {
	float hole_diam, hole_len, back_to_det, intrinsic_fwhm, sensitivity;
	int fft_convolve, grf_in_bck;
	char *drf_fname;
	DrfTab_t *drf;
} irl_detector;

/* ESSE scatter model prepared on the host (krnlprj3d.c:403-547): the
   kernel in its file form, the weighted mean of mu over it and the FFT
   grid the device expands it to (irlcu_esse) */
typedef struct {
	int on;                 /* 0 when the kernel's scatter factor is 0 */
	int kx, ky, kz, collapse, nterms;
	float mu0, mu_avg, pix, cntr_pix_fac;
	int noffs, ndepths;     /* NumXYoffs, NumDists */
	float *krnl_file;       /* [ndepths][noffs][noffs] */
	float *mu_file;         /* [ndepths][noffs][noffs] */
	float kmu_outside;      /* K (mu - mu_avg) where K is 0: (0 - mu_avg) * 0 */
} irl_esse_host;

void irl_setup_parms(IrlParms_t *ip, Options_t *op, float *atn, char *krnl_fname, irl_parms *p);
irl_view *irl_setup_views(IrlParms_t *ip, PrjView_t *pv);
/* reads or computes the DRF tables of all detectors and assigns them to
   the views (IrlSetup.c:504-658); returns the detector count */
int irl_setup_drf_tables(irl_parms *p, Options_t *op, irl_view *views, char *drf_fname,
	irl_detector **pdets);
void irl_free_run_tables(void);

/* the per-call run tables (detectors, extra view data) of one
   reconstruction, parked while another one is current */
typedef struct {
	void **dets;
	int ndet, extra_nviews;
	float *acq_times;
	int *det_nums;
} irl_run_tables;
void irl_run_tables_park(irl_run_tables *t);
void irl_run_tables_unpark(const irl_run_tables *t);
DrfTab_t *irl_free_drftab(DrfTab_t *t);
void irl_esse_prepare(const char *krnl_fname, const irl_parms *p, int collapse, irl_esse_host *e);
void irl_esse_free(irl_esse_host *e);

/* GRF table (gendrf.c:218-427) */
void irl_gendrf(float col_thick, float hole_diam, float gap, float intrinsic, float max_err,
	float bin_size, float drf_spacing, float min_dist, int ndist, int noffs, Drf_t *tab);

/* the initial estimate from a precomputed irl_projection_sum */
float *irl_initial_estimate_sum(const irl_parms *p, int contour_support, float atn_thresh,
	const irl_view *views, float prj_sum, const float *atn, float *init);
float irl_projection_sum(const float *prj, size_t count);
float *irl_initial_estimate(const irl_parms *p, int contour_support, float atn_thresh,
	const irl_view *views, const float *prj, const float *atn, float *init);

/* subsets (osemrecon.c:395-456): returns the count; angles[s*per+i] */
int irl_compute_subsets(int nangles, int per_subset, int **angles);

/* external [z][y][x] <-> internal [y][z][x] */
void irl_reorder(int d0, int d1, int d2, const float *in, float *out);

/* fn(lo, hi, ctx) over [0, n) in chunks of at least grain elements, on up
   to 16 host threads (irl_par.c); for element-wise work only */
typedef void (*irl_range_fn)(size_t lo, size_t hi, void *ctx);
void irl_parallel_for(size_t n, size_t grain, irl_range_fn fn, void *ctx);
#define IRL_PAR_GRAIN ((size_t)1 << 18)

/* uploads the DRF tables of every view to the device (slot 0 projector,
   slot 1 backprojector when any detector has a separate GRF table) */
void irl_upload_drf(const irl_parms *p, irl_view *views, int ndet, irl_detector *dets);

/* device set-up: irl_device_geometry (context, rotation tables,
   measured-column masks), then the attenuation tables, then
   irl_device_tables (DRF and ESSE); irl_device_setup runs all three, from
   an attenuation map already in the internal layout */
void irl_device_geometry(irl_parms *p, irl_view *views, int fast_rotate, int max_batch);
void irl_device_tables(irl_parms *p, irl_view *views, const irl_esse_host *esse);
void irl_device_setup(irl_parms *p, irl_view *views, const float *atn_internal,
	const irl_esse_host *esse, int fast_rotate, int max_batch);

/* hook state (osemrecon.c:34-90) */
typedef void (*irl_hook_fn)(sOsemData *, void *);
extern irl_hook_fn g_irl_hooks[6];
extern void *g_irl_hook_ctx;
extern sAdvOptions g_irl_adv;
enum { HOOK_PREV_ITER, HOOK_POST_ITER, HOOK_PREV_SUBSET, HOOK_POST_SUBSET, HOOK_PREV_ANGLE, HOOK_POST_ANGLE };

/* per-view acquisition times and detector numbers (IrlSetup.c:22-49) */
extern int g_irl_extra_nviews;
extern float *g_irl_acq_times;
extern int *g_irl_det_nums;
extern int g_irl_ndet;
extern void **g_irl_dets;

#ifdef __cplusplus
}
#endif
#endif
