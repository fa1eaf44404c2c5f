/*
 * irl_setup.c -- run set-up of libirl_b200 on the host: parameters, views,
 * per-view extra data and detectors, DRF tables (read or computed GRF),
 * ESSE kernel preparation, initial estimate, subsets.
 *
 * Each routine follows the libirl routine named beside it; expressions that
 * decide integer indices or table sizes keep libirl's float/double types so
 * the decisions are identical.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "irl_err.h"
#include "irl_host.h"
#include "irl_geom.h"
#include "irlcu.h"

#ifndef MAX
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#endif
#ifndef MIN
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#endif

/* ------------------------------------------------ extra view data / detectors */

int g_irl_extra_nviews = 0;
float *g_irl_acq_times = NULL;
int *g_irl_det_nums = NULL;
int g_irl_ndet = 0;
void **g_irl_dets = NULL;

/* IrlSetup.c:350-402 */
int iSetupExtraPrjViewData(int iNumPrjViews, float *pfAcqTimes, int *piDetectorNums)
{
	int i, err = 0;
	g_irl_extra_nviews = iNumPrjViews;
	if (pfAcqTimes != NULL)
		g_irl_acq_times = pfAcqTimes;
	if (piDetectorNums != NULL)
		g_irl_det_nums = piDetectorNums;
	if (iNumPrjViews < 0)
		err = 1;
	if (iNumPrjViews > 0 && pfAcqTimes == NULL && piDetectorNums == NULL)
		err = 1;
	if (iNumPrjViews == 0 && (pfAcqTimes != NULL || piDetectorNums != NULL))
		err = 1;
	if (pfAcqTimes != NULL)
		for (i = 0; i < iNumPrjViews; ++i)
			if (pfAcqTimes[i] < 0.0)
				err |= 2;
	if (piDetectorNums != NULL)
		for (i = 0; i < iNumPrjViews; ++i)
			if (piDetectorNums[i] < 0)
				err |= 4;
	return err;
}

/* IrlSetup.c:415-439 */
void *pvStoreDetectorData(float fHoleDiam, float fHoleLen, float fBackToDet, float fIntrinsicFWHM,
	float fSensitivity, int bFFTconvolve, int bUseGrfInBck, char *pchDrfTabFname)
{
	irl_detector *d = (irl_detector *)calloc(1, sizeof(irl_detector));
	if (d == NULL)
		return NULL;
	d->hole_diam = fHoleDiam;
	d->hole_len = fHoleLen;
	d->back_to_det = fBackToDet;
	d->intrinsic_fwhm = fIntrinsicFWHM;
	d->sensitivity = fSensitivity;
	d->fft_convolve = bFFTconvolve;
	d->grf_in_bck = bUseGrfInBck;
	d->drf_fname = pchDrfTabFname;
	d->drf = NULL;
	return d;
}

/* IrlSetup.c:441-462 */
int iSetupDetectors(int iNumDetectors, void **ppsDetectors)
{
	int err = 0;
	g_irl_ndet = iNumDetectors;
	g_irl_dets = ppsDetectors;
	if (iNumDetectors < 0)
		err = 1;
	if (iNumDetectors > 0 && ppsDetectors == NULL)
		err = 2;
	if (iNumDetectors == 0 && ppsDetectors != NULL)
		err = 4;
	return err;
}

/* end-of-run release of caller-supplied tables (IrlSetup.c:404-413,
   464-481): the arrays, detector records and DRF file names are freed */
void irl_free_run_tables(void)
{
	int i;
	free(g_irl_acq_times);
	g_irl_acq_times = NULL;
	free(g_irl_det_nums);
	g_irl_det_nums = NULL;
	g_irl_extra_nviews = 0;
	if (g_irl_dets != NULL) {
		for (i = 0; i < g_irl_ndet; ++i) {
			irl_detector *d = (irl_detector *)g_irl_dets[i];
			if (d == NULL)
				continue;
			free(d->drf_fname);
			d->drf = irl_free_drftab(d->drf);
			free(d);
			g_irl_dets[i] = NULL;
		}
		free(g_irl_dets);
	}
	g_irl_dets = NULL;
	g_irl_ndet = 0;
}

void irl_run_tables_park(irl_run_tables *t)
{
	t->dets = g_irl_dets;
	t->ndet = g_irl_ndet;
	t->extra_nviews = g_irl_extra_nviews;
	t->acq_times = g_irl_acq_times;
	t->det_nums = g_irl_det_nums;
	g_irl_dets = NULL;
	g_irl_ndet = 0;
	g_irl_extra_nviews = 0;
	g_irl_acq_times = NULL;
	g_irl_det_nums = NULL;
}

void irl_run_tables_unpark(const irl_run_tables *t)
{
	g_irl_dets = t->dets;
	g_irl_ndet = t->ndet;
	g_irl_extra_nviews = t->extra_nviews;
	g_irl_acq_times = t->acq_times;
	g_irl_det_nums = t->det_nums;
}

/* ------------------------------------------------------------ parameters */

/* vSetupParms, IrlSetup.c:51-91 */
void irl_setup_parms(IrlParms_t *ip, Options_t *op, float *atn, char *krnl_fname, irl_parms *p)
{
	int srf, drf, at;
	memset(p, 0, sizeof(*p));
	p->n = ip->NumPixels;
	p->nbins = ip->NumPixels;
	p->nviews = ip->NumViews;
	p->nz = ip->NumSlices;
	p->pix = ip->BinWidth;
	p->atn_scale = ip->fAtnScaleFac;
	p->srf_iters = ip->iNumSrfIterations;
	p->scatest_fac = ip->fScatEstFac;
	p->hole_len = ip->fHoleLen;
	p->hole_diam = ip->fHoleDiam;
	p->back_to_det = ip->fBackToDet;
	p->max_frac_err = 0.05f;
	p->intrinsic_fwhm = ip->fIntrinsicFWHM;
	srf = krnl_fname == NULL ? 0 : MODEL_SRF;
	drf = op->bModelDrf ? MODEL_DRF : 0;
	at = atn == NULL ? 0 : MODEL_ATN;
	p->prj_model = srf | at | drf;
	p->bck_model = at | drf;
	p->model = srf | at | drf;
	p->ang_per_subset = ip->NumAngPerSubset;
	p->norm_base = ip->pchNormImageBase;
	p->iterations = ip->NumIterations;
	p->start_iteration = 0;
	p->pad_len = op->iAxialPadLength;
	p->avg_len = op->iAxialAvgLength;
	if (p->n <= 0 || p->nz <= 0 || p->nviews <= 0)
		irl_fatal(IRL_E_VALUE, "SetupParms", "NumPixels, NumSlices and NumViews must be positive");
	if (p->pix <= 0.0f)
		irl_fatal(IRL_E_VALUE, "SetupParms", "BinWidth must be positive, not %g", p->pix);
}

/* psSetupViews, IrlSetup.c:101-144 */
irl_view *irl_setup_views(IrlParms_t *ip, PrjView_t *pv)
{
	int i, n = ip->NumViews;
	irl_view *v = (irl_view *)irl_calloc(sizeof(irl_view) * n, "views");
	for (i = 0; i < n; ++i) {
		v[i].angle = pv[i].Angle;
		v[i].cfcr = pv[i].CFCR;
		v[i].right = pv[i].Right;
		v[i].left = pv[i].Left;
		v[i].view_time = 1.0f;
		v[i].sensitivity = 1.0f;
		v[i].drf = NULL;
		v[i].det = 0;
	}
	if (g_irl_acq_times != NULL) {
		if (g_irl_extra_nviews != n)
			irl_fatal(IRL_E_VALUE, "SetupViews", "Number of Prj Views passed to SetupExtrPrjViewData is incorrect");
		for (i = 0; i < n; ++i)
			v[i].view_time = g_irl_acq_times[i];
	}
	return v;
}

/* ------------------------------------------------------------ GRF tables */
/* irl_gendrf (the GRF table generator) lives in irl_grf.c */

/* vComputeDrfs, IrlSetup.c:243-334 */
static void compute_drfs(DrfTab_t *t, float fPixelWidth, float fBinWidth, int iReconMatSize, float fMinDist,
	float fMaxDist)
{
	int iNumDrfOffs = (int)(iReconMatSize * 0.5);
	int iNumDists = ((fMaxDist - fMinDist) / fPixelWidth + 1 + 0.5);
	t->psDrfs = (Drf_t *)irl_calloc(iNumDists * sizeof(Drf_t), "GRF table");
	t->iNumDistances = iNumDists;
	t->fStartDistance = fMinDist;
	t->fDrfSpacing = fPixelWidth;
	t->fPixSize = fPixelWidth;
	t->bIncKrnl = 0;
	irl_gendrf(t->fColThick, t->fHoleDiam, t->fGap, t->fIntrinsicFWHM, t->fMaxFracErr, fBinWidth, fPixelWidth,
		fMinDist, iNumDists, iNumDrfOffs, t->psDrfs);
}

#define RELDIF(a, b) (2.0 * fabs((a) - (b)) / (((fabs(a) + fabs(b)) == 0.0) ? 1 : (fabs(a) + fabs(b))))
#define CMPRFLOAT(a, b, tol) (RELDIF((a), (b)) <= tol)

/* vCheckDrfTab, IrlSetup.c:202-241 */
static void check_drftab(const DrfTab_t *t, float fPixWid, float fMinDist, float fMaxDist, const char *fname)
{
	float fTabMax;
	if (!CMPRFLOAT(t->fPixSize, fPixWid, 0.01))
		irl_fatal(IRL_E_VALUE, "vCheckDrfTab",
			"The pixel size in Drf Table %s is %.4f, and not %.4f as needed for recon.", fname, t->fPixSize,
			fPixWid);
	fTabMax = t->fStartDistance + (t->iNumDistances - 1) * t->fDrfSpacing;
	if (!(((CMPRFLOAT(fMinDist, t->fStartDistance, 0.0001) || fMinDist > t->fStartDistance) &&
		      (CMPRFLOAT(fMaxDist, fTabMax, 0.0001) || fMaxDist < fTabMax)) ||
		    (fMaxDist > fTabMax)))
		irl_warn("vCheckDrfTab",
			"The range of distances in %s is (%.2f to %.2f), reconstruction needs (%.2f to %.2f). "
			"Approximations will be used",
			fname, t->fStartDistance, fTabMax, fMinDist, fMaxDist);
	if (!CMPRFLOAT(t->fDrfSpacing, fPixWid, 0.01))
		irl_warn("vCheckDrfTab", "The distance between Drfs in %s is %.4f, not %.4f. NN interp will be used",
			fname, t->fDrfSpacing, fPixWid);
}

/* psDrfSetup, IrlSetup.c:504-588 */
static DrfTab_t *drf_setup(float fMinCFCR, float fMaxCFCR, float fPixelWidth, float fBinWidth, int n,
	float fMaxFracErr, irl_detector *d)
{
	DrfTab_t *t = (DrfTab_t *)irl_calloc(sizeof(DrfTab_t), "DRF table");
	float fMinDist = fMinCFCR - n / 2 * fPixelWidth + fPixelWidth / 2;
	float fMaxDist;
	if (fMinDist < 0)
		fMinDist = fPixelWidth / 2;
	fMaxDist = fMaxCFCR + n / 2 * fPixelWidth - fPixelWidth / 2;
	t->fGap = d->back_to_det;
	t->fHoleDiam = d->hole_diam;
	t->fColThick = d->hole_len;
	t->fIntrinsicFWHM = d->intrinsic_fwhm;
	t->fMaxFracErr = fMaxFracErr;
	if (d->drf_fname != NULL) {
		char *title = NULL, *col = NULL;
		DrfTab_t r = sReadDrfTab(d->drf_fname, &title, &col);
		free(title);
		free(col);
		r.psBckDrfTab = NULL;
		*t = r;
		check_drftab(t, fPixelWidth, fMinDist, fMaxDist, d->drf_fname);
		if (d->grf_in_bck) {
			DrfTab_t *b = (DrfTab_t *)irl_calloc(sizeof(DrfTab_t), "GRF table");
			b->fGap = d->back_to_det;
			b->fHoleDiam = d->hole_diam;
			b->fColThick = d->hole_len;
			b->fIntrinsicFWHM = d->intrinsic_fwhm;
			b->fMaxFracErr = fMaxFracErr;
			compute_drfs(b, fPixelWidth, fBinWidth, n, fMinDist, fMaxDist);
			b->psBckDrfTab = NULL;
			b->bFFTconvolve = 0;
			t->psBckDrfTab = b;
		}
	} else {
		compute_drfs(t, fPixelWidth, fBinWidth, n, fMinDist, fMaxDist);
	}
	t->bFFTconvolve = d->fft_convolve;
	return t;
}

/* vSetupDrfTables, IrlSetup.c:590-658 */
int irl_setup_drf_tables(irl_parms *p, Options_t *op, irl_view *views, char *drf_fname, irl_detector **pdets)
{
	int a, k;
	float fMin, fMax;
	if (g_irl_ndet == 0) {
		void **arr = (void **)irl_malloc(sizeof(void *), "detector table");
		arr[0] = pvStoreDetectorData(p->hole_diam, p->hole_len, p->back_to_det, p->intrinsic_fwhm, 1.0f,
			op->bFFTConvolve, op->bUseGrfInBck, drf_fname);
		if (arr[0] == NULL)
			irl_fatal(IRL_E_MALLOC, "vSetupDrfTables", "out of memory");
		iSetupDetectors(1, arr);
	}
	fMin = fMax = views[0].cfcr;
	for (a = 0; a < p->nviews; ++a) {
		fMin = fMin > views[a].cfcr ? views[a].cfcr : fMin;
		fMax = fMax < views[a].cfcr ? views[a].cfcr : fMax;
	}
	for (k = 0; k < g_irl_ndet; ++k) {
		irl_detector *d = (irl_detector *)g_irl_dets[k];
		if (p->prj_model & MODEL_DRF)
			d->drf = drf_setup(fMin, fMax, p->pix, p->pix, p->n, p->max_frac_err, d);
		else
			d->drf = NULL;
	}
	for (a = 0; a < p->nviews; ++a) {
		if (g_irl_det_nums == NULL) {
			views[a].det = 0;
			views[a].drf = ((irl_detector *)g_irl_dets[0])->drf;
			views[a].sensitivity = 1.0f;
		} else {
			int dn = g_irl_det_nums[a];
			if (dn < 0 || dn >= g_irl_ndet)
				irl_fatal(IRL_E_VALUE, "vSetupDrfTables", "Illegal detector specified for view %d (%d)", a, dn);
			views[a].det = dn;
			views[a].drf = ((irl_detector *)g_irl_dets[dn])->drf;
			views[a].sensitivity = ((irl_detector *)g_irl_dets[dn])->sensitivity;
		}
	}
	*pdets = NULL;
	return g_irl_ndet;
}

/* Concatenates the tables of all detectors, pads every PSF to the common
   half-width and uploads the per-view row -> table index map. */
static void upload_one(const irl_parms *p, irl_view *views, int bck)
{
	int ndet = g_irl_ndet, k, a, i, halo = 0, total = 0, w;
	int *base = (int *)irl_calloc(sizeof(int) * (ndet + 1), "DRF offsets");
	DrfTab_t **tabs = (DrfTab_t **)irl_calloc(sizeof(DrfTab_t *) * (ndet + 1), "DRF tables");
	float *psf;
	int *pad, *rows, *taps;
	irlcu_drf D;
	for (k = 0; k < ndet; ++k) {
		DrfTab_t *t = ((irl_detector *)g_irl_dets[k])->drf;
		if (t != NULL && bck && t->psBckDrfTab != NULL)
			t = t->psBckDrfTab;
		tabs[k] = t;
		base[k] = total;
		if (t == NULL)
			continue;
		for (i = 0; i < t->iNumDistances; ++i) {
			halo = MAX(halo, t->psDrfs[i].MaxOffsX - 1);
			halo = MAX(halo, t->psDrfs[i].MaxOffsY - 1);
		}
		total += t->iNumDistances;
	}
	w = 2 * halo + 1;
	psf = (float *)irl_calloc(sizeof(float) * (size_t)total * w * w, "padded PSFs");
	pad = (int *)irl_calloc(sizeof(int) * (total > 0 ? total : 1), "pad rows");
	taps = (int *)irl_calloc(sizeof(int) * (total > 0 ? total : 1), "PSF taps");
	for (k = 0; k < ndet; ++k) {
		DrfTab_t *t = tabs[k];
		if (t == NULL)
			continue;
		for (i = 0; i < t->iNumDistances; ++i) {
			const Drf_t *d = &t->psDrfs[i];
			int wx = 2 * d->MaxOffsX - 1, wy = 2 * d->MaxOffsY - 1, yy, xx;
			int oy = halo - (d->MaxOffsY - 1), ox = halo - (d->MaxOffsX - 1);
			float *dst = psf + (size_t)(base[k] + i) * w * w;
			for (yy = 0; yy < wy; ++yy)
				for (xx = 0; xx < wx; ++xx)
					dst[(size_t)(yy + oy) * w + xx + ox] = d->Psf[yy * wx + xx];
			/* conv2d_ypad.c:54-57: iPadY = clamp(iAxialPadLength, 0, bCtrY);
			   conv2dPsfFFT zero pads instead (convolve_ypad.c:63-94) */
			pad[base[k] + i] = t->bFFTconvolve ? 0 : MIN(MAX(p->pad_len, 0), d->MaxOffsY - 1);
			taps[base[k] + i] = wx * wy;
		}
	}
	rows = (int *)irl_malloc(sizeof(int) * (size_t)p->nviews * p->n, "DRF rows");
	for (a = 0; a < p->nviews; ++a) {
		DrfTab_t *t = tabs[views[a].det];
		if (t == NULL) {
			for (i = 0; i < p->n; ++i)
				rows[(size_t)a * p->n + i] = -1;
			continue;
		}
		irl_drf_rows(views[a].cfcr, p->pix, p->n, t->fStartDistance, t->fDrfSpacing, t->iNumDistances,
			rows + (size_t)a * p->n);
		for (i = 0; i < p->n; ++i)
			if (rows[(size_t)a * p->n + i] >= 0)
				rows[(size_t)a * p->n + i] += base[views[a].det];
	}
	D.ndist = total;
	D.halo = halo;
	D.psf = psf;
	D.pad_rows = pad;
	D.row_idist = rows;
	D.avg_rows = MIN(MAX(p->avg_len, 0), p->nz);
	D.taps = taps;
	irl_cu(irlcu_set_drf(bck, total > 0 ? &D : NULL), "SetupDrf");
	free(psf);
	free(pad);
	free(taps);
	free(rows);
	free(base);
	free(tabs);
}

void irl_upload_drf(const irl_parms *p, irl_view *views, int ndet, irl_detector *dets)
{
	int k, separate = 0;
	(void)ndet;
	(void)dets;
	upload_one(p, views, 0);
	for (k = 0; k < g_irl_ndet; ++k) {
		DrfTab_t *t = ((irl_detector *)g_irl_dets[k])->drf;
		if (t != NULL && t->psBckDrfTab != NULL)
			separate = 1;
	}
	if (separate)
		upload_one(p, views, 1);
	else
		irl_cu(irlcu_set_drf(1, NULL), "SetupDrf");
}

/* ------------------------------------------------------------------- ESSE */

/* pfReorder3dKrnl, krnlprj3d.c:43-128, puts the file's one-quadrant kernel
   [depth][y offset][x offset] into a wrap-around grid [depth][slice][offset]
   of oxd x oyd x ozd with the depth axis flipped: offset ix < xmin =
   min(noffs, oxd/2) lands on x = ix and, for ix > 0, on its mirror
   oxd - ix; the same along y; depth izin on the plane
   ozd/2 - izin + ndepths/2 - 1, rotated by half the axis.  Everything else
   is 0.  The device builds the grids (irlcu_esse_expand); the host only
   needs the grid indices that hold kernel values, in increasing order, with
   the file index each one comes from. */
typedef struct {
	size_t count;
	size_t *grid;   /* grid index, increasing */
	int *file;      /* index into the file's arrays */
} krnl_support_map;

static krnl_support_map krnl_support(int noffs, int ndepths, int oxd, int oyd, int ozd)
{
	int xmin = MIN(noffs, oxd / 2), ymin = MIN(noffs, oyd / 2), nxs = 0, nys = 0, iz, iy, ix, t;
	int *xs = (int *)irl_malloc(sizeof(int) * 2 * (size_t)(xmin + 1), "kernel support");
	int *xf = (int *)irl_malloc(sizeof(int) * 2 * (size_t)(xmin + 1), "kernel support");
	int *ys = (int *)irl_malloc(sizeof(int) * 2 * (size_t)(ymin + 1), "kernel support");
	int *yf = (int *)irl_malloc(sizeof(int) * 2 * (size_t)(ymin + 1), "kernel support");
	int *zin = (int *)irl_malloc(sizeof(int) * (size_t)ozd, "kernel support");
	krnl_support_map m;
	for (t = 0; t < xmin; ++t, ++nxs)
		xs[nxs] = xf[nxs] = t;
	for (t = oxd - xmin + 1; t < oxd; ++t, ++nxs) {
		xs[nxs] = t;
		xf[nxs] = oxd - t;
	}
	for (t = 0; t < ymin; ++t, ++nys)
		ys[nys] = yf[nys] = t;
	for (t = oyd - ymin + 1; t < oyd; ++t, ++nys) {
		ys[nys] = t;
		yf[nys] = oyd - t;
	}
	for (iz = 0; iz < ozd; ++iz)
		zin[iz] = -1;
	for (t = 0; t < ndepths; ++t) {
		int z = ozd / 2 - t + ndepths / 2 - 1;
		if (z < 0 || z >= ozd)
			continue;
		z += z < ozd / 2 ? ozd / 2 : -ozd / 2;
		zin[z] = t;
	}
	m.count = 0;
	m.grid = (size_t *)irl_malloc(sizeof(size_t) * ((size_t)nxs * nys * ozd + 1), "kernel support");
	m.file = (int *)irl_malloc(sizeof(int) * ((size_t)nxs * nys * ozd + 1), "kernel support");
	for (iz = 0; iz < ozd; ++iz)
		if (zin[iz] >= 0)
			for (iy = 0; iy < nys; ++iy)
				for (ix = 0; ix < nxs; ++ix) {
					m.grid[m.count] = xs[ix] + (size_t)oxd * (ys[iy] + (size_t)oyd * iz);
					m.file[m.count++] = xf[ix] + noffs * (yf[iy] + noffs * zin[iz]);
				}
	free(xs);
	free(xf);
	free(ys);
	free(yf);
	free(zin);
	return m;
}

/* pvInitESSEScatterModel + pvInitScatterPrj, krnlprj3d.c:956-1009, 403-547,
   with libirl's hard-coded parameters "2 2 2 3" (IrlSetup.c:169-174):
   xy pad 2, z pad 2, two Taylor terms, 3D geometry.  The kernel stays in
   its file form; its grids K and K (mu - mu_avg) are built on the device. */
void irl_esse_prepare(const char *fname, const irl_parms *p, int c, irl_esse_host *e)
{
	const float xypad = 2, zpad = 2;
	const int nterms = 2;
	KrnlData_t *k;
	int nx, ny, nz;
	size_t q, fcount;
	float fKs = 0.0f, fKMs = 0.0f;
	krnl_support_map sup;
	memset(e, 0, sizeof(*e));
	if (c < 1 || c > 4)
		irl_fatal(IRL_E_VALUE, "SrfSetup", "srf_collapse_fac = %d: must be 1 (no collapse) to 4", c);
	k = psReadKrnlFile((char *)fname, 1);
	if (k->fScatFac == 0.0) {
		psFreeKrnlData(k, 1);
		return;
	}
	e->on = 1;
	e->mu0 = k->fKrnlMu0;
	e->pix = p->pix;
	e->cntr_pix_fac = k->fCntrPixFac;
	e->nterms = nterms;
	e->collapse = c;
	nx = p->n / c;
	ny = p->n / c;
	nz = p->nz / c;
	nx = (int)ceil(xypad * (float)(nx));
	ny = (int)ceil(xypad * (float)(ny));
	nz = (int)ceil(zpad * (float)nz);
	e->kx = nx;
	e->ky = ny;
	e->kz = nz;
	e->noffs = k->iNumXYoffs;
	e->ndepths = k->iNumDists;
	fcount = (size_t)e->noffs * e->noffs * e->ndepths;
	e->krnl_file = (float *)irl_malloc(sizeof(float) * fcount, "ESSE kernel");
	e->mu_file = (float *)irl_malloc(sizeof(float) * fcount, "ESSE mu kernel");
	memcpy(e->krnl_file, k->pfKrnl, sizeof(float) * fcount);
	memcpy(e->mu_file, k->pfKrnlMu, sizeof(float) * fcount);
	/* libirl's float sums run over the whole reordered grid in index order
	   (krnlprj3d.c:495-510).  Outside the kernel's support both grids hold
	   +0, and adding +0 (or the product +0 * 0) to a float sum that starts at
	   +0 leaves it unchanged, so summing the support in the same order gives
	   the same bits. */
	sup = krnl_support(e->noffs, e->ndepths, nx, nz, ny);
	for (q = 0; q < sup.count; ++q) {
		const float kv = e->krnl_file[sup.file[q]];
		fKs += kv;
		fKMs += kv * e->mu_file[sup.file[q]];
	}
	free(sup.grid);
	free(sup.file);
	if (fKs == 0.0) {
		irl_warn("InitScatterPrj", "Sum of Krnl is 0!");
		e->mu_avg = k->fKrnlMu0;
	} else {
		e->mu_avg = fKMs / fKs;
	}
	/* K (mu - mu_avg) outside the support: (0 - mu_avg) * 0 */
	e->kmu_outside = (0.0f - e->mu_avg) * 0.0f;
	if (fabs(k->fPixSize - p->pix * c) > 0.02)
		irl_warn("vInitESSEScatterModel", "Pixel size after collapse=%.3g, Pixel size in kernel=%.3g",
			c * p->pix, k->fPixSize);
	if (p->n % c != 0 || p->nz % c != 0)
		irl_fatal(IRL_E_VALUE, "CollapseByFac", "factor %d does not evenly divide image dimensions %d, %d",
			c, p->n, p->nz);
	psFreeKrnlData(k, 1);
}

void irl_esse_free(irl_esse_host *e)
{
	free(e->krnl_file);
	free(e->mu_file);
	memset(e, 0, sizeof(*e));
}

/* ------------------------------------------------------ initial estimate */

/* vZeroBehind, initial_est.c:160-180 */
static void zero_behind(int nd, float fSin, float fCos, float fRadius, float *pix)
{
	int ix, iy;
	float fX, fY, fR;
	for (iy = 0; iy < nd; ++iy) {
		fY = iy - (float)nd / 2.0;
		for (ix = 0; ix < nd; ++ix) {
			fX = ix - (float)nd / 2.0;
			fR = floor(fX * fCos + fY * fSin + 0.5);
			if (fR > fRadius)
				pix[ix + iy * nd] = 0.0;
		}
	}
}

/* One pass over the estimate's rows (r, s) writes what libirl's three
   passes leave (initial_est.c:97-157): the mean or the contour image, 0 where
   the attenuation map is below the threshold, 0 outside the circle. */
typedef struct {
	float *init;
	float v;                      /* the mean, when img is NULL */
	const float *img;             /* contour image [r][c], or NULL */
	const unsigned char *outside; /* [r][c]: beyond the reconstruction circle */
	const float *atn;             /* internal layout, or NULL for no map mask */
	float thresh;
	int n, nz;
} init_ctx;

static void init_range(size_t lo, size_t hi, void *c)
{
	const init_ctx *f = (const init_ctx *)c;
	const int n = f->n;
	size_t q;
	int x;
	for (q = lo; q < hi; ++q) {
		const size_t r = q / (size_t)f->nz;
		float *out = f->init + q * n;
		const float *a = f->atn != NULL ? f->atn + q * n : NULL;
		for (x = 0; x < n; ++x) {
			float v = f->img != NULL ? f->img[x + r * n] : f->v;
			if ((a != NULL && a[x] < f->thresh) || f->outside[r * n + x])
				v = 0.0f;
			out[x] = v;
		}
	}
}

/* pfComputeInitialEstimate, initial_est.c:29-158 (internal layout) */
/* libirl's float sum of all projection bins, in index order
   (initial_est.c:89-95) */
float irl_projection_sum(const float *prj, size_t count)
{
	float fSum = 0.0f;
	size_t i;
	for (i = 0; i < count; ++i)
		fSum += prj[i];
	return fSum;
}

float *irl_initial_estimate(const irl_parms *p, int contour, float thresh, const irl_view *views, const float *prj,
	const float *atn, float *init)
{
	return irl_initial_estimate_sum(p, contour, thresh, views,
		irl_projection_sum(prj, (size_t)p->n * p->nz * p->nviews), atn, init);
}

float *irl_initial_estimate_sum(const irl_parms *p, int contour, float thresh, const irl_view *views, float fSum,
	const float *atn, float *init)
{
	int n = p->n, nz = p->nz, na = p->nviews, a, r, c2, use_map = 0;
	size_t i;
	float fNum = (float)(n * n * nz), fAvg, fMapThresh = 0.0f;
	fNum *= M_PI / 4.0;
	fAvg = fSum / (fNum * na);
	if (atn != NULL) {
		fMapThresh = thresh;
		fMapThresh *= p->pix;
		if (fMapThresh < 0.0)
			irl_warn("ComputeInitialEstimate", "atnmap_support_thresh must be > 0, not %.3f. Ignoring",
				fMapThresh);
		else
			use_map = fMapThresh > 0.0;
	}
	{
		float *img = NULL;
		unsigned char *outside = (unsigned char *)irl_malloc((size_t)n * n, "circle mask");
		float fRadius = (float)n * 0.5, fX, fY, fCent = fRadius;
		init_ctx ic;
		if (contour) {
			img = (float *)irl_malloc(sizeof(float) * n * n, "contour image");
			for (i = 0; i < (size_t)n * n; ++i)
				img[i] = fAvg;
			for (a = 0; a < na; ++a) {
				double d = views[a].angle;
				zero_behind(n, (float)sin(d), (float)cos(d), views[a].cfcr / p->pix, img);
			}
		}
		for (r = 0; r < n; ++r) {
			fY = (float)r - fCent;
			if (fY > 0)
				fY += 1;
			for (c2 = 0; c2 < n; ++c2) {
				fX = (float)c2 - fCent;
				if (fX > 0)
					fX += 1;
				outside[(size_t)r * n + c2] = hypot(fX, fY) > fRadius;
			}
		}
		ic.init = init;
		ic.v = fAvg;
		ic.img = img;
		ic.outside = outside;
		ic.atn = use_map ? atn : NULL;
		ic.thresh = fMapThresh;
		ic.n = n;
		ic.nz = nz;
		irl_parallel_for((size_t)n * nz, (IRL_PAR_GRAIN + n - 1) / n, init_range, &ic);
		free(img);
		free(outside);
	}
	return init;
}

/* ---------------------------------------------------------------- subsets */

/* iComputeSubsets, osemrecon.c:395-456 */
int irl_compute_subsets(int na, int per, int **angles)
{
	int ns, s, m, a;
	if (per <= 0 || na % per)
		irl_fatal(IRL_E_VALUE, "iComputeSubsets",
			"No. of angles not an integer multiple of the no. of angles per subset\n NumAngles=%d, NumAngPerSet=%d",
			na, per);
	ns = na / per;
	if (ns != 1 && ns % 2)
		irl_fatal(IRL_E_VALUE, "iComputeSubsets", "Number of subsets (%d) for num_ang_per_set=%d is not even",
			ns, per);
	*angles = (int *)irl_malloc(sizeof(int) * na, "subset angles");
	for (s = 0; s < ns; ++s) {
		a = s / 2 + (s % 2) * ns / 2;
		for (m = 0; m < per; ++m) {
			(*angles)[s * per + m] = a;
			a += ns;
		}
	}
	return ns;
}

typedef struct {
	int d0, d1, d2;
	const float *in;
	float *out;
} reorder_ctx;

static void reorder_range(size_t lo, size_t hi, void *c)
{
	const reorder_ctx *r = (const reorder_ctx *)c;
	size_t j;
	int i, k;
	for (j = lo; j < hi; ++j)
		for (k = 0; k < r->d0; ++k)
			for (i = 0; i < r->d2; ++i)
				r->out[(j * r->d0 + k) * r->d2 + i] = r->in[((size_t)k * r->d1 + j) * r->d2 + i];
}

void irl_reorder(int d0, int d1, int d2, const float *in, float *out)
{
	reorder_ctx c = {d0, d1, d2, in, out};
	const size_t row = (size_t)d0 * d2;
	irl_parallel_for((size_t)d1, row ? (IRL_PAR_GRAIN + row - 1) / row : 1, reorder_range, &c);
}
