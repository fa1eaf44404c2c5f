/*
 * irl_osem.c -- IrlOsem and the OSEM driver of libirl_b200.
 *
 * Control flow, argument handling, in-place mutation of the caller's arrays,
 * hooks and callbacks follow libirl irlosem.c:22-290 and
 * osemrecon.c:557-897.  The per-subset work runs on the GPU through
 * include/irlcu.h: every view of a subset is projected, compared with the
 * data and backprojected in one batched stage, and the clamped accumulation
 * keeps libirl's view order.
 *
 * IrlOsem = IrlOsemBegin (set-up, normalisation images, iteration-0
 * callback) + IrlOsemIterate (the iterations) + IrlOsemEnd (result copy and
 * release); the three are exported (include/irl_b200.h).
 */
#include <pthread.h>
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "irl_b200.h"
#include "irl_err.h"
#include "irl_geom.h"
#include "irl_host.h"
#include "irlcu.h"

irl_hook_fn g_irl_hooks[6] = {NULL, NULL, NULL, NULL, NULL, NULL};
void *g_irl_hook_ctx = NULL;
sAdvOptions g_irl_adv = {1, 0};

int OsemSetAdvOptions(sAdvOptions *pOpt)
{
	memcpy(&g_irl_adv, pOpt, sizeof(sAdvOptions));
	return 1;
}
#define HOOK_SETTER(name, idx)                                                   \
	int name(void (*f)(sOsemData *, void *), void *ctx)                          \
	{                                                                            \
		g_irl_hooks[idx] = f;                                                    \
		g_irl_hook_ctx = ctx;                                                    \
		return 1;                                                                \
	}
HOOK_SETTER(OsemSetPrevIterHook, HOOK_PREV_ITER)
HOOK_SETTER(OsemSetPostIterHook, HOOK_POST_ITER)
HOOK_SETTER(OsemSetPrevSubsetHook, HOOK_PREV_SUBSET)
HOOK_SETTER(OsemSetPostSubsetHook, HOOK_POST_SUBSET)
HOOK_SETTER(OsemSetPrevAngleHook, HOOK_PREV_ANGLE)
HOOK_SETTER(OsemSetPostAngleHook, HOOK_POST_ANGLE)

char *pchIrlErrorString(void) { return (char *)irl_last_error(); }

static double now_s(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* set-up step timings at message level 6, from the start of IrlOsemBegin */
static double g_mark_t0;
static void mark(const char *what)
{
	irl_msg(6, "  mark %s (%.4f s)\n", what, now_s() - g_mark_t0);
}

/* ---------------------------------------------------------------- session */

typedef struct {
	int open;
	irl_parms p;
	irl_view *views;
	irl_esse_host esse;
	FILE *logfp, *msgfp;
	float *recon;            /* caller's image: internal layout during the run */
	float *prjscat;          /* host copy of the stored scatter projections */
	float *tmp;              /* external-layout callback image */
	float *norm_host, *upd_host;
	void (*cb)(int, float *);
	int use_scatest;
	int *ang, ns, per, max_batch;
	int it;                  /* last completed iteration */
	int this_srf, next_srf;
	irlcu_view_parm *vp;
	sOsemData hd;            /* hook data (osemhooks.h:18-27) */
	int hook_norm;           /* subset whose norm the hooks see, or -1 */
	size_t vox, prjn;
	irlcu_sur *sur;          /* learned scatter surrogate, or NULL */
	float *sur_nrmse;        /* per view, after the first scatter iteration */
	int sur_pending;         /* NRMSE check still to run */
} osem_session;

/* learned scatter surrogate for the next sessions (IrlSetScatterSurrogate) */
static char *g_sur_fname = NULL;
static float g_sur_fallback = 0.02f;

static osem_session S;

static void session_close(void)
{
	if (S.sur != NULL) {
		irlcu_set_surrogate(NULL, NULL);
		irlcu_sur_destroy(S.sur);
	}
	free(S.sur_nrmse);
	irlcu_shutdown();
	irl_free_run_tables();
	free(S.views);
	free(S.prjscat);
	free(S.tmp);
	free(S.norm_host);
	free(S.upd_host);
	free(S.ang);
	free(S.vp);
	irl_esse_free(&S.esse);
	if (S.logfp != NULL) {
		fclose(S.logfp);
		irl_set_log_file(NULL);
	}
	if (S.msgfp != NULL) {
		fclose(S.msgfp);
		irl_set_msg_file(NULL);
	}
	memset(&S, 0, sizeof(S));
}

/* copies the device state to the hook mirrors, calls the hook, copies back */
static void hook_call(int which)
{
	irl_hook_fn f = g_irl_hooks[which];
	if (f == NULL)
		return;
	irl_cu(irlcu_download(IRLCU_BUF_EST, 0, S.hd.pfEst, S.vox), "hook");
	irl_cu(irlcu_download(IRLCU_BUF_UPDATE, 0, S.hd.pfUpdate, S.vox), "hook");
	if (S.hook_norm >= 0)
		irl_cu(irlcu_download(IRLCU_BUF_NORM, S.hook_norm, S.hd.pfNorm, S.vox), "hook");
	if (S.hd.pfSct != NULL)
		irl_cu(irlcu_download(IRLCU_BUF_PRJSCAT, 0, S.hd.pfSct, S.prjn), "hook");
	f(&S.hd, g_irl_hook_ctx);
	irl_cu(irlcu_upload(IRLCU_BUF_EST, 0, S.hd.pfEst, S.vox), "hook");
	irl_cu(irlcu_upload(IRLCU_BUF_UPDATE, 0, S.hd.pfUpdate, S.vox), "hook");
	if (S.hd.pfSct != NULL)
		irl_cu(irlcu_upload(IRLCU_BUF_PRJSCAT, 0, S.hd.pfSct, S.prjn), "hook");
}

static void norm_file(const char *base, int s, const float *img, size_t vox, int del)
{
	char *name = (char *)irl_malloc(strlen(base) + 40, "norm name");
	FILE *fp;
	sprintf(name, "%s.norm.%d.dat", base, s);
	if (del) {
		unlink(name);
		free(name);
		return;
	}
	fp = fopen(name, "wb");
	if (fp == NULL) {
		free(name);
		irl_fatal(IRL_E_IO, "writedat", "IO error opening to %s.norm.%d.dat for writing", base, s);
	}
	if (fwrite(img, sizeof(float), vox, fp) != vox || ferror(fp)) {
		fclose(fp);
		free(name);
		irl_fatal(IRL_E_IO, "writedat", "IO error while writing norm image %d", s);
	}
	fclose(fp);
	free(name);
}

/* opens the log and message files (irlosem.c:113-141) */
static void open_logs(const char *logname, const char *msgname, int level, FILE **plog, FILE **pmsg)
{
	*plog = *pmsg = NULL;
	if (logname == NULL) {
		irl_set_log_file(NULL);
	} else if (strcmp(logname, "stderr") == 0) {
		irl_set_log_file(stderr);
	} else {
		*plog = fopen(logname, "w");
		irl_set_log_file(*plog);
		if (*plog == NULL)
			irl_fatal(IRL_E_IO, "IrlOsem", "Error opening log file %s", logname);
	}
	irl_set_msg_level(level);
	if (msgname == NULL) {
		irl_set_msg_file(NULL);
	} else if (strcmp(msgname, "stderr") == 0) {
		irl_set_msg_file(stderr);
	} else {
		*pmsg = fopen(msgname, "w");
		irl_set_msg_file(*pmsg);
		if (*pmsg == NULL)
			irl_fatal(IRL_E_IO, "IrlOsem", "Error opening messages file %s", msgname);
	}
}

typedef struct {
	float *p;
	float s;
} fspan;

static void zero_neg_range(size_t lo, size_t hi, void *c)
{
	float *p = ((fspan *)c)->p;
	size_t i;
	for (i = lo; i < hi; ++i)
		if (p[i] < 0.0f)
			p[i] = 0.0f;
}

static void scale_range(size_t lo, size_t hi, void *c)
{
	float *p = ((fspan *)c)->p, s = ((fspan *)c)->s;
	size_t i;
	for (i = lo; i < hi; ++i)
		p[i] *= s;
}

static void zero_neg(float *p, size_t n)
{
	fspan c = {p, 0.0f};
	irl_parallel_for(n, IRL_PAR_GRAIN, zero_neg_range, &c);
}

static void scale_f(float *p, size_t n, float s)
{
	fspan c = {p, s};
	irl_parallel_for(n, IRL_PAR_GRAIN, scale_range, &c);
}

/* device context, rotation tables and column masks: everything that
   depends only on the geometry and the views */
void irl_device_geometry(irl_parms *p, irl_view *views, int fast_rotate, int max_batch)
{
	irlcu_geom g;
	float *angles = (float *)irl_malloc(sizeof(float) * p->nviews, "angles");
	unsigned char *mask = (unsigned char *)irl_malloc((size_t)p->nviews * p->n, "column masks");
	unsigned char *m1 = (unsigned char *)irl_malloc(p->n, "mask"), *m2 = (unsigned char *)irl_malloc(p->n, "mask");
	int a, i, rc;
	g.n = p->n;
	g.nz = p->nz;
	g.nviews = p->nviews;
	g.fast_rotate = fast_rotate;
	g.max_batch = max_batch;
	for (a = 0; a < p->nviews; ++a) {
		angles[a] = views[a].angle;
		/* PWid = PixelWidth / BinWidth = 1 (IrlSetup.c:65-66) */
		irl_measured_columns(views[a].left, p->pix / p->pix, p->n, p->nbins, m1);
		irl_norm_columns(views[a].left, views[a].right, p->pix / p->pix, p->n, p->nbins, m2);
		for (i = 0; i < p->n; ++i)
			mask[(size_t)a * p->n + i] = (unsigned char)(m1[i] | (m2[i] << 1));
	}
	rc = irlcu_init(&g);
	if (rc == 0)
		rc = irlcu_set_angles(angles);
	if (rc == 0)
		rc = irlcu_set_column_mask(mask);
	free(angles);
	free(mask);
	free(m1);
	free(m2);
	irl_cu(rc, "device set-up");
}

/* DRF tables and the ESSE kernel spectra */
void irl_device_tables(irl_parms *p, irl_view *views, const irl_esse_host *esse)
{
	if (p->model & MODEL_DRF)
		irl_upload_drf(p, views, 0, NULL);
	if ((p->model & MODEL_SRF) && esse != NULL && esse->on) {
		irlcu_esse e;
		e.kx = esse->kx;
		e.ky = esse->ky;
		e.kz = esse->kz;
		e.collapse = esse->collapse;
		e.nterms = esse->nterms;
		e.mu0 = esse->mu0;
		e.mu_avg = esse->mu_avg;
		e.pix = esse->pix;
		e.cntr_pix_fac = esse->cntr_pix_fac;
		e.noffs = esse->noffs;
		e.ndepths = esse->ndepths;
		e.krnl = esse->krnl_file;
		e.mu = esse->mu_file;
		e.kmu_outside = esse->kmu_outside;
		irl_cu(irlcu_set_esse(&e), "ESSE set-up");
	} else if (p->model & MODEL_SRF) {
		irl_cu(irlcu_set_esse(NULL), "ESSE set-up");
	}
}

/* the whole device set-up of IrlGenprj, from an attenuation map already
   in the internal layout */
void irl_device_setup(irl_parms *p, irl_view *views, const float *atn_internal, const irl_esse_host *esse,
	int fast_rotate, int max_batch)
{
	irl_device_geometry(p, views, fast_rotate, max_batch);
	if (atn_internal != NULL) {
		irl_cu(irlcu_upload(IRLCU_BUF_ATN, 0, atn_internal, (size_t)p->n * p->nz * p->n), "device set-up");
		irl_cu(irlcu_prepare_attenuation((p->model & MODEL_SRF) != 0), "device set-up");
	}
	irl_device_tables(p, views, esse);
}

/* normalisation images of every subset (psComputeNormImages,
   osemrecon.c:223-343), into the norm buffers irlcu_alloc_norm made */
static void compute_norms(void)
{
	irl_parms *p = &S.p;
	float *vt = (float *)irl_malloc(sizeof(float) * S.per, "view times");
	float *img = NULL;
	int s, m;
	double t0 = now_s();
	for (s = 0; s < S.ns; ++s) {
		for (m = 0; m < S.per; ++m)
			vt[m] = S.views[S.ang[s * S.per + m]].view_time;
		irl_cu(irlcu_norm_subset(S.per, S.ang + s * S.per, vt, p->bck_model, s), "ComputeNormImages");
		if (p->norm_base != NULL) {
			if (img == NULL)
				img = (float *)irl_malloc(sizeof(float) * S.vox, "norm image");
			irl_cu(irlcu_download(IRLCU_BUF_NORM, s, img, S.vox), "ComputeNormImages");
			norm_file(p->norm_base, s, img, S.vox, 0);
		}
	}
	free(vt);
	free(img);
	irl_msg(5, "Done Computing Norm Matrix (%.3f s)\n", now_s() - t0);
}

/* the surrogate network of this session from g_sur_fname: "IRLSUR01",
   uint32 parameter count, float32 parameters (little-endian) */
static void sur_load(void)
{
	char magic[8];
	unsigned int n = 0;
	float *w;
	size_t want;
	FILE *fp = fopen(g_sur_fname, "rb");
	if (fp == NULL)
		irl_fatal(IRL_E_IO, "ScatterSurrogate", "cannot open %s", g_sur_fname);
	if (fread(magic, 1, 8, fp) != 8 || memcmp(magic, "IRLSUR01", 8) != 0 || fread(&n, 4, 1, fp) != 1) {
		fclose(fp);
		irl_fatal(IRL_E_IO, "ScatterSurrogate", "%s is not a surrogate weights file", g_sur_fname);
	}
	irl_cu(irlcu_sur_create(S.max_batch, 1, &S.sur), "ScatterSurrogate");
	want = irlcu_sur_nparams(S.sur);
	if (n != want) {
		fclose(fp);
		irl_fatal(IRL_E_VALUE, "ScatterSurrogate", "%s holds %u parameters, the network has %zu", g_sur_fname, n,
			want);
	}
	w = (float *)irl_malloc(sizeof(float) * want, "surrogate weights");
	if (fread(w, sizeof(float), want, fp) != want) {
		free(w);
		fclose(fp);
		irl_fatal(IRL_E_IO, "ScatterSurrogate", "%s is truncated", g_sur_fname);
	}
	fclose(fp);
	irl_cu(irlcu_sur_set_weights(S.sur, w, want), "ScatterSurrogate");
	free(w);
	S.sur_nrmse = (float *)irl_calloc(sizeof(float) * S.p.nviews, "surrogate NRMSE");
	S.sur_pending = 1;
}

/* after the first scatter iteration (ESSE on every view): per-view NRMSE of
   the surrogate against ESSE on the current estimate; views above the
   fallback threshold keep ESSE, the others use the network from now on */
static void sur_check(int model)
{
	unsigned char *flags;
	int *all;
	int v, nflag = 0;
	all = (int *)irl_malloc(sizeof(int) * S.p.nviews, "surrogate views");
	for (v = 0; v < S.p.nviews; ++v)
		all[v] = v;
	irl_cu(irlcu_sur_check(S.sur, S.p.nviews, all, model, S.sur_nrmse), "ScatterSurrogate");
	free(all);
	flags = (unsigned char *)irl_calloc(S.p.nviews, "surrogate flags");
	for (v = 0; v < S.p.nviews; ++v)
		if (!(S.sur_nrmse[v] <= g_sur_fallback)) {
			flags[v] = 1;
			++nflag;
		}
	irl_cu(irlcu_set_surrogate(S.sur, flags), "ScatterSurrogate");
	free(flags);
	S.sur_pending = 0;
	irl_msg(4, "scatter surrogate: %d of %d views above NRMSE %.3f keep ESSE\n", nflag, S.p.nviews,
		g_sur_fallback);
}

int IrlSetScatterSurrogate(const char *pchWeightsFname, float fFallbackNrmse)
{
	free(g_sur_fname);
	g_sur_fname = pchWeightsFname != NULL ? irl_strdup(pchWeightsFname) : NULL;
	g_sur_fallback = fFallbackNrmse > 0 ? fFallbackNrmse : 0.02f;
	return 0;
}

int IrlGetScatterSurrogateNrmse(float *pfNrmse, int iNumViews)
{
	int v;
	if (!S.open || S.sur == NULL || S.sur_pending || pfNrmse == NULL || iNumViews != S.p.nviews)
		return IRL_E_VALUE;
	for (v = 0; v < iNumViews; ++v)
		pfNrmse[v] = S.sur_nrmse[v];
	return 0;
}

/* Host work of the set-up that runs on helper threads while the device
   builds its tables.  Neither allocates nor raises an error (a failed
   upload is returned in prj_job.rc).
   - prj_job: libirl's serial float sum of the projections (the initial
     estimate's mean, initial_est.c:89-95), then the clamp of the caller's
     projections (irlosem.c:205), then their upload beside the queued
     kernels; the sum reads them before the clamp, as libirl's does.
   - atn_job: the caller's attenuation map reordered in place to the
     internal layout (irlosem.c:170-176), through the session's temporary
     volume.  It starts once the device has its own copy of the map. */
typedef struct {
	float *prj;
	size_t count;
	int need_sum;
	float sum;
	int rc;
} prj_job;

typedef struct {
	int n, nz;
	float *atn, *tmp;
} atn_job;

static void *prj_thread(void *arg)
{
	prj_job *j = (prj_job *)arg;
	if (j->need_sum)
		j->sum = irl_projection_sum(j->prj, j->count);
	zero_neg(j->prj, j->count);
	j->rc = irlcu_upload_now(IRLCU_BUF_PRJ, 0, j->prj, j->count);
	return NULL;
}

static void *atn_thread(void *arg)
{
	atn_job *j = (atn_job *)arg;
	const size_t vox = (size_t)j->n * j->nz * j->n;
	irl_reorder(j->nz, j->n, j->n, j->atn, j->tmp);
	memcpy(j->atn, j->tmp, sizeof(float) * vox);
	return NULL;
}

/* runs fn(arg) on a new thread, or here when none can be started */
static int start_helper(pthread_t *th, void *(*fn)(void *), void *arg)
{
	if (pthread_create(th, NULL, fn, arg) == 0)
		return 1;
	fn(arg);
	return 0;
}

/* The set-up keeps the device busy while the host works: the device gets
   the attenuation map first (transposed, scaled and clamped on the device)
   and builds the per-view tables while the host reads the scatter kernel
   and the DRF tables; the normalisation images are queued before the host
   computes the initial estimate and the caller-visible changes of its
   arrays.  The results are those of libirl's serial order
   (irlosem.c:150-243): every step reads what it read there. */
int IrlOsemBegin(IrlParms_t *ip, Options_t *op, PrjView_t *pv, char *drf_fname, char *krnl_fname,
	void (*cb)(int, float *), float *scatest, float *atn, float *prj, float *recon, char *logname, char *msgname)
{
	jmp_buf env;
	int err, m;
	double t0 = now_s();
	g_mark_t0 = t0;
	/* static: read after a longjmp back to the trap (the library keeps one
	   session per process) */
	static prj_job pjob;
	static atn_job ajob;
	static pthread_t prj_th, atn_th;
	static volatile int prj_running, atn_running;
	if (S.open)
		session_close();
	memset(&S, 0, sizeof(S));
	S.open = 1;
	S.hook_norm = -1;
	if ((err = setjmp(env)) != 0) {
		if (prj_running)
			pthread_join(prj_th, NULL);
		if (atn_running)
			pthread_join(atn_th, NULL);
		prj_running = atn_running = 0;
		fprintf(stderr, "FATAL ERROR Trapped: err_num=%d\nErrMsg=%s\n", err, irl_last_error());
		irl_msg(1, "aborted\n");
		irl_untrap();
		session_close();
		return err;
	}
	irl_trap(&env);
	prj_running = atn_running = 0;
	open_logs(logname, msgname, op->iMsgLevel, &S.logfp, &S.msgfp);
	irl_setup_parms(ip, op, atn, krnl_fname, &S.p);
	S.vox = (size_t)S.p.n * S.p.nz * S.p.n;
	S.prjn = (size_t)S.p.n * S.p.nz * S.p.nviews;
	S.views = irl_setup_views(ip, pv);
	if ((S.p.model & MODEL_SRF) && atn == NULL)
		irl_fatal(IRL_E_VALUE, "SrfSetup", "scatter modelling needs an attenuation map");
	S.tmp = (float *)irl_malloc(sizeof(float) * S.vox, "IrlOsem:Temp");
	S.per = S.p.ang_per_subset;
	S.max_batch = S.per > 32 ? 32 : S.per;
	S.ns = irl_compute_subsets(S.p.nviews, S.per, &S.ang);
	mark("parms and views");

	/* device: geometry, then the attenuation map and its per-view tables
	   (queued; they build while the host reads the kernel and DRF files) */
	irl_device_geometry(&S.p, S.views, g_irl_adv.bFastRotate, S.max_batch);
	if (prj == NULL)
		irl_fatal(IRL_E_VALUE, "IrlOsem", "no projections given");
	pjob.prj = prj;
	pjob.count = S.prjn;
	pjob.need_sum = !op->bReconIsInitEst;
	pjob.sum = 0.0f;
	pjob.rc = 0;
	prj_running = start_helper(&prj_th, prj_thread, &pjob);
	if (atn != NULL) {
		irl_cu(irlcu_upload_external(IRLCU_BUF_ATN, atn, ip->fAtnScaleFac, 1), "IrlOsem");
		irl_cu(irlcu_prepare_attenuation((S.p.model & MODEL_SRF) != 0), "IrlOsem");
		ajob.n = S.p.n;
		ajob.nz = S.p.nz;
		ajob.atn = atn;
		ajob.tmp = S.tmp;
		atn_running = start_helper(&atn_th, atn_thread, &ajob);
	}
	mark("attenuation queued");
	if (S.p.model & MODEL_SRF)
		irl_esse_prepare(krnl_fname, &S.p, ip->SrfCollapseFac, &S.esse);
	irl_msg(5, "Done scatter kernel (%.3f s)\n", now_s() - t0);
	{
		irl_detector *d;
		/* libirl calls vSetupDrfTables unconditionally (irlosem.c:158-160) */
		irl_setup_drf_tables(&S.p, op, S.views, drf_fname, &d);
	}
	irl_msg(5, "Done DRF tables (%.3f s)\n", now_s() - t0);
	irl_device_tables(&S.p, S.views, &S.esse);
	irl_msg(5, "Done device set-up (%.3f s)\n", now_s() - t0);

	if ((S.p.prj_model & MODEL_SRF) && S.p.srf_iters > 0) {
		S.prjscat = (float *)irl_calloc(sizeof(float) * S.prjn, "OsemRecon:PrjScatEst");
		irl_cu(irlcu_zero(IRLCU_BUF_PRJSCAT, 0), "IrlOsem");
	}
	irl_cu(irlcu_alloc_norm(S.ns), "OsemRecon");
	{
		/* every subset's views on the device, for whole-iteration launches */
		const int tot = S.ns * S.per;
		irlcu_view_parm *all = (irlcu_view_parm *)irl_calloc(sizeof(irlcu_view_parm) * tot, "subset views");
		int i;
		for (i = 0; i < tot; ++i) {
			all[i].view_time = S.views[S.ang[i]].view_time;
			all[i].sensitivity = S.views[S.ang[i]].sensitivity;
		}
		m = irlcu_set_subsets(S.ns, S.per, S.ang, all);
		free(all);
		irl_cu(m, "OsemRecon");
	}
	compute_norms();
	mark("norms queued");

	/* host: the initial estimate and the caller-visible changes of the
	   attenuation map and the scatter estimate, while the norms run */
	if (atn_running) {
		pthread_join(atn_th, NULL);
		atn_running = 0;
	}
	if (prj_running) {
		pthread_join(prj_th, NULL);
		prj_running = 0;
	}
	irl_cu(pjob.rc, "IrlOsem");
	if (!op->bReconIsInitEst) {
		irl_initial_estimate_sum(&S.p, op->bUseContourSupport, op->fAtnMapThresh, S.views, pjob.sum, atn,
			recon);
	} else {
		irl_reorder(S.p.nz, S.p.n, S.p.n, recon, S.tmp);
		memcpy(recon, S.tmp, sizeof(float) * S.vox);
	}
	mark("initial estimate");
	if (atn != NULL) {
		if (ip->fAtnScaleFac > 0 && ip->fAtnScaleFac != 1.0)
			scale_f(atn, S.vox, ip->fAtnScaleFac);
		zero_neg(atn, S.vox);
	}
	if (scatest != NULL) {
		if (ip->fScatEstFac > 0 && ip->fScatEstFac != 1.0)
			scale_f(scatest, S.prjn, ip->fScatEstFac);
		zero_neg(scatest, S.prjn);
	}
	zero_neg(recon, S.vox);
	if (cb != NULL) {
		irl_reorder(S.p.n, S.p.nz, S.p.n, recon, S.tmp);
		cb(0, S.tmp);
	}
	irl_msg(5, "Done host set-up (%.3f s)\n", now_s() - t0);
	/* beside the norms still running: no queued kernel reads the estimate */
	irl_cu(irlcu_upload_now(IRLCU_BUF_EST, 0, recon, S.vox), "IrlOsem");
	if (scatest != NULL)
		irl_cu(irlcu_upload(IRLCU_BUF_SCATEST, 0, scatest, S.prjn), "IrlOsem");
	S.use_scatest = scatest != NULL;
	S.recon = recon;
	S.cb = cb;
	irl_msg(5, "Done Initialization (%.3f s)\n", now_s() - t0);
	if (g_sur_fname != NULL && (S.p.prj_model & MODEL_SRF) && S.p.srf_iters > 0)
		sur_load();
	for (m = 0; m < 6; ++m)
		if (g_irl_hooks[m] != NULL && S.norm_host == NULL) {
			S.norm_host = (float *)irl_calloc(sizeof(float) * S.vox, "norm mirror");
			S.upd_host = (float *)irl_calloc(sizeof(float) * S.vox, "update mirror");
		}
	S.hd.pfEst = recon;
	S.hd.pfSct = S.prjscat;
	S.hd.pfNorm = S.norm_host;
	S.hd.pfUpdate = S.upd_host;
	if (S.p.prj_model & MODEL_SRF)
		S.next_srf = S.p.start_iteration + 1 <= S.p.srf_iters;
	S.p.start_iteration = g_irl_adv.iStartIteration;
	S.it = S.p.start_iteration;
	S.vp = (irlcu_view_parm *)irl_calloc(sizeof(irlcu_view_parm) * S.per, "view parameters");
	mark("set-up returns");
	irl_untrap();
	return 0;
}

static int any_hook(void)
{
	int h;
	for (h = 0; h < 6; ++h)
		if (g_irl_hooks[h] != NULL)
			return 1;
	return 0;
}

/* the iteration callback with the snapshot of iteration it */
static void deliver_snapshot(int it)
{
	float *img = NULL;
	irl_cu(irlcu_snapshot_end(it & 1, &img), "OsemRecon");
	S.cb(it, img);
}

/* one OSEM iteration: subset loop of osemrecon.c:637-883; with deliver_cb
   the iteration callback gets the result before this returns */
static void one_iteration(int deliver_cb)
{
	irl_parms *p = &S.p;
	int it = S.it + 1, s = 0, m, model = p->prj_model, mode = 0;
	int angle_hooks = g_irl_hooks[HOOK_PREV_ANGLE] || g_irl_hooks[HOOK_POST_ANGLE];
	double ti = now_s();
	S.hd.iIterationIdx = it;
	hook_call(HOOK_PREV_ITER);
	if (p->prj_model & MODEL_SRF) {
		S.this_srf = S.next_srf;
		S.next_srf = (it == p->iterations) ? S.this_srf : (it + 1 <= p->srf_iters);
		model = S.this_srf ? p->prj_model : (p->prj_model & ~MODEL_SRF);
		mode = !S.this_srf ? 1 : (!S.next_srf ? 2 : 0);
	}
	if (!angle_hooks && !g_irl_hooks[HOOK_PREV_SUBSET] && !g_irl_hooks[HOOK_POST_SUBSET]) {
		/* no host work between subsets: the whole iteration in one call
		   (replayed from a CUDA graph after its first runs) */
		irl_cu(irlcu_osem_iteration(model, p->bck_model, S.use_scatest, mode), "OsemRecon");
		S.hook_norm = S.ns - 1;
		s = S.ns;
	}
	for (s = s == S.ns ? S.ns : 0; s < S.ns; ++s) {
		const int *va = S.ang + s * S.per;
		S.hd.iSubsetIdx = s;
		hook_call(HOOK_PREV_SUBSET);
		for (m = 0; m < S.per; ++m) {
			S.vp[m].view_time = S.views[va[m]].view_time;
			S.vp[m].sensitivity = S.views[va[m]].sensitivity;
			S.vp[m].scat_mode = mode;
		}
		if (angle_hooks) {
			for (m = 0; m < S.per; ++m) {
				S.hd.iAngleIdx = va[m];
				hook_call(HOOK_PREV_ANGLE);
				irl_cu(irlcu_osem_subset(1, va + m, S.vp + m, model, p->bck_model, s, S.use_scatest,
					       m == S.per - 1, m > 0),
					"OsemRecon");
				if (m == S.per - 1)
					S.hook_norm = s;
				hook_call(HOOK_POST_ANGLE);
			}
		} else {
			int m0;
			for (m0 = 0; m0 < S.per; m0 += S.max_batch) {
				int nb = S.per - m0 < S.max_batch ? S.per - m0 : S.max_batch;
				irl_cu(irlcu_osem_subset(nb, va + m0, S.vp + m0, model, p->bck_model, s, S.use_scatest,
					       m0 + nb >= S.per, m0 > 0),
					"OsemRecon");
			}
			S.hook_norm = s;
		}
		hook_call(HOOK_POST_SUBSET);
	}
	hook_call(HOOK_POST_ITER);
	if (S.sur != NULL && S.sur_pending && S.this_srf)
		sur_check(model);
	/* bCheckIfSaveIteration is true for every iteration with libirl's
	   SaveInterval of 1 (IrlSetup.c:87-88, osemrecon.c:513-555) */
	if (deliver_cb && S.cb != NULL) {
		irl_cu(irlcu_download_external(IRLCU_BUF_EST, S.tmp), "OsemRecon");
		S.cb(it, S.tmp);
	}
	S.it = it;
	irl_msg(4, "----Done iteration %d (%.3f s)\n", it, now_s() - ti);
}

int IrlOsemIterate(int niter)
{
	jmp_buf env;
	int err, k;
	if (!S.open)
		return IRL_E_VALUE;
	if ((err = setjmp(env)) != 0) {
		fprintf(stderr, "FATAL ERROR Trapped: err_num=%d\nErrMsg=%s\n", err, irl_last_error());
		irl_untrap();
		session_close();
		return err;
	}
	irl_trap(&env);
	if (S.cb == NULL || any_hook()) {
		for (k = 0; k < niter && S.it < S.p.iterations; ++k)
			one_iteration(1);
	} else {
		/* the callback of iteration i runs while iteration i + 1 computes:
		   its estimate is snapshotted on the device after iteration i and
		   copied to pinned memory on a stream of its own
		   (irlcu_snapshot_*); the callback still sees every iteration's
		   result, in order, before this call returns */
		int pending = -1;
		for (k = 0; k < niter && S.it < S.p.iterations; ++k) {
			one_iteration(0);
			irl_cu(irlcu_snapshot_begin(S.it & 1), "OsemRecon");
			if (pending >= 0)
				deliver_snapshot(pending);
			pending = S.it;
		}
		if (pending >= 0)
			deliver_snapshot(pending);
	}
	irl_untrap();
	return 0;
}

int IrlOsemEnd(float *recon)
{
	jmp_buf env;
	int err;
	if (!S.open)
		return 0;
	if ((err = setjmp(env)) != 0) {
		irl_untrap();
		session_close();
		return err;
	}
	irl_trap(&env);
	if (S.p.norm_base != NULL) {
		int s;
		for (s = 0; s < S.ns; ++s)
			norm_file(S.p.norm_base, s, NULL, 0, 1);
	}
	g_mark_t0 = now_s();
	if (recon != NULL)
		irl_cu(irlcu_download_external(IRLCU_BUF_EST, recon), "IrlOsem");
	mark("end: image download");
	irl_untrap();
	session_close();
	return 0;
}

/* ----------------------------------------------------------------- batch */

/* a reconstruction set aside while another one is current: its host
   session, its device context and its per-call run tables */
typedef struct {
	osem_session s;
	void *dev;
	irl_run_tables run;
} parked_session;

static parked_session *session_park(void)
{
	parked_session *h = (parked_session *)irl_malloc(sizeof(parked_session), "batch session");
	h->s = S;
	memset(&S, 0, sizeof(S));
	h->dev = irlcu_ctx_detach();
	irl_run_tables_park(&h->run);
	return h;
}

static void session_unpark(parked_session *h)
{
	S = h->s;
	(void)irlcu_ctx_attach(h->dev);  /* every other context is parked */
	irl_run_tables_unpark(&h->run);
	free(h);
}

/* ends parked problem p (result copy unless a problem failed) */
static int batch_end(parked_session **h, IrlOsemProblem_t *pp, int p, int err)
{
	int e;
	if (h[p] == NULL)
		return 0;
	session_unpark(h[p]);
	h[p] = NULL;
	e = IrlOsemEnd(err ? NULL : pp[p].pfReconImage);
	if (!pp[p].iStatus)
		pp[p].iStatus = e;
	return e;
}

/* problems of a batch in flight at once (IRL_BATCH_DEPTH, default 4) */
static int batch_depth(void)
{
	const char *e = getenv("IRL_BATCH_DEPTH");
	int d = e != NULL ? atoi(e) : 4;
	return d < 1 ? 1 : d > 64 ? 64 : d;
}

/* a generous estimate of one problem's device memory: the per-view
   attenuation tables (three with the scatter model), the norm images and
   the batch work space, in volumes */
static double batch_need_bytes(const IrlOsemProblem_t *q)
{
	const IrlParms_t *ip = q->psIrlParms;
	const double vox = (double)ip->NumPixels * ip->NumPixels * ip->NumSlices;
	return 4.0 * vox * (3.0 * ip->NumViews + 96.0);
}

int IrlOsemBatch(int nprob, IrlOsemProblem_t *pp)
{
	jmp_buf env;
	parked_session **h = NULL;
	int p, m, err = 0, trials = 1, graphs = 1, depth, oldest = 0;
	if ((err = setjmp(env)) != 0) {
		irl_untrap();
		return err;
	}
	irl_trap(&env);
	if (nprob <= 0 || pp == NULL)
		irl_fatal(IRL_E_VALUE, "IrlOsemBatch", "no problems given");
	for (m = 0; m < 6; ++m)
		if (g_irl_hooks[m] != NULL)
			irl_fatal(IRL_E_VALUE, "IrlOsemBatch", "hooks are not supported in a batch");
	if (g_irl_extra_nviews > 0 || g_irl_dets != NULL || g_irl_acq_times != NULL || g_irl_det_nums != NULL)
		irl_fatal(IRL_E_VALUE, "IrlOsemBatch",
			"per-call view or detector data (iSetupExtraPrjViewData / iSetupDetectors) is pending");
	if (S.open)
		irl_fatal(IRL_E_VALUE, "IrlOsemBatch", "an IrlOsemBegin session is open");
	h = (parked_session **)irl_calloc(sizeof(parked_session *) * nprob, "batch sessions");
	irl_untrap();
	trials = irlcu_shape_trials(0);  /* no host waits inside the pipelined batch */
	graphs = irlcu_iteration_graphs(0);  /* eager iterations: faster with problems in flight */
	depth = batch_depth();
	/* pipelined: problem p is set up and all its iterations are enqueued
	   (asynchronous device work on its own stream); the host then sets up
	   p + 1 while the device runs p and the problems before it.  Up to
	   `depth` problems are in flight; the oldest is ended (waiting for its
	   device work) before a new one would exceed that, or the device
	   memory */
	for (p = 0; p < nprob && !err; ++p) {
		IrlOsemProblem_t *q = pp + p;
		/* the oldest problems end first while the next one might not fit */
		while (oldest < p && !err) {
			size_t fr = 0;
			if (p - oldest < depth && (irlcu_mem_info(&fr, NULL) != 0 || (double)fr >= batch_need_bytes(q)))
				break;
			{
				const int e = batch_end(h, pp, oldest++, err);
				if (!err)
					err = e;
			}
		}
		if (err)
			break;
		q->iStatus = IrlOsemBegin(q->psIrlParms, q->psOptions, q->psViews, q->pchDrfTabFname,
			q->pchScatKrnlFname, NULL, q->pfScatterEstimate, q->pfAtnMap, q->pfPrjImage, q->pfReconImage,
			NULL, NULL);
		if (q->iStatus) {
			err = q->iStatus;
			break;
		}
		{
			const int e = IrlOsemIterate(S.p.iterations);
			if (e) {  /* IrlOsemIterate closed the session */
				q->iStatus = err = e;
				break;
			}
		}
		h[p] = session_park();
	}
	for (p = 0; p < nprob; ++p) {
		const int e = batch_end(h, pp, p, err);
		if (!err)
			err = e;
	}
	free(h);
	irlcu_shape_trials(trials);
	irlcu_iteration_graphs(graphs);
	return err;
}

int IrlOsem(IrlParms_t *ip, Options_t *op, PrjView_t *pv, char *drf_fname, char *krnl_fname,
	void (*cb)(int, float *), float *scatest, float *atn, float *prj, float *recon, char *logname, char *msgname)
{
	int err = IrlOsemBegin(ip, op, pv, drf_fname, krnl_fname, cb, scatest, atn, prj, recon, logname, msgname);
	if (err)
		return err;
	err = IrlOsemIterate(S.p.iterations);
	if (err)
		return err;
	return IrlOsemEnd(recon);
}
