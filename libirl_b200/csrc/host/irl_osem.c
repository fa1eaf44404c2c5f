/*
 * irl_osem.c -- IrlOsem and the OSEM driver of libirl_b200.
 *
 * Control flow, argument handling, in-place mutation of the caller's arrays,
 * hooks and callbacks follow libirl irlosem.c:22-290 and
 * osemrecon.c:557-897.  The per-subset work runs on the GPU through
 * include/irlcu.h: every view of a subset is projected, compared with the
 * data and backprojected in one batched stage, and the clamped accumulation
 * keeps libirl's view order.
 */
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

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

/* host mirrors handed to hooks (osemhooks.h:18-27) */
typedef struct {
	sOsemData d;
	int any;
	size_t vox, prjn;
	int norm_subset;
} hook_state;

static void hook_call(hook_state *h, int which)
{
	irl_hook_fn f = g_irl_hooks[which];
	if (f == NULL)
		return;
	irl_cu(irlcu_download(IRLCU_BUF_EST, 0, h->d.pfEst, h->vox), "hook");
	irl_cu(irlcu_download(IRLCU_BUF_UPDATE, 0, h->d.pfUpdate, h->vox), "hook");
	if (h->norm_subset >= 0)
		irl_cu(irlcu_download(IRLCU_BUF_NORM, h->norm_subset, h->d.pfNorm, h->vox), "hook");
	if (h->d.pfSct != NULL)
		irl_cu(irlcu_download(IRLCU_BUF_PRJSCAT, 0, h->d.pfSct, h->prjn), "hook");
	f(&h->d, g_irl_hook_ctx);
	irl_cu(irlcu_upload(IRLCU_BUF_EST, 0, h->d.pfEst, h->vox), "hook");
	irl_cu(irlcu_upload(IRLCU_BUF_UPDATE, 0, h->d.pfUpdate, h->vox), "hook");
	if (h->d.pfSct != NULL)
		irl_cu(irlcu_upload(IRLCU_BUF_PRJSCAT, 0, h->d.pfSct, h->prjn), "hook");
}

static void write_norm_file(const char *base, int s, const float *img, size_t vox)
{
	char *name = (char *)irl_malloc(strlen(base) + 40, "norm name");
	FILE *fp;
	sprintf(name, "%s.norm.%d.dat", base, s);
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

static void delete_norm_files(const char *base, int ns)
{
	char *name = (char *)irl_malloc(strlen(base) + 40, "norm name");
	int s;
	for (s = 0; s < ns; ++s) {
		sprintf(name, "%s.norm.%d.dat", base, s);
		unlink(name);
	}
	free(name);
}

/* the OSEM loop (vOsemRecon, osemrecon.c:557-897); the estimate is on the
   device in internal layout */
static void osem_loop(irl_parms *p, irl_view *views, int use_scatest, float *est_host, float *prjscat_host,
	void (*cb)(int, float *), int max_batch)
{
	int *ang = NULL, ns, s, m, it, per = p->ang_per_subset;
	int prj_srf = p->prj_model & MODEL_SRF, this_srf = 0, next_srf = 0;
	int angle_hooks = g_irl_hooks[HOOK_PREV_ANGLE] || g_irl_hooks[HOOK_POST_ANGLE];
	size_t vox = (size_t)p->n * p->nz * p->n;
	hook_state h;
	float *tmp = NULL, *norm_host = NULL, *upd_host = NULL;
	irlcu_view_parm *vp = NULL;
	float *vt = NULL;
	double t0 = now_s();

	ns = irl_compute_subsets(p->nviews, per, &ang);
	irl_cu(irlcu_alloc_norm(ns), "OsemRecon");
	vt = (float *)irl_malloc(sizeof(float) * per, "view times");
	for (s = 0; s < ns; ++s) {
		for (m = 0; m < per; ++m)
			vt[m] = views[ang[s * per + m]].view_time;
		irl_cu(irlcu_norm_subset(per, ang + s * per, vt, p->bck_model, s), "ComputeNormImages");
		if (p->norm_base != NULL) {
			if (tmp == NULL)
				tmp = (float *)irl_malloc(sizeof(float) * vox, "norm image");
			irl_cu(irlcu_download(IRLCU_BUF_NORM, s, tmp, vox), "ComputeNormImages");
			write_norm_file(p->norm_base, s, tmp, vox);
		}
	}
	irl_msg(5, "Done Computing Norm Matrix (%.3f s)\n", now_s() - t0);

	memset(&h, 0, sizeof(h));
	h.vox = vox;
	h.prjn = (size_t)p->nviews * p->nz * p->n;
	h.norm_subset = -1;
	h.any = 0;
	for (m = 0; m < 6; ++m)
		h.any |= g_irl_hooks[m] != NULL;
	if (h.any) {
		norm_host = (float *)irl_calloc(sizeof(float) * vox, "norm mirror");
		upd_host = (float *)irl_calloc(sizeof(float) * vox, "update mirror");
	}
	h.d.pfEst = est_host;
	h.d.pfSct = prjscat_host;
	h.d.pfNorm = norm_host;
	h.d.pfUpdate = upd_host;

	if (prj_srf)
		next_srf = p->start_iteration + 1 <= p->srf_iters;
	p->start_iteration = g_irl_adv.iStartIteration;
	vp = (irlcu_view_parm *)irl_calloc(sizeof(irlcu_view_parm) * per, "view parameters");
	if (cb != NULL && tmp == NULL)
		tmp = (float *)irl_malloc(sizeof(float) * vox, "callback image");

	for (it = p->start_iteration + 1; it <= p->iterations; ++it) {
		int model = p->prj_model, mode = 0;
		double ti = now_s();
		h.d.iIterationIdx = it;
		hook_call(&h, HOOK_PREV_ITER);
		if (prj_srf) {
			this_srf = next_srf;
			next_srf = (it == p->iterations) ? this_srf : (it + 1 <= p->srf_iters);
			model = this_srf ? p->prj_model : (p->prj_model & ~MODEL_SRF);
			mode = !this_srf ? 1 : (!next_srf ? 2 : 0);
		}
		for (s = 0; s < ns; ++s) {
			const int *va = ang + s * per;
			h.d.iSubsetIdx = s;
			hook_call(&h, HOOK_PREV_SUBSET);
			for (m = 0; m < per; ++m) {
				vp[m].view_time = views[va[m]].view_time;
				vp[m].sensitivity = views[va[m]].sensitivity;
				vp[m].scat_mode = mode;
			}
			if (angle_hooks) {
				for (m = 0; m < per; ++m) {
					h.d.iAngleIdx = va[m];
					hook_call(&h, HOOK_PREV_ANGLE);
					irl_cu(irlcu_osem_subset(1, va + m, vp + m, model, p->bck_model, s, use_scatest,
						       m == per - 1, m > 0),
						"OsemRecon");
					if (m == per - 1)
						h.norm_subset = s;
					hook_call(&h, HOOK_POST_ANGLE);
				}
			} else {
				int m0;
				for (m0 = 0; m0 < per; m0 += max_batch) {
					int nb = per - m0 < max_batch ? per - m0 : max_batch;
					irl_cu(irlcu_osem_subset(nb, va + m0, vp + m0, model, p->bck_model, s, use_scatest,
						       m0 + nb >= per, m0 > 0),
						"OsemRecon");
				}
				h.norm_subset = s;
			}
			hook_call(&h, HOOK_POST_SUBSET);
		}
		hook_call(&h, HOOK_POST_ITER);
		if (cb != NULL) {
			irl_cu(irlcu_download_external(IRLCU_BUF_EST, tmp), "OsemRecon");
			cb(it, tmp);
		}
		irl_msg(4, "----Done iteration %d (%.3f s)\n", it, now_s() - ti);
	}
	if (p->norm_base != NULL)
		delete_norm_files(p->norm_base, ns);
	free(ang);
	free(vt);
	free(vp);
	free(tmp);
	free(norm_host);
	free(upd_host);
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

static void zero_neg(float *p, size_t n)
{
	size_t i;
	for (i = 0; i < n; ++i)
		if (p[i] < 0.0f)
			p[i] = 0.0f;
}

static void scale_f(float *p, size_t n, float s)
{
	size_t i;
	for (i = 0; i < n; ++i)
		p[i] *= s;
}

/* shared device set-up of IrlOsem and IrlGenprj */
void irl_device_setup(irl_parms *p, irl_view *views, const float *atn_internal, const irl_esse_host *esse,
	int fast_rotate, int max_batch)
{
	irlcu_geom g;
	float *angles = (float *)irl_malloc(sizeof(float) * p->nviews, "angles");
	unsigned char *mask = (unsigned char *)irl_malloc((size_t)p->nviews * p->n, "column masks");
	unsigned char *m1 = (unsigned char *)irl_malloc(p->n, "mask"), *m2 = (unsigned char *)irl_malloc(p->n, "mask");
	int a, i;
	g.n = p->n;
	g.nz = p->nz;
	g.nviews = p->nviews;
	g.fast_rotate = fast_rotate;
	g.max_batch = max_batch;
	irl_cu(irlcu_init(&g), "device set-up");
	for (a = 0; a < p->nviews; ++a)
		angles[a] = views[a].angle;
	irl_cu(irlcu_set_angles(angles), "device set-up");
	for (a = 0; a < p->nviews; ++a) {
		/* PWid = PixelWidth / BinWidth = 1 (IrlSetup.c:65-66) */
		float pw = p->pix / p->pix;
		irl_measured_columns(views[a].left, pw, p->n, p->nbins, m1);
		irl_norm_columns(views[a].left, views[a].right, pw, p->n, p->nbins, m2);
		for (i = 0; i < p->n; ++i)
			mask[(size_t)a * p->n + i] = (unsigned char)(m1[i] | (m2[i] << 1));
	}
	irl_cu(irlcu_set_column_mask(mask), "device set-up");
	if (atn_internal != NULL) {
		irl_cu(irlcu_upload(IRLCU_BUF_ATN, 0, atn_internal, (size_t)p->n * p->nz * p->n), "device set-up");
		irl_cu(irlcu_prepare_attenuation((p->model & MODEL_SRF) != 0), "device set-up");
	}
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
		e.krnl = esse->krnl;
		e.kmu = esse->kmu;
		e.kmu2 = esse->kmu2;
		irl_cu(irlcu_set_esse(&e), "ESSE set-up");
	} else if (p->model & MODEL_SRF) {
		irl_cu(irlcu_set_esse(NULL), "ESSE set-up");
	}
	free(angles);
	free(mask);
	free(m1);
	free(m2);
}

int IrlOsem(IrlParms_t *ip, Options_t *op, PrjView_t *pv, char *drf_fname, char *krnl_fname,
	void (*cb)(int, float *), float *scatest, float *atn, float *prj, float *recon, char *logname, char *msgname)
{
	jmp_buf env;
	int err = 0;
	/* static: their contents must survive the longjmp of a fatal error */
	static irl_parms p;
	static irl_esse_host esse;
	irl_view *volatile views = NULL;
	float *volatile tmp = NULL;
	float *volatile prjscat = NULL;
	FILE *volatile logfp = NULL;
	FILE *volatile msgfp = NULL;
	double t0 = now_s();

	memset(&esse, 0, sizeof(esse));
	if ((err = setjmp(env)) != 0) {
		fprintf(stderr, "FATAL ERROR Trapped: err_num=%d\nErrMsg=%s\n", err, irl_last_error());
		irl_msg(1, "aborted\n");
		goto abort;
	}
	irl_trap(&env);
	{
		FILE *l, *m;
		open_logs(logname, msgname, op->iMsgLevel, &l, &m);
		logfp = l;
		msgfp = m;
	}
	irl_setup_parms(ip, op, atn, krnl_fname, &p);
	views = irl_setup_views(ip, pv);
	if (p.model & MODEL_SRF) {
		if (atn == NULL)
			irl_fatal(IRL_E_VALUE, "SrfSetup", "scatter modelling needs an attenuation map");
		irl_esse_prepare(krnl_fname, &p, ip->SrfCollapseFac, &esse);
	}
	{
		irl_detector *d;
		/* libirl calls vSetupDrfTables unconditionally (irlosem.c:158-160) */
		irl_setup_drf_tables(&p, op, views, drf_fname, &d);
	}
	{
		size_t vox = (size_t)p.n * p.nz * p.n, prjn = (size_t)p.n * p.nz * p.nviews;
		tmp = (float *)irl_malloc(sizeof(float) * vox, "IrlOsem:Temp");
		if (atn != NULL) {
			irl_reorder(p.nz, p.n, p.n, atn, tmp);
			memcpy(atn, tmp, sizeof(float) * vox);
		}
		if (!op->bReconIsInitEst) {
			irl_initial_estimate(&p, op->bUseContourSupport, op->fAtnMapThresh, views, prj, atn, recon);
		} else {
			irl_reorder(p.nz, p.n, p.n, recon, tmp);
			memcpy(recon, tmp, sizeof(float) * vox);
		}
		zero_neg(prj, prjn);
		if (atn != NULL) {
			if (ip->fAtnScaleFac > 0 && ip->fAtnScaleFac != 1.0)
				scale_f(atn, vox, ip->fAtnScaleFac);
			zero_neg(atn, vox);
		}
		if (scatest != NULL) {
			if (ip->fScatEstFac > 0 && ip->fScatEstFac != 1.0)
				scale_f(scatest, prjn, ip->fScatEstFac);
			zero_neg(scatest, prjn);
		}
		zero_neg(recon, vox);
		if (cb != NULL) {
			irl_reorder(p.n, p.nz, p.n, recon, tmp);
			cb(0, tmp);
		}
		irl_device_setup(&p, views, atn, &esse, g_irl_adv.bFastRotate, p.ang_per_subset > 32 ? 32 : p.ang_per_subset);
		irl_cu(irlcu_upload(IRLCU_BUF_PRJ, 0, prj, prjn), "IrlOsem");
		irl_cu(irlcu_upload(IRLCU_BUF_EST, 0, recon, vox), "IrlOsem");
		if (scatest != NULL)
			irl_cu(irlcu_upload(IRLCU_BUF_SCATEST, 0, scatest, prjn), "IrlOsem");
		if ((p.prj_model & MODEL_SRF) && p.srf_iters > 0) {
			prjscat = (float *)irl_calloc(sizeof(float) * prjn, "OsemRecon:PrjScatEst");
			irl_cu(irlcu_zero(IRLCU_BUF_PRJSCAT, 0), "IrlOsem");
		}
		irl_msg(5, "Done Initialization (%.3f s)\n", now_s() - t0);
		osem_loop(&p, views, scatest != NULL, recon, prjscat, cb, p.ang_per_subset > 32 ? 32 : p.ang_per_subset);
		irl_cu(irlcu_download_external(IRLCU_BUF_EST, recon), "IrlOsem");
		irl_msg(4, "done (%.3f s)\n", now_s() - t0);
	}
abort:
	irl_untrap();
	irlcu_shutdown();
	irl_free_run_tables();
	free(views);
	free(tmp);
	free(prjscat);
	irl_esse_free(&esse);
	if (logfp != NULL) {
		fclose(logfp);
		irl_set_log_file(NULL);
	}
	if (msgfp != NULL) {
		fclose(msgfp);
		irl_set_msg_file(NULL);
	}
	return err;
}
