/*
 * irl_genprj.c -- IrlGenprj of libirl_b200 (libirl irlgenprj.c:23-309).
 *
 * Projections of an activity image: the activity is rotated, attenuated,
 * blurred by the DRF and (optionally) given the ESSE scatter source on the
 * GPU in batches of views; the per-view scatter-estimate addition, time and
 * sensitivity scaling, the view callback and the final 1/NumAngles scaling
 * stay on the host, in libirl's order.
 *
 * Difference from libirl: libirl's IrlGenprj inverts its "stderr" test for
 * the log and message file names (irlgenprj.c:121, 137); here they are
 * handled as in IrlOsem.
 */
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "irl_err.h"
#include "irl_host.h"
#include "irlcu.h"

static void open_logs2(const char *logname, const char *msgname, int level, FILE **plog, FILE **pmsg)
{
	*plog = *pmsg = NULL;
	if (logname == NULL)
		irl_set_log_file(NULL);
	else if (strcmp(logname, "stderr") == 0)
		irl_set_log_file(stderr);
	else {
		*plog = fopen(logname, "w");
		irl_set_log_file(*plog);
		if (*plog == NULL)
			irl_fatal(IRL_E_IO, "IrlGenprj", "Error opening log file %s", logname);
	}
	irl_set_msg_level(level);
	if (msgname == NULL)
		irl_set_msg_file(NULL);
	else if (strcmp(msgname, "stderr") == 0)
		irl_set_msg_file(stderr);
	else {
		*pmsg = fopen(msgname, "w");
		irl_set_msg_file(*pmsg);
		if (*pmsg == NULL)
			irl_fatal(IRL_E_IO, "IrlGenprj", "Error opening messages file %s", msgname);
	}
}

int IrlGenprj(IrlParms_t *ip, Options_t *op, PrjView_t *pv, char *drf_fname, char *krnl_fname,
	void (*cb)(int, float *), float *scatest, float *act, float *atn, float *prj, float fPrimaryFac,
	char *logname, char *msgname)
{
	jmp_buf env;
	int err = 0;
	static irl_parms p;
	static irl_esse_host esse;
	irl_view *volatile views = NULL;
	float *volatile tmp = NULL;
	float *volatile calc = NULL;
	int *volatile vidx = NULL;
	FILE *volatile logfp = NULL;
	FILE *volatile msgfp = NULL;

	memset(&esse, 0, sizeof(esse));
	if ((err = setjmp(env)) != 0) {
		fprintf(stderr, "FATAL ERROR Trapped: err_num=%d\nErrMsg=%s\n", err, irl_last_error());
		irl_msg(1, "aborted\n");
		goto abort;
	}
	irl_trap(&env);
	{
		FILE *l, *m;
		open_logs2(logname, msgname, op->iMsgLevel, &l, &m);
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
	if (p.model & MODEL_DRF) {
		irl_detector *d;
		irl_setup_drf_tables(&p, op, views, drf_fname, &d);
	}
	{
		const size_t vox = (size_t)p.n * p.nz * p.n, pln = (size_t)p.n * p.nz, prjn = pln * p.nviews;
		const int B = p.nviews < 32 ? p.nviews : 32;
		size_t i;
		int a, v0;
		tmp = (float *)irl_malloc(sizeof(float) * vox, "IrlGenprj:Temp");
		irl_reorder(p.nz, p.n, p.n, act, tmp);
		memcpy(act, tmp, sizeof(float) * vox);
		for (i = 0; i < vox; ++i)
			if (act[i] < 0.0f)
				act[i] = 0.0f;
		if (atn != NULL) {
			if (ip->fAtnScaleFac > 0 && ip->fAtnScaleFac != 1.0)
				for (i = 0; i < vox; ++i)
					atn[i] *= ip->fAtnScaleFac;
			for (i = 0; i < vox; ++i)
				if (atn[i] < 0.0f)
					atn[i] = 0.0f;
			irl_reorder(p.nz, p.n, p.n, atn, tmp);
			memcpy(atn, tmp, sizeof(float) * vox);
		}
		if (scatest != NULL) {
			if (ip->fScatEstFac > 0 && ip->fScatEstFac != 1.0)
				for (i = 0; i < prjn; ++i)
					scatest[i] *= ip->fScatEstFac;
			for (i = 0; i < prjn; ++i)
				if (scatest[i] < 0.0f)
					scatest[i] = 0.0f;
		}
		memset(prj, 0, sizeof(float) * prjn);
		/* IrlGenprj always uses the three-shear rotator (irlgenprj.c:19-21) */
		irl_device_setup(&p, views, atn, &esse, 1, B);
		irl_cu(irlcu_upload(IRLCU_BUF_EST, 0, act, vox), "IrlGenprj");
		calc = (float *)irl_malloc(sizeof(float) * pln * B, "IrlGenprj:CalcPrj");
		vidx = (int *)irl_malloc(sizeof(int) * B, "views");
		for (v0 = 0; v0 < p.nviews; v0 += B) {
			const int nb = p.nviews - v0 < B ? p.nviews - v0 : B;
			for (a = 0; a < nb; ++a)
				vidx[a] = v0 + a;
			irl_cu(irlcu_project(nb, vidx, p.prj_model, fPrimaryFac, calc, 0), "IrlGenprj");
			for (a = 0; a < nb; ++a) {
				const int iAngle = v0 + a;
				float *c = calc + pln * a, *o = prj + pln * iAngle;
				if (scatest != NULL)
					for (i = 0; i < pln; ++i)
						c[i] += scatest[pln * iAngle + i];
				for (i = 0; i < pln; ++i)
					o[i] = c[i] * views[iAngle].view_time * views[iAngle].sensitivity;
				if (cb != NULL)
					cb(iAngle, o);
			}
		}
		{
			const float s = 1.0 / (float)p.nviews;
			for (i = 0; i < prjn; ++i)
				prj[i] *= s;
		}
		irl_reorder(p.n, p.nz, p.n, act, tmp);
		memcpy(act, tmp, sizeof(float) * vox);
		if (atn != NULL) {
			irl_reorder(p.n, p.nz, p.n, atn, tmp);
			memcpy(atn, tmp, sizeof(float) * vox);
		}
	}
abort:
	irl_untrap();
	irlcu_shutdown();
	free(calc);
	free(vidx);
	free(views);
	free(tmp);
	irl_free_run_tables();
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
