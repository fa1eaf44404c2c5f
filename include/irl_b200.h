/*
 * irl_b200.h -- entry points of libirl_b200 beyond libirl's API.
 *
 * IrlOsem (irl.h) is exactly IrlOsemBegin + IrlOsemIterate(NumIterations)
 * + IrlOsemEnd.  The split lets a caller keep a reconstruction resident on
 * the GPU and run its iterations in steps (benchmarks, interactive use,
 * stopping rules).  libirl has no counterpart of these three functions.
 *
 * One session at a time per process (the library is non-reentrant, like
 * libirl); IrlOsemBatch runs several side by side internally.  The caller's arrays follow IrlOsem's contract: pfAtnMap,
 * pfPrjImage and pfScatterEstimate are modified in place by Begin, and
 * pfReconImage must stay valid until End (hooks see it in the internal
 * layout, as in libirl).
 */
#ifndef IRL_B200_H
#define IRL_B200_H

#include "irl.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Set-up of IrlOsem (everything before the first iteration, including the
   normalisation images and the iteration-0 callback).  Returns 0 or an
   error code (pchIrlErrorString gives the message); on error the session
   is closed. */
int IrlOsemBegin(IrlParms_t *psIrlParms, Options_t *psOptions, PrjView_t *psViews,
	char *pchDrfTabFname, char *pchScatKrnlFname,
	void (*pIterationCallbackFunc)(int IterationNumber, float *pfCurrentEst),
	float *pfScatterEstimate, float *pfAtnMap, float *pfPrjImage, float *pfReconImage,
	char *pchLogFname, char *pchMessageFname);

/* Runs up to iNumIterations further iterations (never past NumIterations)
   with hooks and callbacks as in IrlOsem; returns 0 or an error code. */
int IrlOsemIterate(int iNumIterations);

/* Copies the estimate (external layout) into pfReconImage and closes the
   session.  Always safe to call; returns the session's error code. */
int IrlOsemEnd(float *pfReconImage);

/* One reconstruction of a batch: IrlOsem's arguments without the
   callback, log and message files.  iStatus receives its return code. */
typedef struct {
	IrlParms_t *psIrlParms;
	Options_t *psOptions;
	PrjView_t *psViews;
	char *pchDrfTabFname;       /* malloc'd; freed by the library, as in IrlOsem */
	char *pchScatKrnlFname;
	float *pfScatterEstimate;
	float *pfAtnMap;
	float *pfPrjImage;
	float *pfReconImage;
	int iStatus;
} IrlOsemProblem_t;

/* Runs nprob independent OSEM reconstructions, each exactly as IrlOsem
   would run it alone (same results).  Every problem has its own device
   context and stream; they run pipelined: while the device iterates the
   problems enqueued so far (all iterations of each at once), the host sets
   up the next.  Up to IRL_BATCH_DEPTH (environment, default 4) problems are
   resident at a time, fewer when the next one might not fit in device
   memory; the oldest is finished first.
   Not allowed with hooks, or with iSetupExtraPrjViewData /
   iSetupDetectors data pending (those are per-call state of IrlOsem).
   Returns 0, or the first non-zero iStatus. */
int IrlOsemBatch(int nprob, IrlOsemProblem_t *psProblems);

/* Learned scatter surrogate for the following IrlOsem / IrlOsemBegin /
   IrlOsemBatch calls (128^3 volumes with the ESSE scatter model).
   pchWeightsFname is a weights file written by the training in
   libirl_b200/surrogate (NULL switches the surrogate off).  The first
   scatter iteration runs ESSE on every view; then each view's NRMSE of the
   surrogate against ESSE (||s - e|| / ||e|| of the scatter projection, on
   the estimate at that point) is measured, views above fFallbackNrmse
   (default 0.02) keep ESSE and the others use the network. */
int IrlSetScatterSurrogate(const char *pchWeightsFname, float fFallbackNrmse);

/* Those per-view NRMSEs of the open session (after its first scatter
   iteration); returns 0 or an error code. */
int IrlGetScatterSurrogateNrmse(float *pfNrmse, int iNumViews);

#ifdef __cplusplus
}
#endif

#endif /* IRL_B200_H */
