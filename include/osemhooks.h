/*
 * osemhooks.h -- OSEM hooks, advanced options and multi-detector set-up of
 * libirl_b200.  Same types, names and return values as libirl's
 * osemhooks.h:18-79.
 *
 * Hooks receive host pointers to the estimate, scatter estimate, inverted
 * normalisation image and update image in the internal layout
 * float[NumPixels(y)][NumSlices][NumPixels(x)].  libirl_b200 keeps these
 * arrays in GPU memory; it copies them to host mirrors before each hook
 * and back afterwards, so a hook may read and modify them as with libirl.
 * One context pointer is shared by all hooks (the last setter wins).
 */
#ifndef OSEMHOOKS_H
#define OSEMHOOKS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct _OsemData {
	int iIterationIdx;
	int iSubsetIdx;
	int iAngleIdx;
	float *pfEst;
	float *pfSct;
	float *pfNorm;
	float *pfUpdate;
} sOsemData, *psOsemData;

typedef struct _AdvOptions {
	int bFastRotate;       /* 1: three-shear rotation (default); 0: bilinear */
	int iStartIteration;   /* resume: iterations already done */
} sAdvOptions, *psAdvOptions;

/* each setter returns 1 (libirl osemrecon.c:44-90) */
int OsemSetAdvOptions(sAdvOptions *pOpt);
int OsemSetPrevIterHook(void (*pPrevIterHookFunc)(sOsemData *psData, void *ctx), void *ctx);
int OsemSetPostIterHook(void (*pPostIterHookFunc)(sOsemData *psData, void *ctx), void *ctx);
int OsemSetPrevSubsetHook(void (*pPrevSubsetHookFunc)(sOsemData *psData, void *ctx), void *ctx);
int OsemSetPostSubsetHook(void (*pPostSubsetHookFunc)(sOsemData *psData, void *ctx), void *ctx);
int OsemSetPrevAngleHook(void (*pPrevAngleHookFunc)(sOsemData *psData, void *ctx), void *ctx);
int OsemSetPostAngleHook(void (*pPostAngleHookFunc)(sOsemData *psData, void *ctx), void *ctx);

/*
 * Per-view acquisition times and detector numbers (libirl
 * IrlSetup.c:350-402).  The arrays must come from malloc: the library
 * frees them at the end of the next IrlOsem / IrlGenprj call.  Returns a
 * bit mask of argument errors (0 = OK).
 */
int iSetupExtraPrjViewData(int iNumPrjViews, float *pfAcqTimes, int *piDetectorNums);

/* Detector table (libirl IrlSetup.c:441-462); returns 0 or an error mask.
   The pointer array and its entries are freed after the next run. */
int iSetupDetectors(int iNumDetectors, void **ppsDetectors);

/* One detector's collimator and DRF description (libirl IrlSetup.c:415).
   pchDrfTabFname is kept, not copied, and freed after the next run. */
void *pvStoreDetectorData(float fHoleDiam, float fHoleLen, float fBackToDet,
	float fIntrinsicFWHM, float fSensitivity, int bFFTconvolve,
	int bUseGrfInBck, char *pchDrfTabFname);

#ifdef __cplusplus
}
#endif

#endif /* OSEMHOOKS_H */
