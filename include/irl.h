/*
 * irl.h -- public C API of libirl_b200, the B200 implementation of libirl's
 * OSEM projector/backprojector path.
 *
 * Drop-in boundary: the structs and entry points below have the same
 * layout, names, argument meaning and return codes as libirl's irl.h
 * (irl.h:39-124 structs, irl.h:145-318 entry points) so that an
 * application built against libirl links against libirl_b200.so
 * unchanged.  Host code is C; the projector, backprojector, rotations,
 * DRF convolution, ESSE scatter model and EM update run as CUDA kernels
 * behind include/irlcu.h.
 *
 * Array layouts at this boundary (unchanged from libirl, irl.h:189-201):
 *   volumes      float[NumSlices][NumPixels][NumPixels]   x fastest, then y
 *   projections  float[NumViews][NumSlices][NumPixels]    bin fastest
 */
#ifndef IRL_H
#define IRL_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

/* bits of the projector / backprojector model masks */
#define MODEL_ATN 1
#define MODEL_DRF 2
#define MODEL_SRF 4

/* Reconstruction / projection parameters (libirl irl.h:39-79). */
typedef struct {
	int NumPixels;          /* pixels per image row and column; equals the
	                           number of transaxial projection bins */
	int NumSlices;          /* axial slices */
	int NumViews;           /* projection views */
	float BinWidth;         /* bin width = pixel width, cm */
	float fAtnScaleFac;     /* multiplies the attenuation map to give
	                           attenuation per pixel at the primary energy */
	int iNumSrfIterations;  /* iterations in which scatter is modelled */
	float fScatEstFac;      /* multiplies the additive scatter estimate */
	int NumAngPerSubset;    /* views per OSEM subset; divides NumViews */
	int NumIterations;
	char *pchNormImageBase; /* if non-NULL, per-subset normalisation images
	                           are written to <base>.norm.<subset>.dat */
	int SrfCollapseFac;     /* ESSE coarse-grid factor, 1..4 */
	/* collimator description, used when the DRF is computed on the fly */
	float fHoleDiam;
	float fHoleLen;
	float fBackToDet;
	float fIntrinsicFWHM;
} IrlParms_t;

/* Reconstruction options (libirl irl.h:81-124). */
typedef struct {
	int bModelDrf;          /* model the depth-dependent response */
	int bReconIsInitEst;    /* pfReconImage holds the initial estimate */
	int bUseGrfInBck;       /* backproject with the computed GRF table */
	int bFFTConvolve;       /* DRF convolution in the frequency domain */
	int bUseContourSupport; /* zero the initial estimate outside the orbit */
	float fAtnMapThresh;    /* > 0: zero the initial estimate where the
	                           attenuation map is below this (per cm) */
	int iMsgLevel;          /* 1..9 verbosity of the message file */
	int iAxialPadLength;    /* axial padding rows for the DRF convolution */
	int iAxialAvgLength;    /* rows averaged to fill the axial padding */
} Options_t;

/* Per-view geometry (libirl irl.h:127-143). */
typedef struct {
	float Angle;            /* radians from the x axis */
	float Left;             /* first measured bin position */
	float Right;            /* last measured bin position */
	float CFCR;             /* centre of rotation to collimator face, cm */
} PrjView_t;

/*
 * OSEM reconstruction (libirl irlosem.c:22).  Returns 0 on success or a
 * non-zero error code whose message pchIrlErrorString() returns.  As in
 * libirl, pfAtnMap is reordered and scaled in place, pfPrjImage and
 * pfScatterEstimate are clamped at zero in place, and the iteration
 * callback is called for iteration 0 and after every iteration.
 */
int IrlOsem(IrlParms_t *psIrlParms, Options_t *psOptions, PrjView_t *psViews,
	char *pchDrfTabFname, char *pchScatKrnlFname,
	void (*pIterationCallbackFunc)(int IterationNumber, float *pfCurrentEst),
	float *pfScatterEstimate, float *pfAtnMap, float *pfPrjImage,
	float *pfReconImage, char *pchLogFname, char *pchMessageFname);

/* Projection generation (libirl irlgenprj.c:23). */
int IrlGenprj(IrlParms_t *psIrlParms, Options_t *psOptions, PrjView_t *psPrjViews,
	char *pchDrfTabFname, char *pchScatKrnlFname,
	void (*pPrjViewCallbackFunc)(int PrjViewNumber, float *pfCurrentPrjView),
	float *pfScatterEstimate, float *pfActImage, float *pfAtnMap,
	float *pfPrjImage, float fPrimaryFac, char *pchLogFname,
	char *pchMessageFname);

/* Per-view CFCR from a body outline (libirl computeorbit.c:21).  Returns 0,
   1 on an allocation failure, 2 for an unsupported orbit type. */
int ComputeOrbit(float *pfPixels, IrlParms_t *psParms, float fMargin,
	float *pfMargins, float fThresh, int OrbitType, PrjView_t *psViews);

/* Message of the last fatal error (libirl irlosem.c:287). */
char *pchIrlErrorString(void);

#ifdef __cplusplus
}
#endif

#endif /* IRL_H */
