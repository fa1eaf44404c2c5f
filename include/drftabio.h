/*
 * drftabio.h -- DRF table types and the "DRFT" binary file format of
 * libirl_b200.  Types, field order and the two entry points match libirl's
 * drftabio.h:7-42 so that DRFT files and callers are interchangeable.
 *
 * DRFT file (native byte order; a reader accepts the opposite order too):
 *   char[4] "DRFT"; int version = 1; char title[80]; char collimator[20];
 *   float pixel size (cm); float spacing between tables (cm);
 *   float distance of the first table (cm); int number of tables;
 *   int incremental-kernel flag; then per table:
 *   int MaxOffsX, int MaxOffsY, float psf[(2*MaxOffsY-1)][(2*MaxOffsX-1)].
 */
#ifndef DRFTABIO_H
#define DRFTABIO_H

#ifdef __cplusplus
extern "C" {
#endif

/* One depth's point-spread function, centre at (MaxOffsY-1, MaxOffsX-1). */
typedef struct {
	int MaxOffsX;
	int MaxOffsY;
	int bFFTdone;
	float *Psf;
} Drf_t;

/* A table of PSFs for distances fStartDistance + i*fDrfSpacing. */
typedef struct DrfTab_s {
	int iNumDistances;
	float fStartDistance;
	float fDrfSpacing;
	float fPixSize;
	int bIncKrnl;
	int bDrfFromFile;
	struct DrfTab_s *psBckDrfTab; /* table used by the backprojector, or NULL */
	float fGap, fHoleDiam, fColThick, fIntrinsicFWHM, fMaxFracErr;
	Drf_t *psDrfs;
	int bFFTconvolve;
} DrfTab_t;

/* Writes a DRFT file (libirl drftabio.c:57).  Unlike libirl the file is
   closed before returning. */
void vWriteDrfTab(DrfTab_t *psOutDrfTab, char *pchOutFname, char *pchTitle,
	char *pchColName);

/* Reads a DRFT file (libirl drftabio.c:150).  Errors are fatal: inside
   IrlOsem/IrlGenprj they abort the call with a non-zero return. */
DrfTab_t sReadDrfTab(char *pchInFname, char **ppchInTitle, char **ppchInColName);

#ifdef __cplusplus
}
#endif

#endif /* DRFTABIO_H */
