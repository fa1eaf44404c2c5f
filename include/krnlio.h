/*
 * krnlio.h -- ESSE scatter-kernel type and the "KRNL" binary file format of
 * libirl_b200.  Same type and entry points as libirl's krnlio.h:10-35.
 *
 * KRNL file (native byte order; a reader accepts the opposite order too):
 *   char[4] "KRNL"; int version = 1; char title[80]; char isotope[20];
 *   float mu0; float high energy; float low energy; float pixel size;
 *   float primary factor; float scatter factor; float centre-pixel factor;
 *   int NumXYoffs; int NumDists;
 *   float kernel[NumDists][NumXYoffs][NumXYoffs];
 *   float mu kernel[NumDists][NumXYoffs][NumXYoffs].
 */
#ifndef KRNLIO_H
#define KRNLIO_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
	char *pchTitle;
	char *pchIsotope;
	int iNumXYoffs, iNumDists;
	float fKrnlMu0;
	float fPixSize;
	float fHighEnergy, fLowEnergy;
	float fPriFac, fScatFac, fCntrPixFac;
	float *pfKrnl, *pfKrnlMu;
} KrnlData_t;

void vWriteKrnlFile(KrnlData_t *psKrnl, char *pchKrnlFname);
/* Reads a KRNL file (libirl krnlio.c:196).  libirl byte-swaps the wrong
   field when it reads NumXYoffs from an opposite-endian file
   (krnlio.c:293); this reader swaps NumXYoffs itself. */
KrnlData_t *psReadKrnlFile(char *pchKrnlFname, int bReadArrays);
KrnlData_t *psFreeKrnlData(KrnlData_t *psKrnl, int bFreeArrays);

#ifdef __cplusplus
}
#endif

#endif /* KRNLIO_H */
