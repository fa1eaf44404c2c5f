/*
 * irl_tabio.c -- DRFT (DRF table) and KRNL (ESSE kernel) file formats.
 *
 * Byte layouts are libirl's (drftabio.c:26-48, krnlio.c:31-63; described in
 * include/drftabio.h and include/krnlio.h).  Files are written in native
 * byte order; a reader recognises the opposite order from the version word
 * and swaps every 4-byte field.  Errors are fatal through irl_fatal().
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "drftabio.h"
#include "krnlio.h"
#include "irl_err.h"
#include "irl_host.h"

#define DRF_TITLESIZE 80
#define DRF_COLSIZE 20
#define KRNL_TITLESIZE 80
#define KRNL_ISOSIZE 20

static void swap4(void *p, size_t n)
{
	unsigned char *b = (unsigned char *)p, t;
	size_t i;
	for (i = 0; i < n; ++i, b += 4) {
		t = b[0];
		b[0] = b[3];
		b[3] = t;
		t = b[1];
		b[1] = b[2];
		b[2] = t;
	}
}

static void wr(FILE *fp, const void *p, size_t sz, size_t n, const char *fname, const char *what)
{
	if (fwrite(p, sz, n, fp) != n)
		irl_fatal(IRL_E_IO, "write table", "IO error writing %s to %s", what, fname);
}

static void rd(FILE *fp, void *p, size_t sz, size_t n, int swapped, const char *fname, const char *what)
{
	if (fread(p, sz, n, fp) != n) {
		fclose(fp);
		irl_fatal(IRL_E_IO, "read table", "file %s is truncated (reading %s)", fname, what);
	}
	if (swapped && sz == 4)
		swap4(p, n);
}

static void wr_str(FILE *fp, const char *s, int width, const char *fname, const char *what)
{
	char buf[128];
	size_t len = s ? strlen(s) : 0;
	memset(buf, 0, sizeof(buf));
	if ((int)len >= width) {
		irl_warn("write table", "%s is longer than %d characters; truncated", what, width - 1);
		len = width - 1;
	}
	if (len)
		memcpy(buf, s, len);
	wr(fp, buf, 1, width, fname, what);
}

/* returns 1 if the file's byte order is swapped, fatal on a bad version */
static int check_version(FILE *fp, const char *fname, const char *sig)
{
	char got[5] = {0};
	int ver;
	rd(fp, got, 1, 4, 0, fname, "signature");
	if (memcmp(got, sig, 4) != 0) {
		fclose(fp);
		irl_fatal(IRL_E_VALUE, "read table", "signature in %s is \"%s\", should be \"%s\"", fname, got, sig);
	}
	rd(fp, &ver, 4, 1, 0, fname, "version");
	if (ver == 1)
		return 0;
	swap4(&ver, 1);
	if (ver == 1)
		return 1;
	swap4(&ver, 1);
	fclose(fp);
	irl_fatal(IRL_E_VALUE, "read table", "version in %s is %x hex, should be 1", fname, ver);
	return 0;
}

static char *rd_str(FILE *fp, int width, const char *fname, const char *what)
{
	char buf[128];
	rd(fp, buf, 1, width, 0, fname, what);
	buf[width] = '\0';
	return irl_strdup(buf);
}

void vWriteDrfTab(DrfTab_t *t, char *fname, char *title, char *colname)
{
	FILE *fp = fopen(fname, "wb");
	const int ver = 1;
	int i;
	if (fp == NULL)
		irl_fatal(IRL_E_IO, "vWriteDrfTab", "cannot open DRF table file %s", fname);
	wr(fp, "DRFT", 1, 4, fname, "signature");
	wr(fp, &ver, 4, 1, fname, "version");
	wr_str(fp, title, DRF_TITLESIZE, fname, "title");
	wr_str(fp, colname, DRF_COLSIZE, fname, "collimator name");
	wr(fp, &t->fPixSize, 4, 1, fname, "pixel size");
	wr(fp, &t->fDrfSpacing, 4, 1, fname, "spacing");
	wr(fp, &t->fStartDistance, 4, 1, fname, "start distance");
	wr(fp, &t->iNumDistances, 4, 1, fname, "number of distances");
	wr(fp, &t->bIncKrnl, 4, 1, fname, "incremental flag");
	for (i = 0; i < t->iNumDistances; ++i) {
		const Drf_t *d = &t->psDrfs[i];
		wr(fp, &d->MaxOffsX, 4, 1, fname, "MaxOffsX");
		wr(fp, &d->MaxOffsY, 4, 1, fname, "MaxOffsY");
		wr(fp, d->Psf, 4, (size_t)(2 * d->MaxOffsX - 1) * (2 * d->MaxOffsY - 1), fname, "PSF");
	}
	if (fclose(fp) != 0)
		irl_fatal(IRL_E_IO, "vWriteDrfTab", "IO error closing %s", fname);
}

DrfTab_t sReadDrfTab(char *fname, char **ptitle, char **pcolname)
{
	DrfTab_t t;
	FILE *fp;
	int swapped, i;
	memset(&t, 0, sizeof(t));
	t.bDrfFromFile = 1;
	fp = fopen(fname, "rb");
	if (fp == NULL)
		irl_fatal(IRL_E_IO, "sReadDrfTab", "cannot open DRF table file %s", fname);
	swapped = check_version(fp, fname, "DRFT");
	*ptitle = rd_str(fp, DRF_TITLESIZE, fname, "title");
	*pcolname = rd_str(fp, DRF_COLSIZE, fname, "collimator name");
	rd(fp, &t.fPixSize, 4, 1, swapped, fname, "pixel size");
	rd(fp, &t.fDrfSpacing, 4, 1, swapped, fname, "spacing");
	rd(fp, &t.fStartDistance, 4, 1, swapped, fname, "start distance");
	rd(fp, &t.iNumDistances, 4, 1, swapped, fname, "number of distances");
	rd(fp, &t.bIncKrnl, 4, 1, swapped, fname, "incremental flag");
	if (t.iNumDistances <= 0 || t.iNumDistances > 100000) {
		fclose(fp);
		irl_fatal(IRL_E_VALUE, "sReadDrfTab", "bad number of distances %d in %s", t.iNumDistances, fname);
	}
	t.psDrfs = (Drf_t *)irl_calloc(sizeof(Drf_t) * t.iNumDistances, "DRF table");
	for (i = 0; i < t.iNumDistances; ++i) {
		Drf_t *d = &t.psDrfs[i];
		size_t cnt;
		rd(fp, &d->MaxOffsX, 4, 1, swapped, fname, "MaxOffsX");
		rd(fp, &d->MaxOffsY, 4, 1, swapped, fname, "MaxOffsY");
		if (d->MaxOffsX < 1 || d->MaxOffsY < 1 || d->MaxOffsX > 4096 || d->MaxOffsY > 4096) {
			fclose(fp);
			irl_fatal(IRL_E_VALUE, "sReadDrfTab", "bad PSF size %d x %d at distance %d in %s",
				d->MaxOffsX, d->MaxOffsY, i, fname);
		}
		cnt = (size_t)(2 * d->MaxOffsX - 1) * (2 * d->MaxOffsY - 1);
		d->Psf = (float *)irl_malloc(cnt * sizeof(float), "PSF");
		d->bFFTdone = 0;
		rd(fp, d->Psf, 4, cnt, swapped, fname, "PSF");
	}
	fclose(fp);
	return t;
}

DrfTab_t *irl_free_drftab(DrfTab_t *t)
{
	int i;
	if (t == NULL)
		return NULL;
	if (t->psBckDrfTab != NULL)
		t->psBckDrfTab = irl_free_drftab(t->psBckDrfTab);
	if (t->psDrfs != NULL) {
		for (i = 0; i < t->iNumDistances; ++i)
			free(t->psDrfs[i].Psf);
		free(t->psDrfs);
	}
	free(t);
	return NULL;
}

void vWriteKrnlFile(KrnlData_t *k, char *fname)
{
	FILE *fp = fopen(fname, "wb");
	const int ver = 1;
	size_t cnt;
	if (fp == NULL)
		irl_fatal(IRL_E_IO, "vWriteKrnlFile", "cannot open kernel file %s", fname);
	wr(fp, "KRNL", 1, 4, fname, "signature");
	wr(fp, &ver, 4, 1, fname, "version");
	wr_str(fp, k->pchTitle, KRNL_TITLESIZE, fname, "title");
	wr_str(fp, k->pchIsotope, KRNL_ISOSIZE, fname, "isotope");
	wr(fp, &k->fKrnlMu0, 4, 1, fname, "mu0");
	wr(fp, &k->fHighEnergy, 4, 1, fname, "high energy");
	wr(fp, &k->fLowEnergy, 4, 1, fname, "low energy");
	wr(fp, &k->fPixSize, 4, 1, fname, "pixel size");
	wr(fp, &k->fPriFac, 4, 1, fname, "primary factor");
	wr(fp, &k->fScatFac, 4, 1, fname, "scatter factor");
	wr(fp, &k->fCntrPixFac, 4, 1, fname, "centre pixel factor");
	wr(fp, &k->iNumXYoffs, 4, 1, fname, "NumXYoffs");
	wr(fp, &k->iNumDists, 4, 1, fname, "NumDists");
	cnt = (size_t)k->iNumXYoffs * k->iNumXYoffs * k->iNumDists;
	wr(fp, k->pfKrnl, 4, cnt, fname, "kernel");
	wr(fp, k->pfKrnlMu, 4, cnt, fname, "mu kernel");
	if (fclose(fp) != 0)
		irl_fatal(IRL_E_IO, "vWriteKrnlFile", "IO error closing %s", fname);
}

KrnlData_t *psReadKrnlFile(char *fname, int bReadArrays)
{
	KrnlData_t *k;
	FILE *fp;
	int swapped;
	size_t cnt;
	fp = fopen(fname, "rb");
	if (fp == NULL)
		irl_fatal(IRL_E_IO, "psReadKrnlFile", "cannot open kernel file %s", fname);
	swapped = check_version(fp, fname, "KRNL");
	k = (KrnlData_t *)irl_calloc(sizeof(KrnlData_t), "kernel data");
	k->pchTitle = rd_str(fp, KRNL_TITLESIZE, fname, "title");
	k->pchIsotope = rd_str(fp, KRNL_ISOSIZE, fname, "isotope");
	rd(fp, &k->fKrnlMu0, 4, 1, swapped, fname, "mu0");
	rd(fp, &k->fHighEnergy, 4, 1, swapped, fname, "high energy");
	rd(fp, &k->fLowEnergy, 4, 1, swapped, fname, "low energy");
	rd(fp, &k->fPixSize, 4, 1, swapped, fname, "pixel size");
	rd(fp, &k->fPriFac, 4, 1, swapped, fname, "primary factor");
	rd(fp, &k->fScatFac, 4, 1, swapped, fname, "scatter factor");
	rd(fp, &k->fCntrPixFac, 4, 1, swapped, fname, "centre pixel factor");
	rd(fp, &k->iNumXYoffs, 4, 1, swapped, fname, "NumXYoffs");
	rd(fp, &k->iNumDists, 4, 1, swapped, fname, "NumDists");
	if (k->iNumDists <= 0 || k->iNumXYoffs < 0 || k->iNumXYoffs > 4096 || k->iNumDists > 4096) {
		fclose(fp);
		irl_fatal(IRL_E_VALUE, "psReadKrnlFile", "sizes of kernel must be > 0, not numdists=%d, numXYoffs=%d",
			k->iNumDists, k->iNumXYoffs);
	}
	if (bReadArrays) {
		cnt = (size_t)k->iNumXYoffs * k->iNumXYoffs * k->iNumDists;
		k->pfKrnl = (float *)irl_malloc(cnt * 4, "kernel");
		k->pfKrnlMu = (float *)irl_malloc(cnt * 4, "mu kernel");
		rd(fp, k->pfKrnl, 4, cnt, swapped, fname, "kernel");
		rd(fp, k->pfKrnlMu, 4, cnt, swapped, fname, "mu kernel");
	}
	fclose(fp);
	return k;
}

KrnlData_t *psFreeKrnlData(KrnlData_t *k, int bFreeArrays)
{
	if (k == NULL)
		return NULL;
	free(k->pchTitle);
	free(k->pchIsotope);
	if (bFreeArrays) {
		free(k->pfKrnl);
		free(k->pfKrnlMu);
	}
	free(k);
	return NULL;
}
