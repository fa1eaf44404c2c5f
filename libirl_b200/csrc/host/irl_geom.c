/*
 * irl_geom.c -- exact geometry tables for the device kernels.
 *
 * Every expression below keeps the operand types of the libirl code it
 * follows (float variables, double literals and double libm calls) so the
 * rounded results are identical; the kernels then only apply them.
 */
#include <math.h>

#include "irl_geom.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

void irl_shear_table(float fAngle, int n, irl_shear_tab *t)
{
	/* angle reduction to (-45, 45] degrees with index flips
	   (fastrotate.c:360-375) */
	int b90 = 0, b180 = 0, j, i, iAdd, mDim, iTmp;
	float fCntr, tCntr, yDist, xDist, fDelta, f1, f2;

	while (fAngle > 0.75 * M_PI) {
		fAngle -= M_PI;
		b180++;
		if (b180 == 2)
			b180 = 0;
	}
	while (fAngle <= -M_PI / 4.0) {
		fAngle += M_PI;
		b180++;
		if (b180 == 2)
			b180 = 0;
	}
	if (fAngle > M_PI / 4.0) {
		b90 = 1;
		fAngle -= M_PI / 2.0;
	}
	/* size of the intermediate images (fastrotate.c:378-388) */
	fCntr = ((float)n - 1.0) * 0.5;
	iAdd = 0;
	for (j = n / 4; j < n / 2; j++) {
		yDist = (float)j - fCntr;
		fDelta = fabs(yDist * tan((double)(fAngle * 0.5)));
		fDelta -= fCntr - sqrt(fCntr * fCntr - yDist * yDist);
		iTmp = ceil(fDelta);
		if (iTmp > iAdd)
			iAdd = iTmp;
	}
	mDim = n + 2 * iAdd;
	tCntr = ((float)mDim - 1.0) * 0.5;
	t->b90 = b90;
	t->b180 = b180;
	t->iadd = iAdd;
	t->mdim = mDim;
	/* x shifts, identical in passes 1 and 3 (fastrotate.c:403-408, 528-532) */
	for (j = 0; j < n; j++) {
		yDist = (float)j - fCntr;
		fDelta = -1.0 * yDist * tan((double)(fAngle * 0.5));
		iTmp = floorf(fDelta);
		f2 = fDelta - (float)iTmp;
		f1 = 1.0 - f2;
		t->row_sh[j] = iTmp;
		t->row_f1[j] = f1;
		t->row_f2[j] = f2;
	}
	/* y shifts of pass 2 (fastrotate.c:498-504) */
	for (i = 0; i < mDim; i++) {
		int jTmp;
		xDist = (float)i - tCntr;
		fDelta = xDist * sin((double)(fAngle));
		jTmp = floorf(fDelta);
		f2 = fDelta - (float)jTmp;
		f1 = 1.0 - f2;
		t->col_sh[i] = jTmp;
		t->col_f1[i] = f1;
		t->col_f2[i] = f2;
	}
}

void irl_shear_support(int n, int *start, int *end)
{
	int j, iLen;
	float fTmp, fCntr = (n - 1) * 0.5;
	for (j = 0; j < n; j++) {
		fTmp = ((float)j - fCntr);
		iLen = 2 * floor(sqrt(fCntr * fCntr - fTmp * fTmp)) + 2;
		start[j] = (n - iLen) / 2;
		end[j] = start[j] + iLen;
	}
}

void irl_rot3dpar_sincos(float fAngle, float *s, float *c)
{
	*s = (float)sin(fAngle);
	*c = (float)cos(fAngle);
}

void irl_drf_rows(float fCFCR, float fPixelWidth, int iNumRotPixs, float fStart,
	float fSpacing, int iNumDistances, int *row_idist)
{
	int iRow, iDist;
	float fStartDist = fCFCR - fPixelWidth * iNumRotPixs / 2 + 0.5 * fPixelWidth;
	for (iRow = 0; iRow < iNumRotPixs; iRow++) {
		float fDist = fStartDist + iRow * fPixelWidth;
		iDist = (int)floor((fDist - fStart) / fSpacing + 0.5);
		iDist = iDist < 0 ? 0 : iDist;
		iDist = iDist > iNumDistances - 1 ? iNumDistances - 1 : iDist;
		row_idist[iRow] = fDist > 0.0 ? iDist : -1;
	}
}

void irl_measured_columns(float left, float PWid, int nRotPixs, int nBins, unsigned char *mask)
{
	float PixelLeft = left, PixelRight;
	int iPixel, BinLeft, BinRight;
	for (iPixel = 0; iPixel < nRotPixs; iPixel++) {
		PixelRight = PixelLeft + PWid;
		BinLeft = floor((double)PixelLeft);
		BinRight = floor((double)PixelRight);
		mask[iPixel] = !((BinRight <= 0) || (BinLeft >= nBins));
		PixelLeft = PixelRight;
	}
}

void irl_norm_columns(float left, float right, float PWid, int nRotPixs, int nBins,
	unsigned char *mask)
{
	float PixelLeft = left, PixelRight;
	int iPixel, BinLeft, BinRight;
	for (iPixel = 0; iPixel < nRotPixs; iPixel++)
		mask[iPixel] = 0;
	for (iPixel = 0; iPixel < nRotPixs; iPixel++) {
		PixelRight = PixelLeft + PWid;
		BinLeft = floor((double)PixelLeft);
		BinRight = floor((double)PixelRight);
		if (BinLeft > right)
			break;
		mask[iPixel] = (BinRight > 0) && (BinLeft < nBins);
		PixelLeft = PixelRight;
	}
}
