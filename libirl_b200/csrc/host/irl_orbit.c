/*
 * irl_orbit.c -- ComputeOrbit of libirl_b200 (libirl computeorbit.c:21-150).
 *
 * The body outline is rotated onto a sqrt(2)-larger grid with the bilinear
 * rotator (rot3dpar.c:19-198) for each view and the first non-empty row
 * from the detector gives the camera radius.  A single 2D image per view is
 * far below the size where a GPU launch pays, so this runs on the host with
 * the same arithmetic as the device rotator.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "irl_host.h"

/* bilinear rotation of one n_old x n_old slice onto n_new x n_new */
static void rot2d(float fAngle, const float *Old, float *New, int OldDim, int NewDim)
{
	int NewX, NewY, OldX, OldY, HeadPixel, TailPixel, NumPix;
	float FloatX, FloatY, X, Y, z0, z1, z2, z3, z01, z23, z0123;
	float NewAxis, OldAxis, Radius, Sin, Cos;
	int z0out, z1out, z2out, z3out;
	Sin = (float)sin(fAngle);
	Cos = (float)cos(fAngle);
	memset(New, 0, sizeof(float) * NewDim * NewDim);
	NewAxis = 0.5 * (NewDim - 1);
	OldAxis = 0.5 * (OldDim - 1);
	Radius = 0.5 * NewDim;
	for (NewY = 0; NewY < NewDim; NewY++) {
		Y = NewY - NewAxis;
		NumPix = (int)(sqrt(Radius * Radius - (Radius - NewY - .5) * (Radius - NewY - .5)) + .5);
		NumPix *= 2;
		HeadPixel = (int)(0.5 * (NewDim - NumPix));
		TailPixel = HeadPixel + NumPix - 1;
		for (NewX = HeadPixel; NewX <= TailPixel; NewX++) {
			X = NewX - NewAxis;
			FloatX = X * Cos - Y * Sin + OldAxis;
			FloatY = X * Sin + Y * Cos + OldAxis;
			OldX = (int)FloatX;
			OldY = (int)FloatY;
			z0out = z1out = z2out = z3out = 0;
			if (OldX < 0 || OldX >= OldDim)
				z0out = z1out = 1;
			if (OldY < 0 || OldY >= OldDim)
				z0out = z2out = 1;
			if (OldX + 1 < 0 || OldX + 1 >= OldDim)
				z2out = z3out = 1;
			if (OldY + 1 < 0 || OldY + 1 >= OldDim)
				z1out = z3out = 1;
			z0 = z0out ? 0.0f : Old[OldY * OldDim + OldX];
			z1 = z1out ? 0.0f : Old[(OldY + 1) * OldDim + OldX];
			z2 = z2out ? 0.0f : Old[OldY * OldDim + OldX + 1];
			z3 = z3out ? 0.0f : Old[(OldY + 1) * OldDim + OldX + 1];
			z01 = z0 + (FloatY - OldY) * (z1 - z0);
			z23 = z2 + (FloatY - OldY) * (z3 - z2);
			if (FloatY < 0) {
				z01 = z0;
				z23 = z2;
			}
			z0123 = z01 + (FloatX - OldX) * (z23 - z01);
			if (FloatX < 0)
				z0123 = z01;
			New[NewY * NewDim + NewX] = z0123;
		}
	}
}

int ComputeOrbit(float *pfPixels, IrlParms_t *psParms, float fMargin, float *pfMargins, float fThresh,
	int OrbitType, PrjView_t *psViews)
{
	int iNang = psParms->NumViews, iNdim = psParms->NumPixels, iNumRotPix, iPix, iAng, iRow;
	float fPixSize = psParms->BinWidth, fPixThresh = 0.0f, fMax, fRadius, fSum;
	float *pfRotPix;
	if (OrbitType == 0) {
		for (iAng = 0; iAng < iNang; ++iAng)
			psViews[iAng].CFCR = fMargin;
		return 0;
	} else if (OrbitType > 2 || OrbitType < 0) {
		return 2;
	}
	if (fThresh <= 0.0) {
		fPixThresh = -fThresh;
	} else {
		fMax = pfPixels[0];
		for (iPix = 1; iPix < iNdim * iNdim; ++iPix)
			fMax = pfPixels[iPix] > fMax ? pfPixels[iPix] : fMax;
		fPixThresh = fMax * fThresh;
	}
	for (iPix = 0; iPix < iNdim * iNdim; ++iPix)
		if (pfPixels[iPix] <= fPixThresh)
			pfPixels[iPix] = 0.0;
	iNumRotPix = (int)ceil(sqrt(2.0) * (double)iNdim);
	if ((iNumRotPix % 2) != (iNdim % 2))
		iNumRotPix++;
	pfRotPix = (float *)malloc(sizeof(float) * iNumRotPix * iNumRotPix);
	if (pfRotPix == NULL)
		return 1;
	for (iAng = 0; iAng < iNang; ++iAng) {
		float fAngle = psViews[iAng].Angle;
		int k;
		rot2d((float)(0.5 * M_PI + fAngle), pfPixels, pfRotPix, iNdim, iNumRotPix);
		fSum = 0.0;
		for (iRow = 0; iRow < iNumRotPix / 2 && fSum <= 0.0; ++iRow) {
			fSum = 0.0f;
			for (k = 0; k < iNumRotPix; ++k)
				fSum += pfRotPix[iRow * iNumRotPix + k];
		}
		fRadius = ((float)iNumRotPix / 2.0 - (float)iRow) * fPixSize;
		if (pfMargins != NULL)
			fRadius += pfMargins[iAng];
		else
			fRadius += fMargin;
		psViews[iAng].CFCR = fRadius;
	}
	if (OrbitType == 2) {
		for (iAng = 0; iAng < iNang / 2; ++iAng) {
			if (psViews[iAng].CFCR > psViews[iAng + iNang / 2].CFCR)
				psViews[iAng + iNang / 2].CFCR = psViews[iAng].CFCR;
			else
				psViews[iAng].CFCR = psViews[iAng + iNang / 2].CFCR;
		}
	}
	free(pfRotPix);
	return 0;
}
