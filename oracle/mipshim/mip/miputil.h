/*
 * miputil.h -- project-written stand-in for the utility part of the
 * un-vendored "MIP" library that libirl includes as <mip/miputil.h>.
 *
 * TEST INFRASTRUCTURE ONLY.  This shim exists so that the reference C
 * sources can be compiled, unmodified, into a CPU oracle library.  Nothing
 * in the product links against it.
 *
 * The contract of each routine is inferred from its call sites in libirl
 * (allocation, fills, sums, the axis reorder used at the API boundary and
 * byte swapping for the DRFT/KRNL readers).
 */
#ifndef MIPSHIM_MIPUTIL_H
#define MIPSHIM_MIPUTIL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* float allocation; aborts through the fatal-error trap on failure */
float *vector(int n, char *name);
int *ivector(int n, char *name);
void free_vector(void *p);

void *pvIrlMalloc(size_t n, char *name);
void *pvIrlRealloc(void *p, size_t n, char *name);
void IrlFree(void *p);
char *pchIrlStrdup(char *s);
void vFreeAllMem(void);

void set_float(float *p, int n, float v);
float sum_float(float *p, int n);
void scale_float(float *p, int n, float s);
void vZeroNeg(float *p, int n);

/*
 * reorder(d0, d1, d2, in, out): `in` is a d0 x d1 x d2 array (d2 fastest);
 * `out` receives the same data with the two slow axes exchanged, i.e. a
 * d1 x d0 x d2 array:  out[j][k][i] = in[k][j][i].  Returns out.
 */
float *reorder(int d0, int d1, int d2, float *in, float *out);

/* reverses the byte order of n consecutive 4-byte words in place */
void vSwapWords(void *p, int n);

void PrintTimes(char *label);

#ifdef __cplusplus
}
#endif
#endif
