/*
 * errdefs.h -- project-written stand-in for MIP's error handling header.
 * TEST INFRASTRUCTURE ONLY (see miputil.h).
 *
 * libirl's entry points call setjmp() and register the jump buffer with
 * vTrapFatalErrs(); a fatal vErrorHandler() call longjmps there with a
 * non-zero code, and pchErrorMsg() returns the formatted message.
 * Warnings are written to the error log (if any) and execution continues.
 */
#ifndef MIPSHIM_ERRDEFS_H
#define MIPSHIM_ERRDEFS_H

#include <stdio.h>
#include <setjmp.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error classes; gendrf.c also passes the raw numbers 1 and 2 */
#define ECLASS_FATAL 1
#define ECLASS_WARN 2
#define ECLASS_INFO 3

/* error types (values only need to be distinct and non-zero) */
#define ETYPE_MALLOC 1
#define ETYPE_IO 2
#define ETYPE_ILLEGAL_VALUE 3
#define ETYPE_INFO 4
#define ETYPE_SYNTAX 5
#define ETYPE_UNKNOWN 6

void vErrorHandler(int iClass, int iType, char *pchRoutine, char *pchFmt, ...);
void vTrapFatalErrs(jmp_buf *psEnv);
char *pchErrorMsg(void);
void vSetErrLog(FILE *fp);

#ifdef __cplusplus
}
#endif
#endif
