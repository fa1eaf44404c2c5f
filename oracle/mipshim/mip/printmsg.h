/*
 * printmsg.h -- project-written stand-in for MIP's leveled message output.
 * TEST INFRASTRUCTURE ONLY (see miputil.h).
 */
#ifndef MIPSHIM_PRINTMSG_H
#define MIPSHIM_PRINTMSG_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

void vPrintMsg(int iLevel, char *pchFmt, ...);
void vSetMsgLevel(int iLevel);
void vSetAllMsgFilePtr(FILE *fp);

#ifdef __cplusplus
}
#endif
#endif
