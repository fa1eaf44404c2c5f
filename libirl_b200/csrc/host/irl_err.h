/*
 * irl_err.h -- fatal-error trap, warnings and leveled messages of the
 * libirl_b200 host library.
 *
 * The public entry points arm a setjmp trap; irl_fatal() formats the
 * message (returned later by pchIrlErrorString) and longjmps back so the
 * entry point can free everything and return the non-zero code, as libirl
 * does (irlosem.c:104-111, 258-284).
 */
#ifndef IRL_ERR_H
#define IRL_ERR_H

#include <setjmp.h>
#include <stdio.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes returned by IrlOsem / IrlGenprj */
#define IRL_E_MALLOC 1
#define IRL_E_IO 2
#define IRL_E_VALUE 3
#define IRL_E_DEVICE 4

void irl_trap(jmp_buf *env);
void irl_untrap(void);
void irl_fatal(int code, const char *where, const char *fmt, ...);
void irl_warn(const char *where, const char *fmt, ...);
void irl_msg(int level, const char *fmt, ...);
void irl_set_msg_level(int level);
void irl_set_msg_file(FILE *fp);
void irl_set_log_file(FILE *fp);
const char *irl_last_error(void);

void *irl_malloc(size_t n, const char *what);
void *irl_calloc(size_t n, const char *what);
char *irl_strdup(const char *s);

/* checks an irlcu status; fatal with the device message on failure */
void irl_cu(int status, const char *where);

#ifdef __cplusplus
}
#endif
#endif
