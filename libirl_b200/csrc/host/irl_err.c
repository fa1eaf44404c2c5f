/*
 * irl_err.c -- fatal-error trap, warnings and leveled messages.
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "irl_err.h"
#include "irlcu.h"

static jmp_buf *g_env = NULL;
static char g_msg[1024] = "";
static int g_level = 0;
static FILE *g_msgfp = NULL;
static FILE *g_logfp = NULL;

void irl_trap(jmp_buf *env) { g_env = env; }
void irl_untrap(void) { g_env = NULL; }
void irl_set_msg_level(int level) { g_level = level; }
void irl_set_msg_file(FILE *fp) { g_msgfp = fp; }
void irl_set_log_file(FILE *fp) { g_logfp = fp; }
const char *irl_last_error(void) { return g_msg; }

void irl_fatal(int code, const char *where, const char *fmt, ...)
{
	va_list ap;
	char body[900];
	va_start(ap, fmt);
	vsnprintf(body, sizeof(body), fmt, ap);
	va_end(ap);
	snprintf(g_msg, sizeof(g_msg), "%s: %s", where, body);
	if (g_logfp != NULL)
		fprintf(g_logfp, "FATAL ERROR %s\n", g_msg);
	if (g_env != NULL)
		longjmp(*g_env, code > 0 ? code : 1);
	fprintf(stderr, "libirl_b200: untrapped fatal error: %s\n", g_msg);
	abort();
}

void irl_warn(const char *where, const char *fmt, ...)
{
	va_list ap;
	if (g_logfp == NULL)
		return;
	fprintf(g_logfp, "WARNING %s: ", where);
	va_start(ap, fmt);
	vfprintf(g_logfp, fmt, ap);
	va_end(ap);
	fputc('\n', g_logfp);
}

void irl_msg(int level, const char *fmt, ...)
{
	va_list ap;
	if (g_msgfp == NULL || level > g_level)
		return;
	va_start(ap, fmt);
	vfprintf(g_msgfp, fmt, ap);
	va_end(ap);
	fflush(g_msgfp);
}

void *irl_malloc(size_t n, const char *what)
{
	void *p = malloc(n ? n : 1);
	if (p == NULL)
		irl_fatal(IRL_E_MALLOC, "irl_malloc", "out of memory allocating %s (%zu bytes)", what, n);
	return p;
}

void *irl_calloc(size_t n, const char *what)
{
	void *p = calloc(n ? n : 1, 1);
	if (p == NULL)
		irl_fatal(IRL_E_MALLOC, "irl_calloc", "out of memory allocating %s (%zu bytes)", what, n);
	return p;
}

char *irl_strdup(const char *s)
{
	size_t n = strlen(s) + 1;
	char *p = (char *)irl_malloc(n, "string");
	memcpy(p, s, n);
	return p;
}

void irl_cu(int status, const char *where)
{
	if (status != IRLCU_OK)
		irl_fatal(IRL_E_DEVICE, where, "%s", irlcu_error_string());
}
