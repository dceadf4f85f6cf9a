/*
 * sm_error.c -- per-thread error message behind sm_last_error().
 */
#include "sm_host.h"

#include <stdarg.h>
#include <stdio.h>

static _Thread_local char sm_err_buf[512];

int sm_fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(sm_err_buf, sizeof sm_err_buf, fmt, ap);
    va_end(ap);
    return code;
}

void sm_clear_error(void) { sm_err_buf[0] = '\0'; }

const char *sm_last_error(void) { return sm_err_buf; }

int sm_abi_version(void) { return SM_ABI_VERSION; }
