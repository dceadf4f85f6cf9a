/*
 * sm_host.h -- internal declarations shared by the host C files and the
 * CUDA translation units of libseismod_gpu.
 */
#ifndef SM_HOST_H
#define SM_HOST_H

#include <stddef.h>

#include "../../include/seismod_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* record a printf-style message for sm_last_error() on this thread and
 * return code */
int sm_fail(int code, const char *fmt, ...)
#if defined(__GNUC__)
    __attribute__((format(printf, 2, 3)))
#endif
    ;
void sm_clear_error(void);

#ifdef __cplusplus
}
#endif
#endif
