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

/* host threads for a job of `work` units: 1 below `min_work` (or on one
 * CPU), else the online CPUs, at most SM_MAX_HOST_THREADS */
#define SM_MAX_HOST_THREADS 16
size_t sm_host_threads(size_t work, size_t min_work);
/* fn(items + k * item_size) for every k < n: item 0 on the calling thread,
 * items 1 .. SM_MAX_HOST_THREADS-1 on threads of their own, any further one
 * (and one whose thread cannot be started) on the caller.  Returns when all
 * have run. */
void sm_parallel(void *(*fn)(void *), void *items, size_t item_size, size_t n);

#ifdef __cplusplus
}
#endif
#endif
