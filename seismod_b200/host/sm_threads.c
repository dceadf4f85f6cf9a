/*
 * sm_threads.c -- the few host threads the set-up and I/O paths split their
 * work over (model padding, text model parsing, trace and snapshot files).
 */
#include "sm_host.h"

#include <pthread.h>
#include <unistd.h>

size_t sm_host_threads(size_t work, size_t min_work)
{
    const long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    if (work < min_work || ncpu < 2) return 1;
    return ncpu > SM_MAX_HOST_THREADS ? SM_MAX_HOST_THREADS : (size_t)ncpu;
}

void sm_parallel(void *(*fn)(void *), void *items, size_t item_size, size_t n)
{
    pthread_t tid[SM_MAX_HOST_THREADS];
    int started[SM_MAX_HOST_THREADS] = {0};
    char *base = (char *)items;
    const size_t nt = n < SM_MAX_HOST_THREADS ? n : SM_MAX_HOST_THREADS;
    for (size_t k = 1; k < nt; ++k)
        started[k] = pthread_create(&tid[k], NULL, fn, base + k * item_size) == 0;
    if (n > 0) fn(base);
    for (size_t k = SM_MAX_HOST_THREADS; k < n; ++k) fn(base + k * item_size);   /* beyond the threads */
    for (size_t k = 1; k < nt; ++k) {
        if (started[k]) pthread_join(tid[k], NULL);
        else fn(base + k * item_size);
    }
}
