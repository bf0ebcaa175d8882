/* Oracle (test infrastructure only): thread helpers for the CPU restatement. */
#include "util.h"
#include "oracle.h"
#include <pthread.h>
#include <stdlib.h>
#include <unistd.h>

static int n_threads = 0;

void or_set_threads(int n) { n_threads = n; }

int or_get_threads(void) {
    if (n_threads > 0) return n_threads;
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

typedef struct { or_range_fn fn; void *ctx; size_t lo, hi; } task_t;

static void *run_task(void *p) {
    task_t *t = (task_t *)p;
    t->fn(t->ctx, t->lo, t->hi);
    return NULL;
}

void or_parallel_for(size_t n, size_t min_chunk, or_range_fn fn, void *ctx) {
    if (n == 0) return;
    size_t th = (size_t)or_get_threads();
    if (min_chunk == 0) min_chunk = 1;
    size_t max_by_chunk = (n + min_chunk - 1) / min_chunk;
    if (th > max_by_chunk) th = max_by_chunk;
    if (th <= 1) {
        fn(ctx, 0, n);
        return;
    }
    pthread_t *ids = (pthread_t *)malloc(th * sizeof(pthread_t));
    task_t *ts = (task_t *)malloc(th * sizeof(task_t));
    size_t per = n / th, rem = n % th, lo = 0;
    for (size_t i = 0; i < th; i++) {
        size_t len = per + (i < rem ? 1 : 0);
        ts[i].fn = fn; ts[i].ctx = ctx; ts[i].lo = lo; ts[i].hi = lo + len;
        lo += len;
        pthread_create(&ids[i], NULL, run_task, &ts[i]);
    }
    for (size_t i = 0; i < th; i++) pthread_join(ids[i], NULL);
    free(ids);
    free(ts);
}

void or_parallel_tasks(size_t k, or_range_fn fn, void *ctx) {
    if (k == 0) return;
    if (k == 1) { fn(ctx, 0, 1); return; }
    pthread_t *ids = (pthread_t *)malloc(k * sizeof(pthread_t));
    task_t *ts = (task_t *)malloc(k * sizeof(task_t));
    for (size_t i = 0; i < k; i++) {
        ts[i].fn = fn; ts[i].ctx = ctx; ts[i].lo = i; ts[i].hi = i + 1;
        pthread_create(&ids[i], NULL, run_task, &ts[i]);
    }
    for (size_t i = 0; i < k; i++) pthread_join(ids[i], NULL);
    free(ids);
    free(ts);
}
