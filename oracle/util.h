/* Oracle (test infrastructure only): a small pthread parallel-for used by the CPU restatement. */
#ifndef ZKP_ORACLE_UTIL_H
#define ZKP_ORACLE_UTIL_H
#include <stddef.h>
typedef void (*or_range_fn)(void *ctx, size_t lo, size_t hi);
/* split [0, n) into contiguous ranges of at least min_chunk and run them on the oracle's threads */
void or_parallel_for(size_t n, size_t min_chunk, or_range_fn fn, void *ctx);
/* run fn(ctx, i, i+1) for i in [0, k) concurrently, one thread each */
void or_parallel_tasks(size_t k, or_range_fn fn, void *ctx);
#endif
