/*
 * libzkp_runtime.so: the served form - a continuous-batching request loop for prover-shaped
 * programs on one GPU (no counterpart symbol in the reference; it takes the role of the
 * reference's scheduler, scheduler/src/scheduler.rs:255-426 and scheduler/src/scheduler/
 * core.rs:197-350, and of its memory pool, memory_pool/src/lib.rs, for device memory).
 *
 * A server owns one HBM arena (the admission budget), the resident bases and the per-size
 * constants (root tables, n^-1, 1/Z_H on the coset).  Requests are admitted in arrival order
 * as soon as a slot (stream) is free and the request's planned HBM footprint fits in the
 * arena; admitted requests run concurrently on their own streams and release their memory on
 * completion.  With max_inflight = 1 the same server is the plain per-call path.
 *
 * Program of a request of size k (n = 2^k, N = 2^(k+ext)), all inputs seeded uniform Fr:
 *   a, b, c <- INTT(a), INTT(b), INTT(c)          (three inverse NTTs, n^-1 fused)
 *   e <- coset NTT of c on the 2^ext-times extended domain (shift 7)
 *   q <- (e*e - e - z*z(wX)) / Z_H               (one fused kernel; z seeded on the coset)
 *   msm[0..3] <- MSM(bases, a), (bases, b), (bases, c), (bases, q[0..n))   (one batched launch set)
 *   eval[0..1] <- a(x), b(x)                      (x seeded)
 */
#ifndef ZKP_RUNTIME_H
#define ZKP_RUNTIME_H
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ZkpServer ZkpServer;

/* One set of resident MSM bases: n_tables tables of `rows` affine points (table j starts at
 * point j * rows and holds 2^(j*Wp*window) * P).  A request of size k reads the first 2^k rows
 * of each table. */
typedef struct ZkpServeTableSet {
    const unsigned int *tables_d;
    unsigned long long rows;       /* >= 2^max_k */
    unsigned int window;           /* 0 = library default per size (one table only) */
    unsigned int n_tables;
    unsigned int max_k;            /* the set serves requests of size k <= max_k */
} ZkpServeTableSet;

#define ZKP_SERVE_MAX_SETS 8

typedef struct ZkpServeConfig {
    unsigned long long hbm_bytes;  /* arena size = admission budget for request buffers */
    unsigned int max_inflight;     /* concurrent requests (streams); 1 = plain per-call path */
    unsigned int ext_log;          /* log2 of the coset extension (2 for 4x) */
    unsigned int min_k, max_k;     /* request sizes the server prepares constants for */
    unsigned int msm_window;       /* 0 = library default per size (one table only) */
    unsigned int msm_tables;       /* precomputed tables in bases_d (1 = none); table j holds
                                      2^(j*Wp*msm_window) * P for all n_bases points */
    unsigned int n_sets;           /* 0: one set (bases_d, msm_window, msm_tables) for every
                                      size; else sets[0..n_sets) by ascending max_k, and a
                                      request of size k uses the first set with max_k >= k
                                      (bases_d is then ignored) */
    ZkpServeTableSet sets[ZKP_SERVE_MAX_SETS];
} ZkpServeConfig;

typedef struct ZkpProverRequest {
    unsigned int k;
    unsigned long long seed;       /* inputs a, b, c, z, x are drawn from seed*8 + {0..4} */
    unsigned int inject_fault;     /* host-side fault injection for tests: 1 = allocation
                                      refused, 2 = a launch returns an error */
} ZkpProverRequest;

typedef struct ZkpProverResult {
    int status;                    /* 0 ok; -1 invalid request; -2 larger than the arena;
                                      -3 device/launch error; -4 injected allocation failure */
    unsigned int msm[4][16];       /* affine points */
    unsigned int evals[2][8];
    double submit_s, start_s, done_s;  /* server clock (seconds since creation) */
    unsigned long long footprint;
} ZkpProverResult;

typedef struct ZkpServeStats {
    unsigned long long completed, failed, peak_inflight, peak_bytes, arena_bytes;
} ZkpServeStats;

/* bases_d: msm_tables tables of n_bases affine points resident on the current device
 * (n_bases >= 2^max_k), e.g. built by zkp_msm_precompute_device; or null with n_sets > 0 (a
 * window and table count tuned per size range). */
cudaError_t zkp_serve_create(const ZkpServeConfig *cfg, const unsigned int *bases_d, unsigned long long n_bases,
                             ZkpServer **out);
/* Non-blocking; returns a ticket >= 0.  A malformed request (k outside [min_k, max_k]) or one
 * larger than the whole arena still gets a ticket; its result carries status -1 / -2 and it
 * never touches the device.  Returns -1 only when the server is shutting down. */
long long zkp_serve_submit(ZkpServer *s, const ZkpProverRequest *req);
/* Planned HBM footprint of a request of size k (bytes). */
unsigned long long zkp_serve_footprint(const ZkpServer *s, unsigned int k);
/* Blocks until the ticket completes or timeout_s elapses: returns 0 when done, 1 on timeout. */
int zkp_serve_wait(ZkpServer *s, long long ticket, ZkpProverResult *out, double timeout_s);
void zkp_serve_stats(const ZkpServer *s, ZkpServeStats *out);
double zkp_serve_now(const ZkpServer *s);
void zkp_serve_destroy(ZkpServer *s);

#ifdef __cplusplus
}
#endif
#endif
