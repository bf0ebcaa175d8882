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
/* Admission policy for the latency tail of a mixed-size load, which is made of its largest
 * requests (all fields 0 = the default: one priority, no class limit).  Requests whose planned
 * footprint is at least priority_bytes run on their slot's high-priority stream, so their
 * blocks are scheduled ahead of those of requests admitted around them; at most
 * max_large_inflight requests of at least large_bytes run at once (smaller requests are
 * admitted past a waiting large one, within the look-ahead).  Applies to admissions from now
 * on. */
typedef struct ZkpServePolicy {
    unsigned long long priority_bytes;
    unsigned long long large_bytes;
    unsigned int max_large_inflight;
} ZkpServePolicy;
void zkp_serve_set_policy(ZkpServer *s, const ZkpServePolicy *policy);
double zkp_serve_now(const ZkpServer *s);
void zkp_serve_destroy(ZkpServer *s);

/* ---- compiled programs (the served form of a compiled artifact's instruction chunk)
 * The reference's runtime interprets a program's instruction chunk (runtime/src/runtime.rs:
 * 210-520 over InstructionNode, runtime/src/instructions.rs:51-178).  Here the host side
 * (program.py) resolves a chunk's variables once - allocations to offsets inside a request's
 * device block (HBM arena) or host block (pinned, per slot), rotations / slices / loaded
 * constants / inputs to views - and lowers every data-moving or computing instruction to one
 * ZkpProgOp below.  The served loop then admits requests of that program by its planned
 * device footprint and runs its ops in order on the request's stream, so requests of
 * different programs and sizes overlap on the GPU like the built-in prover program. */

#define ZKP_PROG_MAX_VIEWS 16

enum ZkpProgSpace {
    ZKP_SPACE_NONE = 0,
    ZKP_SPACE_DEVICE = 1,   /* byte offset inside the request's device block */
    ZKP_SPACE_HOST = 2,     /* byte offset inside the request's pinned host block */
    ZKP_SPACE_ABS = 3,      /* absolute device address (a resident constant) */
    ZKP_SPACE_INPUT = 4     /* byte offset inside the request's input buffer `index` (host) */
};

/* a polynomial / scalar / buffer operand: element i is at
 * base + ((i + offset + whole_len - rotate) mod whole_len) * elem_bytes (PolyPtr rules) */
typedef struct ZkpProgView {
    unsigned int space;
    unsigned int index;
    unsigned long long addr;
    unsigned long long len, rotate, offset, whole_len;
} ZkpProgView;

enum ZkpProgOpKind {
    ZKP_OP_COPY = 1,            /* v0 <- v1 element by element; imm0 = element bytes (32, 64) */
    ZKP_OP_ZERO = 2,            /* v0 <- 0; imm0 = element bytes */
    ZKP_OP_NTT = 3,             /* NttPrcompute: v0 poly, v1 root table (ABS); imm0 = Shoup table (ABS) or 0 */
    ZKP_OP_NTT_RECOMPUTE = 4,   /* NttRecompute: v0 poly, v1 pq, v2 omegas; imm0 = pq_deg */
    ZKP_OP_DISTRIBUTE = 5,      /* DistributePowers: v0 poly, v1 powers */
    ZKP_OP_FUSED = 6,           /* FusedArith: imm0 = kernel function, imm1 = num_vars, imm2 = num_mut_vars,
                                   imm3 = len; v[0..nv) vars, v[nv..nv+nm) mut vars; v14 = device argument
                                   buffer, v15 = host staging (both sized for the PolyPtr arrays) */
    ZKP_OP_MSM = 7,             /* Msm: imm0 = tables (ABS), imm1 = n_tables | window << 16, imm2 = rows,
                                   imm3 = tasks m <= 7; v[0..m) scalars, v[m..2m) results (64 B each),
                                   v15 = device workspace */
    ZKP_OP_EVAL = 8,            /* EvaluatePoly: v0 temp, v1 res, v2 poly, v3 x */
    ZKP_OP_INVERT = 9,          /* BatchedInvert: v0 temp, v1 poly */
    ZKP_OP_KATE = 10,           /* KateDivision: v0 temp, v1 q, v2 p, v3 b */
    ZKP_OP_SCAN = 11,           /* the scan of ScanMul (its two copies are COPY ops): v0 temp, v1 target */
    ZKP_OP_ADD = 12,            /* PolyAdd: v0 r, v1 a, v2 b */
    ZKP_OP_SUB = 13,            /* PolySub: v0 r, v1 a, v2 b */
    ZKP_OP_ZERO_POLY = 14,      /* NewZero: v0 */
    ZKP_OP_ONE_LAGRANGE = 15,   /* NewOneLagrange: v0 */
    ZKP_OP_ONE_COEF = 16,       /* NewOneCoef: v0 */
    ZKP_OP_SCALAR_INV = 17,     /* ScalarInvert: v0 */
    ZKP_OP_SCALAR_POW = 18      /* ScalarPow: v0; imm0 = exponent */
};

typedef struct ZkpProgOp {
    unsigned int kind;
    unsigned int n_views;
    unsigned long long imm[4];
    ZkpProgView v[ZKP_PROG_MAX_VIEWS];
} ZkpProgOp;

/* one returned value: `bytes` bytes at `host_offset` of the host block, copied into the
 * caller's result buffer at `result_offset` when the request completes */
typedef struct ZkpProgOut {
    unsigned long long host_offset, bytes, result_offset;
} ZkpProgOut;

typedef struct ZkpProgram ZkpProgram;

/* Registers a lowered program with the server (the ops are copied; the absolute addresses
 * they name must stay valid while the program exists).  device_bytes is the planned HBM
 * footprint of one request, host_bytes its pinned host block, input_bytes[i] the size of the
 * host buffer input i must hold.  Fails with cudaErrorInvalidValue on a malformed op
 * (unknown kind, too many views, a view outside its block or input, an output outside the
 * host block). */
cudaError_t zkp_serve_program_create(ZkpServer *s, const ZkpProgOp *ops, unsigned int n_ops,
                                     unsigned long long device_bytes, unsigned long long host_bytes,
                                     const ZkpProgOut *outs, unsigned int n_outs,
                                     const unsigned long long *input_bytes, unsigned int n_inputs,
                                     ZkpProgram **out);
/* Non-blocking, like zkp_serve_submit: inputs[0..n_inputs) are host buffers (of at least the
 * registered sizes) the program's LoadInput instructions read, `results` receives the outputs
 * (results_bytes >= the outputs' extent, else cudaErrorInvalidValue is the request's error and
 * status -1); both must stay valid until the request completes (zkp_serve_wait).  The
 * request's ZkpProverResult carries status, times and footprint; msm / evals are unused. */
long long zkp_serve_submit_program(ZkpServer *s, const ZkpProgram *prog, const void *const *inputs,
                                   unsigned int n_inputs, void *results, unsigned long long results_bytes);
/* Destroys a program.  Its requests still pending or running complete normally and the last
 * of them releases it; no request may be submitted to it afterwards. */
void zkp_serve_program_destroy(ZkpServer *s, ZkpProgram *prog);

#ifdef __cplusplus
}
#endif
#endif
