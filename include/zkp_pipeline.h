/*
 * libzkp_pipeline.so: a fused elementwise kernel run over HOST-resident polynomials in chunks,
 * with the host-to-device copies, the kernel and the device-to-host copies of consecutive
 * chunks overlapped.  Replaces the reference's pipelined fused kernel
 * (core/src/fused_kernels.rs:198-516, PipelinedFusedKernel::get_fn; chunk count chosen by
 * common/src/arith.rs:338-356, decide_chunking), which the compiler emits when a fused
 * kernel's operands do not fit device memory.
 *
 * Same protocol as the reference: the element range is cut into `divide_parts` equal chunks
 * (divide_parts > 3 and len % divide_parts == 0, as the reference asserts); input polynomials
 * are double-buffered on the device and mutable polynomials triple-buffered (load, compute,
 * store); chunk k runs the kernel with is_first = (k == 0); scalars (mutable or not) are
 * copied to the device once, and mutable scalars back once at the end.  Three streams carry
 * the host-to-device copies, the kernels and the device-to-host copies; events order them.
 * Host polynomials must be page-locked (cudaHostAlloc / cudaHostRegister) for the copies to
 * overlap; pageable memory gives the same results, serialised.
 *
 * The kernel is any generated fused kernel with the reference's signature
 * (core/src/fused_kernels/kernel_gen.rs:286-307).  A periodic input (an addition of this
 * library's generator: element i read at i mod its length) is passed as a scalar-like
 * argument of `whole` elements that is copied once; it requires chunk_len % whole == 0.
 */
#ifndef ZKP_PIPELINE_H
#define ZKP_PIPELINE_H
#include <cuda_runtime.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif
#include "poly_ptr.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef cudaError_t (*ZkpFusedFn)(const ConstPolyPtr *vars_d, const PolyPtr *mut_vars_d, unsigned long long len,
                                  bool is_first, void *local_buffer_d, cudaStream_t stream);

/* One argument: a polynomial of `len` elements (whole = 0) streamed in chunks, or a whole
 * array of `whole` elements (a scalar: whole = 1; a periodic input: its period) copied once. */
typedef struct ZkpPipelineArg {
    unsigned int *host;            /* host elements (32 bytes each); const for inputs */
    unsigned long long whole;      /* 0 = streamed polynomial of len elements */
    unsigned int write_only;       /* mutable polynomial the kernel only writes: not copied in
                                      (the reference copies every mutable polynomial in) */
} ZkpPipelineArg;

/* Device workspace bytes for a run with these arguments and chunk length len / divide_parts
 * (0 if the arguments are invalid). */
unsigned long long zkp_fused_pipelined_workspace(const ZkpPipelineArg *vars, unsigned int n_vars,
                                                 const ZkpPipelineArg *mut_vars, unsigned int n_mut_vars,
                                                 unsigned long long len, unsigned long long divide_parts);

/* Runs `kernel` over the len elements of the host arguments; returns when the results (mutable
 * polynomials and scalars) are back in host memory.  workspace_d: at least
 * zkp_fused_pipelined_workspace(...) bytes of device memory; local_buffer_d is handed to every
 * kernel call (the reference's spill buffer; the kernels of this library need none). */
cudaError_t zkp_fused_pipelined(ZkpFusedFn kernel, const ZkpPipelineArg *vars, unsigned int n_vars,
                                const ZkpPipelineArg *mut_vars, unsigned int n_mut_vars, unsigned long long len,
                                unsigned long long divide_parts, void *workspace_d,
                                unsigned long long workspace_bytes, void *local_buffer_d);

#ifdef __cplusplus
}
#endif
#endif
