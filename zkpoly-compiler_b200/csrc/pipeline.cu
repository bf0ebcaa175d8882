// libzkp_pipeline.so: a generated fused kernel over host-resident polynomials in chunks, with
// copies and kernels of consecutive chunks overlapped on three streams.  Replaces the
// reference's PipelinedFusedKernel (core/src/fused_kernels.rs:198-516) behind the C ABI of
// include/zkp_pipeline.h; the buffering (inputs double-, mutable outputs triple-buffered), the
// event protocol between the copy-in, kernel and copy-out streams, is_first on chunk 0 and the
// one-time scalar copies follow that function.  Host code only: the kernel is the caller's.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/zkp_pipeline.h"

namespace {

constexpr unsigned long long ELEM = 32;  // bytes per field element

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct Plan {
    unsigned long long chunk = 0;
    unsigned n_poly = 0, n_mut_poly = 0;
    size_t args = 0, scalars = 0, polys = 0, mut_polys = 0, total = 0;
    std::vector<size_t> var_whole_off, mut_whole_off;  // offsets of copied-once arrays
};

bool plan(const ZkpPipelineArg *vars, unsigned n_vars, const ZkpPipelineArg *mut, unsigned n_mut,
          unsigned long long len, unsigned long long parts, Plan *p) {
    if (parts <= 3 || len == 0 || len % parts != 0 || (n_vars && !vars) || (n_mut && !mut)) return false;
    p->chunk = len / parts;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += align_up(bytes);
        return o;
    };
    // two input argument arrays (one per input buffer), three mutable ones
    p->args = take((2 * (size_t)n_vars + 3 * (size_t)n_mut) * sizeof(PolyPtr));
    p->var_whole_off.assign(n_vars, 0);
    p->mut_whole_off.assign(n_mut, 0);
    for (unsigned i = 0; i < n_vars; i++) {
        if (!vars[i].host) return false;
        if (vars[i].whole) {
            if (p->chunk % vars[i].whole != 0 && vars[i].whole != 1) return false;
            p->var_whole_off[i] = take(vars[i].whole * ELEM);
        } else {
            p->n_poly++;
        }
    }
    for (unsigned i = 0; i < n_mut; i++) {
        if (!mut[i].host) return false;
        if (mut[i].whole) {
            if (mut[i].whole != 1) return false;  // mutable arrays copied once: scalars only
            p->mut_whole_off[i] = take(ELEM);
        } else {
            p->n_mut_poly++;
        }
    }
    p->polys = take(2 * (size_t)p->n_poly * p->chunk * ELEM);
    p->mut_polys = take(3 * (size_t)p->n_mut_poly * p->chunk * ELEM);
    p->total = off;
    return true;
}

#define PTRY(x)                                    \
    do {                                           \
        cudaError_t e_ = (x);                      \
        if (e_ != cudaSuccess) {                   \
            err = e_;                              \
            goto done;                             \
        }                                          \
    } while (0)

}  // namespace

extern "C" unsigned long long zkp_fused_pipelined_workspace(const ZkpPipelineArg *vars, unsigned int n_vars,
                                                            const ZkpPipelineArg *mut_vars, unsigned int n_mut_vars,
                                                            unsigned long long len, unsigned long long divide_parts) {
    Plan p;
    return plan(vars, n_vars, mut_vars, n_mut_vars, len, divide_parts, &p) ? p.total : 0;
}

extern "C" cudaError_t zkp_fused_pipelined(ZkpFusedFn kernel, const ZkpPipelineArg *vars, unsigned int n_vars,
                                           const ZkpPipelineArg *mut_vars, unsigned int n_mut_vars,
                                           unsigned long long len, unsigned long long divide_parts,
                                           void *workspace_d, unsigned long long workspace_bytes,
                                           void *local_buffer_d) {
    const unsigned n_mut = n_mut_vars;
    Plan p;
    if (!kernel || !workspace_d || !plan(vars, n_vars, mut_vars, n_mut_vars, len, divide_parts, &p) ||
        workspace_bytes < p.total)
        return cudaErrorInvalidValue;
    char *ws = reinterpret_cast<char *>(workspace_d);
    const unsigned long long chunk = p.chunk;
    const size_t chunk_bytes = chunk * ELEM;
    // device buffers: input buffer b holds the chunk of input polynomial j at poly_buf(b, j)
    auto poly_buf = [&](unsigned b, unsigned j) {
        return reinterpret_cast<unsigned int *>(ws + p.polys + ((size_t)b * p.n_poly + j) * chunk_bytes);
    };
    auto mut_buf = [&](unsigned b, unsigned j) {
        return reinterpret_cast<unsigned int *>(ws + p.mut_polys + ((size_t)b * p.n_mut_poly + j) * chunk_bytes);
    };
    // argument arrays, in the kernel's order (the reference's: scalars and polys as the caller
    // lists them); chunk-length views for polynomials, the whole array for copied-once ones
    std::vector<ConstPolyPtr> h_vars(2 * (size_t)n_vars);
    std::vector<PolyPtr> h_mut(3 * (size_t)n_mut);
    for (unsigned b = 0; b < 2; b++) {
        unsigned j = 0;
        for (unsigned i = 0; i < n_vars; i++) {
            ConstPolyPtr &a = h_vars[(size_t)b * n_vars + i];
            if (vars[i].whole) {
                a = {reinterpret_cast<const unsigned int *>(ws + p.var_whole_off[i]), (size_t)vars[i].whole, 0, 0,
                     (size_t)vars[i].whole};
            } else {
                a = {poly_buf(b, j++), (size_t)chunk, 0, 0, (size_t)chunk};
            }
        }
    }
    for (unsigned b = 0; b < 3; b++) {
        unsigned j = 0;
        for (unsigned i = 0; i < n_mut; i++) {
            PolyPtr &a = h_mut[(size_t)b * n_mut + i];
            if (mut_vars[i].whole) {
                a = {reinterpret_cast<unsigned int *>(ws + p.mut_whole_off[i]), 1, 0, 0, 1};
            } else {
                a = {mut_buf(b, j++), (size_t)chunk, 0, 0, (size_t)chunk};
            }
        }
    }
    const ConstPolyPtr *d_vars[2];
    const PolyPtr *d_mut[3];
    {
        ConstPolyPtr *base = reinterpret_cast<ConstPolyPtr *>(ws + p.args);
        d_vars[0] = base;
        d_vars[1] = base + n_vars;
        PolyPtr *mbase = reinterpret_cast<PolyPtr *>(base + 2 * (size_t)n_vars);
        for (unsigned b = 0; b < 3; b++) d_mut[b] = mbase + (size_t)b * n_mut;
    }

    cudaError_t err = cudaSuccess;
    cudaStream_t h2d = nullptr, comp = nullptr, d2h = nullptr;
    cudaEvent_t mut_h2d[3] = {}, mut_comp[3] = {}, mut_d2h[3] = {}, in_h2d[2] = {}, in_comp[2] = {};
    unsigned mb = 0, b = 0;
    PTRY(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
    PTRY(cudaStreamCreateWithFlags(&comp, cudaStreamNonBlocking));
    PTRY(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
    for (int i = 0; i < 3; i++) {
        PTRY(cudaEventCreateWithFlags(&mut_h2d[i], cudaEventDisableTiming));
        PTRY(cudaEventCreateWithFlags(&mut_comp[i], cudaEventDisableTiming));
        PTRY(cudaEventCreateWithFlags(&mut_d2h[i], cudaEventDisableTiming));
    }
    for (int i = 0; i < 2; i++) {
        PTRY(cudaEventCreateWithFlags(&in_h2d[i], cudaEventDisableTiming));
        PTRY(cudaEventCreateWithFlags(&in_comp[i], cudaEventDisableTiming));
    }
    // argument arrays and the copied-once arrays (the host vectors outlive the final sync)
    if (n_vars) PTRY(cudaMemcpyAsync(const_cast<ConstPolyPtr *>(d_vars[0]), h_vars.data(),
                                     h_vars.size() * sizeof(ConstPolyPtr), cudaMemcpyHostToDevice, h2d));
    if (n_mut) PTRY(cudaMemcpyAsync(const_cast<PolyPtr *>(d_mut[0]), h_mut.data(), h_mut.size() * sizeof(PolyPtr),
                                    cudaMemcpyHostToDevice, h2d));
    for (unsigned i = 0; i < n_vars; i++)
        if (vars[i].whole)
            PTRY(cudaMemcpyAsync(ws + p.var_whole_off[i], vars[i].host, vars[i].whole * ELEM, cudaMemcpyHostToDevice,
                                 h2d));
    for (unsigned i = 0; i < n_mut; i++)
        if (mut_vars[i].whole)
            PTRY(cudaMemcpyAsync(ws + p.mut_whole_off[i], mut_vars[i].host, ELEM, cudaMemcpyHostToDevice, h2d));

    for (unsigned long long k = 0; k < divide_parts; k++) {
        const size_t start = (size_t)k * chunk;
        // mutable chunk in (after the store of the chunk that last used this buffer)
        PTRY(cudaStreamWaitEvent(h2d, mut_d2h[mb], 0));
        {
            unsigned j = 0;
            for (unsigned i = 0; i < n_mut; i++) {
                if (mut_vars[i].whole) continue;
                unsigned int *dst = mut_buf(mb, j++);
                if (!mut_vars[i].write_only)
                    PTRY(cudaMemcpyAsync(dst, mut_vars[i].host + start * 8, chunk_bytes, cudaMemcpyHostToDevice,
                                         h2d));
            }
        }
        PTRY(cudaEventRecord(mut_h2d[mb], h2d));
        // input chunk in (after the kernel that last read this buffer)
        PTRY(cudaStreamWaitEvent(h2d, in_comp[b], 0));
        {
            unsigned j = 0;
            for (unsigned i = 0; i < n_vars; i++)
                if (!vars[i].whole)
                    PTRY(cudaMemcpyAsync(poly_buf(b, j++), vars[i].host + start * 8, chunk_bytes,
                                         cudaMemcpyHostToDevice, h2d));
        }
        PTRY(cudaEventRecord(in_h2d[b], h2d));
        // kernel
        PTRY(cudaStreamWaitEvent(comp, mut_h2d[mb], 0));
        PTRY(cudaStreamWaitEvent(comp, in_h2d[b], 0));
        PTRY(kernel(d_vars[b], d_mut[mb], chunk, k == 0, local_buffer_d, comp));
        PTRY(cudaEventRecord(in_comp[b], comp));
        PTRY(cudaEventRecord(mut_comp[mb], comp));
        // mutable chunk out
        PTRY(cudaStreamWaitEvent(d2h, mut_comp[mb], 0));
        {
            unsigned j = 0;
            for (unsigned i = 0; i < n_mut; i++)
                if (!mut_vars[i].whole)
                    PTRY(cudaMemcpyAsync(mut_vars[i].host + start * 8, mut_buf(mb, j++), chunk_bytes,
                                         cudaMemcpyDeviceToHost, d2h));
        }
        PTRY(cudaEventRecord(mut_d2h[mb], d2h));
        mb = (mb + 1) % 3;
        b = (b + 1) % 2;
    }
    // mutable scalars back once
    for (unsigned i = 0; i < n_mut; i++)
        if (mut_vars[i].whole)
            PTRY(cudaMemcpyAsync(mut_vars[i].host, ws + p.mut_whole_off[i], ELEM, cudaMemcpyDeviceToHost, d2h));
done:
    // every stream drains before the streams, events and host argument arrays go away
    for (cudaStream_t s : {h2d, comp, d2h}) {
        if (!s) continue;
        cudaError_t e = cudaStreamSynchronize(s);
        if (err == cudaSuccess) err = e;
    }
    for (int i = 0; i < 3; i++) {
        if (mut_h2d[i]) cudaEventDestroy(mut_h2d[i]);
        if (mut_comp[i]) cudaEventDestroy(mut_comp[i]);
        if (mut_d2h[i]) cudaEventDestroy(mut_d2h[i]);
    }
    for (int i = 0; i < 2; i++) {
        if (in_h2d[i]) cudaEventDestroy(in_h2d[i]);
        if (in_comp[i]) cudaEventDestroy(in_comp[i]);
    }
    for (cudaStream_t s : {h2d, comp, d2h})
        if (s) cudaStreamDestroy(s);
    return err;
}
