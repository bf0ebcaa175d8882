// Shared helpers for the CUDA libraries: PolyPtr views, error propagation, launch set-up.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>

#include "../../include/poly_ptr.h"
#include "field.cuh"

namespace zk {

#define ZK_TRY(expr)                                  \
    do {                                              \
        cudaError_t zk_err__ = (expr);                \
        if (zk_err__ != cudaSuccess) return zk_err__; \
    } while (0)

#define ZK_CHECK_ARG(cond)                                   \
    do {                                                     \
        if (!(cond)) return cudaErrorInvalidValue;           \
    } while (0)

// A resolved PolyPtr: element i sits at base[(off + i) mod whole] (whole >= len, off < whole).
// The kernels avoid the reference's per-access `%` (iter.cuh:63): off + i < 2 * whole, so one
// compare-and-subtract maps it.
struct View {
    u32 *base;
    u64 off;
    u64 whole;
    u64 len;

    ZK_DI u64 phys(u64 i) const {
        u64 p = off + i;
        return p >= whole ? p - whole : p;
    }
    ZK_DI u32 *at(u64 i) const { return base + phys(i) * 8; }
};

// iter.cuh:308-327: rotate r -> offset = len - r, only on whole, unsliced arrays
inline bool make_view(const u32 *ptr, size_t len, size_t rotate, size_t offset, size_t whole_len, View *v) {
    size_t whole = whole_len == 0 ? len : whole_len;
    if (len > whole) return false;
    size_t off = offset;
    if (rotate != 0) {
        if (len != whole || offset != 0 || rotate > len) return false;
        off = len - rotate;
        if (off == len) off = 0;
    }
    if (len > 0 && off >= whole) return false;
    if (len > 0 && ptr == nullptr) return false;
    if ((reinterpret_cast<uintptr_t>(ptr) & 15) != 0) return false;  // 128-bit element access
    v->base = const_cast<u32 *>(ptr);
    v->off = off;
    v->whole = whole;
    v->len = len;
    return true;
}

inline bool make_view(const PolyPtr &p, View *v) { return make_view(p.ptr, p.len, p.rotate, p.offset, p.whole_len, v); }
inline bool make_view(const ConstPolyPtr &p, View *v) {
    return make_view(p.ptr, p.len, p.rotate, p.offset, p.whole_len, v);
}

// true when the view is one contiguous run (no wrap-around)
inline bool contiguous(const View &v) { return v.off + v.len <= v.whole; }

// Sets the dynamic shared-memory limit of a kernel once per device.  Racing first callers
// may both set it, which is harmless; no lock is held on the launch path.
template <typename K>
inline cudaError_t ensure_smem_attr(K kernel, int bytes, std::atomic<uint64_t> &done_mask) {
    int dev = 0;
    ZK_TRY(cudaGetDevice(&dev));
    const uint64_t bit = 1ull << (dev & 63);
    if (done_mask.load(std::memory_order_acquire) & bit) return cudaSuccess;
    ZK_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done_mask.fetch_or(bit, std::memory_order_acq_rel);
    return cudaSuccess;
}

inline int num_sms() {
    static std::atomic<int> cached{0};
    int v = cached.load();
    if (v) return v;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    if (v <= 0) v = 148;
    cached.store(v);
    return v;
}

}  // namespace zk

namespace zk {
// Stage timing with CUDA events on the launching stream, for the benchmark harness.  Off by
// default; when on, a library records an event at each stage boundary of its last call.
struct StageProfiler {
    static constexpr int MAX = 32;
    bool on = false;
    int n = 0;
    const char *names[MAX];
    cudaEvent_t ev[MAX + 1];
    bool created = false;

    void begin(cudaStream_t s) {
        if (!on) return;
        if (!created) {
            for (int i = 0; i <= MAX; i++) cudaEventCreate(&ev[i]);
            created = true;
        }
        n = 0;
        cudaEventRecord(ev[0], s);
    }
    // closes the stage that started at the previous mark
    void mark(const char *name, cudaStream_t s) {
        if (!on || n >= MAX) return;
        names[n] = name;
        n++;
        cudaEventRecord(ev[n], s);
    }
    int read(float *ms, const char **out_names, int max) {
        if (!created || n == 0) return 0;
        cudaEventSynchronize(ev[n]);
        int k = n < max ? n : max;
        for (int i = 0; i < k; i++) {
            cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
            out_names[i] = names[i];
        }
        return k;
    }
};

inline StageProfiler &profiler() {
    static StageProfiler p;
    return p;
}
}  // namespace zk

// per-library profiling entry points (each shared object carries its own profiler)
#define ZK_DEFINE_PROFILER_API(prefix)                                                               \
    extern "C" void prefix##_profile_enable(int on) { zk::profiler().on = on != 0; }                 \
    extern "C" int prefix##_profile_read(float *ms, const char **names, int max) {                   \
        return zk::profiler().read(ms, names, max);                                                  \
    }
