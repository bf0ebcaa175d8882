// Device runtime for generated fused elementwise kernels.
//
// A generated kernel receives the reference's arguments (core/src/fused_kernels/
// kernel_gen.rs:286-307): device arrays of ConstPolyPtr / PolyPtr, the element count, the
// is_first flag of pipelined chunks, a local (spill) buffer and a stream.  Each block resolves
// the PolyPtr structs once into Views in shared memory; the element loop then reads and writes
// through View::at (no per-access 64-bit `%`, unlike SliceIterator, iter.cuh:63).
#pragma once
#include "common.cuh"

namespace zk {
namespace fused {

// device twin of make_view; an invalid view (rotate on a slice, len > whole_len) yields
// len == 0, which the host wrapper rejects before launch
ZK_DI View device_view(const PolyPtr &p) {
    View v;
    const u64 whole = p.whole_len == 0 ? p.len : p.whole_len;
    u64 off = p.offset;
    if (p.rotate != 0) {
        off = p.len - p.rotate;
        if (off == p.len) off = 0;
    }
    v.base = p.ptr;
    v.off = off;
    v.whole = whole;
    v.len = p.len;
    return v;
}

ZK_DI View device_view(const ConstPolyPtr &p) {
    PolyPtr q;
    q.ptr = const_cast<u32 *>(p.ptr);
    q.len = p.len;
    q.rotate = p.rotate;
    q.offset = p.offset;
    q.whole_len = p.whole_len;
    return device_view(q);
}

// index into a periodic input for element i (its length divides the kernel length)
ZK_DI u64 periodic_index(const View &v, u64 i) {
    return (v.len & (v.len - 1)) == 0 ? (i & (v.len - 1)) : (i % v.len);
}

// element i of a periodic input
ZK_DI u32 *periodic_at(const View &v, u64 i) { return v.at(periodic_index(v, i)); }

// Products by a fixed factor (a scalar input, or a periodic input of at most SHOUP_PERIOD_MAX
// entries) use Fr::mul_shoup: each CTA turns the factor's values into (w, ws) pairs in shared
// memory once, 16 words per value, and every element's product reads them from there.
constexpr u32 SHOUP_PERIOD_MAX = 64;

// pairs for `count` Montgomery values at v[0..count) into sm (16 words each); the caller syncs
ZK_DI void shoup_pairs(const View &v, u64 count, u32 *sm) {
    for (u64 k = threadIdx.x; k < count; k += blockDim.x) {
        Fr w, ws;
        Fr::mul_shoup_table_entry(Fr::load(v.at(k)), &w, &ws);
        w.store(sm + k * 16);
        ws.store(sm + k * 16 + 8);
    }
}

inline u32 fused_grid(u64 len, u32 block) {
    const u64 blocks = (len + block - 1) / block;
    const u64 cap = (u64)num_sms() * 8;
    return (u32)(blocks < cap ? (blocks ? blocks : 1) : cap);
}

}  // namespace fused
}  // namespace zk
