// permute: the lookup-argument permutation of a prover's lookup (reference poly.h:28,
// permute.cuh:74-222; the expected output is restated in core/tests/poly.rs:569-700).
//
// Over the first `usable` rows: res_input = the input values sorted ascending by canonical value;
// res_table holds, at the first row of every run of equal values in res_input, that value
// (one occurrence taken from the table), and at every other row the table values left over,
// ascending, in row order.  Every input value must occur in the table (as the reference
// requires).  Outputs are Montgomery form.
//
// Steps: canonical keys (32 bytes, most significant word first for the sort), two radix sorts,
// run starts of the sorted input, a binary search of each run's value in the sorted table that
// marks the entry it takes, two exclusive scans (run starts; free table entries), the
// compaction of the free entries, and one pass that writes both outputs.  Sorting and scanning
// use CUB (CUDA toolkit headers), the rest is kernels of this library.
#pragma once
#include <cub/cub.cuh>

namespace zk {
namespace perm {

struct __align__(16) Key {
    u32 w[8];  // canonical value, little-endian words
};

struct KeyOrder {  // most significant word first
    __host__ __device__ ::cuda::std::tuple<u32 &, u32 &, u32 &, u32 &, u32 &, u32 &, u32 &, u32 &> operator()(
        Key &k) const {
        return {k.w[7], k.w[6], k.w[5], k.w[4], k.w[3], k.w[2], k.w[1], k.w[0]};
    }
};

ZK_DI bool key_eq(const Key &a, const Key &b) {
    u32 d = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) d |= a.w[i] ^ b.w[i];
    return d == 0;
}
ZK_DI bool key_lt(const Key &a, const Key &b) {
#pragma unroll
    for (int i = 7; i >= 0; i--)
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i];
    return false;
}

__global__ void __launch_bounds__(256) to_key_kernel(View src, u64 n, Key *out) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Fr x = Fr::load(src.at(i)).to_number();
    Key k;
#pragma unroll
    for (int w = 0; w < 8; w++) k.w[w] = x.v[w];
    out[i] = k;
}

// first[i] = 1 at the first row of a run of equal sorted inputs; free_[i] = 1 (table entries
// start free)
__global__ void __launch_bounds__(256) runs_kernel(const Key *a, u64 n, u32 *first, u32 *free_) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    first[i] = (i == 0 || !key_eq(a[i], a[i - 1])) ? 1u : 0u;
    free_[i] = 1u;
}

// the run starting at i takes one table entry of its value (any of equal entries)
__global__ void __launch_bounds__(256) take_kernel(const Key *a, const u32 *first, const Key *t, u64 n, u32 *free_) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !first[i]) return;
    const Key goal = a[i];
    u64 lo = 0, hi = n;  // first entry not less than goal
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (key_lt(t[mid], goal)) lo = mid + 1; else hi = mid;
    }
    if (lo < n && key_eq(t[lo], goal)) free_[lo] = 0u;  // runs have distinct values: no race
}

__global__ void __launch_bounds__(256) compact_kernel(const Key *t, const u32 *free_, const u32 *lpos, u64 n,
                                                     Key *left) {
    const u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || !free_[j]) return;
    left[lpos[j]] = t[j];
}

__global__ void __launch_bounds__(256) output_kernel(const Key *a, const u32 *first, const u32 *fpos, const Key *left,
                                                    u64 n, View res_input, View res_table) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // a repeated row i takes leftover number (rows before i that are not run starts)
    const Key &kt = first[i] ? a[i] : left[i - fpos[i]];
    Fr x, y;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        x.v[w] = a[i].w[w];
        y.v[w] = kt.w[w];
    }
    Fr::to_mont(x).store(res_input.at(i));
    Fr::to_mont(y).store(res_table.at(i));
}

struct Layout {
    size_t keys_in, keys_a, keys_t, first, fpos, free_, lpos, left, cub, total, cub_bytes;
};

inline Layout layout(u64 n) {
    Layout l{};
    size_t off = 0;
    auto take = [&](size_t b) {
        const size_t o = off;
        off += (b + 255) & ~(size_t)255;
        return o;
    };
    l.keys_in = take(n * sizeof(Key));
    l.keys_a = take(n * sizeof(Key));
    l.keys_t = take(n * sizeof(Key));
    l.first = take(n * 4);
    l.fpos = take(n * 4);
    l.free_ = take(n * 4);
    l.lpos = take(n * 4);
    l.left = take(n * sizeof(Key));
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, (Key *)nullptr, (Key *)nullptr, (int)n, KeyOrder());
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (u32 *)nullptr, (u32 *)nullptr, (int)n);
    l.cub_bytes = sort_bytes > scan_bytes ? sort_bytes : scan_bytes;
    l.cub = take(l.cub_bytes);
    l.total = off;
    return l;
}

}  // namespace perm
}  // namespace zk

extern "C" cudaError_t permute(void *temp_buffer, unsigned long *buffer_size, unsigned long usable, ConstPolyPtr input,
                               ConstPolyPtr table, PolyPtr res_input, PolyPtr res_table, cudaStream_t stream) {
    using namespace zk;
    ZK_CHECK_ARG(usable < (1ull << 31));  // CUB item counts are int
    const perm::Layout l = perm::layout(usable);
    if (temp_buffer == nullptr) {
        ZK_CHECK_ARG(buffer_size != nullptr);
        *buffer_size = l.total;
        return cudaSuccess;
    }
    ZK_CHECK_ARG(buffer_size == nullptr || *buffer_size >= l.total);
    ZK_CHECK_ARG(input.len == table.len && usable <= input.len && res_input.len == usable && res_table.len == usable);
    if (usable == 0) return cudaSuccess;
    View vin, vtab, vri, vrt;
    ZK_CHECK_ARG(make_view(input, &vin) && make_view(table, &vtab) && make_view(res_input, &vri) &&
                 make_view(res_table, &vrt));
    char *base = reinterpret_cast<char *>(temp_buffer);
    auto *keys_in = reinterpret_cast<perm::Key *>(base + l.keys_in);
    auto *keys_a = reinterpret_cast<perm::Key *>(base + l.keys_a);
    auto *keys_t = reinterpret_cast<perm::Key *>(base + l.keys_t);
    auto *first = reinterpret_cast<u32 *>(base + l.first);
    auto *fpos = reinterpret_cast<u32 *>(base + l.fpos);
    auto *free_ = reinterpret_cast<u32 *>(base + l.free_);
    auto *lpos = reinterpret_cast<u32 *>(base + l.lpos);
    auto *left = reinterpret_cast<perm::Key *>(base + l.left);
    void *cub_tmp = base + l.cub;
    size_t cub_bytes = l.cub_bytes;
    const u64 n = usable;
    const u32 grid = (u32)((n + 255) / 256);
    perm::to_key_kernel<<<grid, 256, 0, stream>>>(vin, n, keys_in);
    ZK_TRY(cudaGetLastError());
    ZK_TRY(cub::DeviceRadixSort::SortKeys(cub_tmp, cub_bytes, keys_in, keys_a, (int)n, perm::KeyOrder(), stream));
    perm::to_key_kernel<<<grid, 256, 0, stream>>>(vtab, n, keys_in);
    ZK_TRY(cudaGetLastError());
    cub_bytes = l.cub_bytes;
    ZK_TRY(cub::DeviceRadixSort::SortKeys(cub_tmp, cub_bytes, keys_in, keys_t, (int)n, perm::KeyOrder(), stream));
    perm::runs_kernel<<<grid, 256, 0, stream>>>(keys_a, n, first, free_);
    ZK_TRY(cudaGetLastError());
    perm::take_kernel<<<grid, 256, 0, stream>>>(keys_a, first, keys_t, n, free_);
    ZK_TRY(cudaGetLastError());
    cub_bytes = l.cub_bytes;
    ZK_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, first, fpos, (int)n, stream));
    cub_bytes = l.cub_bytes;
    ZK_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, free_, lpos, (int)n, stream));
    perm::compact_kernel<<<grid, 256, 0, stream>>>(keys_t, free_, lpos, n, left);
    ZK_TRY(cudaGetLastError());
    perm::output_kernel<<<grid, 256, 0, stream>>>(keys_a, first, fpos, left, n, vri, vrt);
    return cudaGetLastError();
}
