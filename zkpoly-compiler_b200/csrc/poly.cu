// libpoly.so: polynomial kernels over BN254 Fr for sm_100a.
//
// Replaces the reference's poly library (core/src/poly/src/poly.h:4-28, poly_basic.cuh,
// poly_eval.cuh, batched_invert.cuh, scan_mul.cuh, kate_division.cuh) behind the same C ABI.
// Temp-buffer protocol as in the reference: a null temp buffer returns the size needed.
//
// The reference builds evaluation, inversion and scans from CUB device scans with a field
// operator.  Here every reduction is a chunked tree of this library's own kernels: each thread
// folds a contiguous chunk of CHUNK elements (Horner step, running product, ...), the chunk
// results form a 1/CHUNK-size array that is folded the same way, and a second sweep pushes the
// combined values back down.  Each element costs one to three Montgomery products and one or
// two passes over HBM.
#include <cuda_runtime.h>
#include <cstring>
#include <vector>

#include "../../include/poly.h"
#include "common.cuh"
#include "curve.cuh"

namespace zk {
namespace poly {

constexpr u32 CHUNK = 64;   // elements folded by one evaluation thread on the first level
// the same for the product scans, inversion and division, whose threads run one dependent
// chain each (evaluation runs four): 32 gives them twice the chains of 64 (2^22: division
// 0.365 -> 0.324 ms, inversion 0.487 -> 0.435 ms, product scan 0.332 -> 0.294 ms; 16 is no
// faster at 2^22 and slower at 2^24)
constexpr u32 SWEEP = 32;
constexpr u32 UPPER = 8;    // on the upper levels: short chains, since those levels are tiny
constexpr u32 BLOCK = 128;

// The level sweeps (evaluation, product scans, inversion, division) fold chunks of `first`
// elements on the input and chunks of UPPER on every level above it: the first level carries
// the work, the upper levels are a few thousand values whose cost is the length of their
// dependent chains.
inline u32 chunk_at(size_t level, u32 first) { return level == 0 ? first : UPPER; }

inline u32 grid_for(u64 items, u32 block, u32 per_sm = 16) {
    const u64 b = (items + block - 1) / block;
    const u64 cap = (u64)num_sms() * per_sm;
    return (u32)(b < cap ? (b == 0 ? 1 : b) : cap);
}

inline View plain_view(void *p, u64 n) {
    View v;
    v.base = reinterpret_cast<u32 *>(p);
    v.off = 0;
    v.whole = n ? n : 1;
    v.len = n;
    return v;
}

// ------------------------------------------------------------------ elementwise
enum Op : u32 { OP_ADD = 0, OP_SUB = 1, OP_MUL = 2, OP_SUBR = 3, OP_SQR = 4 };

// dst[i] = a[i] op b[i] for i < len; dst[i] = a[i] (or -a[i] for reversed subtraction) for
// len <= i < upper (poly_basic.cuh:4-65: the longer operand passes through)
__global__ void __launch_bounds__(256) binary_kernel(View dst, View a, View b, u64 len, u64 upper, u32 op) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < upper; i += stride) {
        Fr x = Fr::load(a.at(i)), r;
        if (i < len) {
            Fr y = Fr::load(b.at(i));
            switch (op) {
                case OP_ADD: r = Fr::add_c(x, y); break;
                case OP_SUB: r = Fr::sub_c(x, y); break;
                case OP_SUBR: r = Fr::sub_c(y, x); break;
                case OP_SQR: r = Fr::sqr(x).canonical(); break;
                default: r = Fr::mul(x, y).canonical(); break;
            }
        } else {
            r = op == OP_SUBR ? Fr::neg(x).canonical() : x;
        }
        r.store(dst.at(i));
    }
}

// coef = true: value at index 0, zero elsewhere (poly_set_coef); else value everywhere
__global__ void __launch_bounds__(256) fill_kernel(View dst, u64 n, u32 kind, bool coef) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr v = (kind == 1 && (!coef || i == 0)) ? Fr::one() : Fr::zero();
        v.store(dst.at(i));
    }
}

__global__ void scalar_kernel(u32 *target, u64 exp, u32 kind) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Fr x = Fr::load(target);
    Fr r = kind == 0 ? inv_binary<FrParams>(x) : Fr::pow_u64(x, exp).canonical();
    r.store(target);
}

// ------------------------------------------------------------------ evaluation
// out[t] = sum_{i in chunk t} a_i X^(i - t*CHUNK), as EVAL_CHAINS interleaved Horner chains of
// EVAL_LEN combined with X^EVAL_LEN; powers[2*level] = X, powers[2*level+1] = X^EVAL_LEN.  Four
// chains (60 registers) measured fastest: eight (100 registers) 0.176 -> 0.190 ms at 2^22,
// sixteen 0.255 ms.
constexpr u32 EVAL_CHAINS = 4, EVAL_LEN = CHUNK / EVAL_CHAINS;
__global__ void __launch_bounds__(BLOCK) eval_level_kernel(View in, u64 n, const u32 *powers, u32 *out) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * CHUNK;
    if (start >= n) return;
    const Fr X = Fr::load(powers), XL = Fr::load(powers + 8);
    Fr h[EVAL_CHAINS];
#pragma unroll
    for (u32 k = 0; k < EVAL_CHAINS; k++) h[k] = Fr::zero();
#pragma unroll 1
    for (int j = (int)EVAL_LEN - 1; j >= 0; j--) {
#pragma unroll
        for (u32 k = 0; k < EVAL_CHAINS; k++) {
            const u64 i = start + (u64)k * EVAL_LEN + j;
            Fr a = i < n ? Fr::load(in.at(i)) : Fr::zero();
            h[k] = Fr::add(Fr::mul(h[k], X), a);
        }
    }
    Fr r = h[EVAL_CHAINS - 1];
#pragma unroll
    for (int k = (int)EVAL_CHAINS - 2; k >= 0; k--) r = Fr::add(Fr::mul(r, XL), h[k]);
    r.canonical().store(out + t * 8);
}

// powers for every level: X_0 = x, X_1 = X_0^CHUNK, X_{k+1} = X_k^UPPER, and X_k^EVAL_LEN
__global__ void eval_powers_kernel(const u32 *x, u32 levels, u32 *powers) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Fr X = Fr::load(x);
    for (u32 k = 0; k < levels; k++) {
        Fr xl = X;
        for (u32 s = 1; s < EVAL_LEN; s <<= 1) xl = Fr::sqr(xl);
        X.canonical().store(powers + (2 * k) * 8);
        xl.canonical().store(powers + (2 * k + 1) * 8);
        if (k == 0) {
            for (u32 s = EVAL_LEN; s < CHUNK; s <<= 1) xl = Fr::sqr(xl);
            X = xl;  // X^CHUNK
        } else {
            for (u32 s = 1; s < UPPER; s <<= 1) X = Fr::sqr(X);  // X^UPPER
        }
    }
}

// an upper level: out[t] = sum_{i in chunk t} a_i X^(i - t*chunk), one Horner chain
__global__ void __launch_bounds__(BLOCK) eval_small_kernel(View in, u64 n, const u32 *powers, u32 chunk, u32 *out) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * chunk;
    if (start >= n) return;
    const u64 end = start + chunk < n ? start + chunk : n;
    const Fr X = Fr::load(powers);
    Fr h = Fr::zero();
    for (u64 i = end; i-- > start;) h = Fr::add(Fr::mul(h, X), Fr::load(in.at(i)));
    h.canonical().store(out + t * 8);
}

// ------------------------------------------------------------------ chunked product sweeps
// up-sweep: prefix[i] = running product (inclusive) within the chunk, zeros skipped when
// skip_zero; tot[t] = chunk product
__global__ void __launch_bounds__(BLOCK) prod_up_kernel(View in, u64 n, u32 *prefix, u32 *tot, bool skip_zero,
                                                      u32 chunk) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * chunk;
    if (start >= n) return;
    const u64 end = start + chunk < n ? start + chunk : n;
    Fr acc = Fr::one();
    for (u64 i = start; i < end; i++) {
        Fr a = Fr::load(in.at(i));
        if (!(skip_zero && a.is_zero())) acc = Fr::mul(acc, a);
        if (prefix) acc.store(prefix + i * 8);
    }
    acc.canonical().store(tot + t * 8);
}

// batched inversion down-sweep: inv_tot[t] = (chunk product)^-1; walks the chunk backwards
__global__ void __launch_bounds__(BLOCK) inv_down_kernel(View data, u64 n, const u32 *prefix, const u32 *inv_tot,
                                                       u32 chunk) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * chunk;
    if (start >= n) return;
    const u64 end = start + chunk < n ? start + chunk : n;
    Fr inv = Fr::load(inv_tot + t * 8);
    for (u64 i = end; i-- > start;) {
        u32 *p = data.at(i);
        Fr a = Fr::load(p);
        if (a.is_zero()) continue;
        Fr before = i > start ? Fr::load(prefix + (i - 1) * 8) : Fr::one();
        Fr r = Fr::mul(inv, before);
        inv = Fr::mul(inv, a);
        r.canonical().store(p);
    }
}

// inclusive product scan down-sweep: `above` is the inclusive scan of the chunk products (or
// null for the top level), so chunk t starts from above[t-1] (1 for t = 0)
__global__ void __launch_bounds__(BLOCK) scan_down_kernel(View data, u64 n, const u32 *above, u32 chunk) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * chunk;
    if (start >= n) return;
    const u64 end = start + chunk < n ? start + chunk : n;
    Fr acc = (above && t > 0) ? Fr::load(above + (t - 1) * 8) : Fr::one();
    for (u64 i = start; i < end; i++) {
        u32 *p = data.at(i);
        acc = Fr::mul(acc, Fr::load(p));
        acc.canonical().store(p);
    }
}

// top of the inversion tree: one thread inverts the product of at most SWEEP values
__global__ void inv_top_kernel(u32 *vals, u64 m) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Fr pre[SWEEP];
    Fr acc = Fr::one();
    for (u64 i = 0; i < m; i++) {
        pre[i] = acc;
        acc = Fr::mul(acc, Fr::load(vals + i * 8));
    }
    Fr inv = inv_binary<FrParams>(acc);
    for (u64 i = m; i-- > 0;) {
        Fr a = Fr::load(vals + i * 8);
        Fr r = Fr::mul(inv, pre[i]);
        inv = Fr::mul(inv, a);
        r.canonical().store(vals + i * 8);
    }
}

// top of the scan tree: exclusive product scan of at most SWEEP values in place
__global__ void scan_top_kernel(u32 *vals, u64 m) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Fr acc = Fr::one();
    for (u64 i = 0; i < m; i++) {
        Fr a = Fr::load(vals + i * 8);
        acc.canonical().store(vals + i * 8);
        acc = Fr::mul(acc, a);
    }
}

// ------------------------------------------------------------------ kate division
// q[i] = sum_{j > i} p_j b^(j-i-1), i.e. q[i] = p[i+1] + b q[i+1] with q[n-1] = 0
// (kate_division.cuh:1-85, halo2 kate_division).  Chunk t holds the local recurrence value
// with zero carry-in; a chunk's carry is q at its first index.  Up-sweep: local value at the
// chunk start (Horner over the chunk from its top); the carries combine as another reversed
// Horner with base b^CHUNK; down-sweep walks each chunk downwards from its carry-in.
__global__ void __launch_bounds__(BLOCK) kate_up_kernel(View p, u64 n, const u32 *b, u32 *loc, u32 chunk) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * chunk;
    if (start >= n) return;
    const u64 end = start + chunk < n ? start + chunk : n;
    const Fr B = Fr::load(b);
    // value of q at `start` from the chunk's own terms: sum_{start < j < end+... }
    Fr acc = Fr::zero();
    for (u64 i = end; i-- > start;) {
        // q[i] = p[i+1] + b q[i+1]; inside the chunk q[end-1] uses p[end] and carry q[end]
        const u64 j = i + 1;
        Fr pj = j < n ? Fr::load(p.at(j)) : Fr::zero();
        acc = Fr::add(Fr::mul(acc, B), pj);
    }
    acc.canonical().store(loc + t * 8);
}

// base of the next level: B^chunk
__global__ void pow_chunk_kernel(const u32 *b, u32 chunk, u32 *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Fr::pow_u64(Fr::load(b), chunk).canonical().store(out);
}

// a short level (n <= SWEEP): one thread runs the recurrence directly
__global__ void kate_small_kernel(View p, View q, u64 n, const u32 *b) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const Fr B = Fr::load(b);
    Fr acc = Fr::zero();
    for (u64 i = n; i-- > 0;) {
        const u64 j = i + 1;
        Fr pj = j < n ? Fr::load(p.at(j)) : Fr::zero();
        acc = Fr::add(Fr::mul(acc, B), pj);
        acc.canonical().store(q.at(i));
    }
}

__global__ void __launch_bounds__(BLOCK) kate_down_kernel(View p, View q, u64 n, const u32 *b, const u32 *carry,
                                                        u32 chunk) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * chunk;
    if (start >= n) return;
    const u64 end = start + chunk < n ? start + chunk : n;
    const Fr B = Fr::load(b);
    // carry[t] = q at the first index of chunk t + 1: with loc the chunk-local values, that is
    // the next level's quotient at t (which is 0 for the last chunk)
    Fr acc = Fr::load(carry + t * 8);
    for (u64 i = end; i-- > start;) {
        const u64 j = i + 1;
        Fr pj = j < n ? Fr::load(p.at(j)) : Fr::zero();
        acc = Fr::add(Fr::mul(acc, B), pj);
        acc.canonical().store(q.at(i));
    }
}

// ------------------------------------------------------------------ temp planning
inline std::vector<u64> level_sizes(u64 n, u32 first) {
    std::vector<u64> s;
    u64 m = n;
    for (size_t k = 0; m > chunk_at(k, first); k++) {
        m = (m + chunk_at(k, first) - 1) / chunk_at(k, first);
        s.push_back(m);
    }
    return s;  // sizes of the chunk-result arrays; the last one fits in one chunk of its level
}

inline size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace poly
}  // namespace zk

using namespace zk;
using namespace zk::poly;

static cudaError_t binary_op(PolyPtr r, ConstPolyPtr a, ConstPolyPtr b, u32 op, cudaStream_t stream) {
    u64 len = a.len < b.len ? a.len : b.len;
    u64 upper = a.len < b.len ? b.len : a.len;
    if (a.len < b.len) {
        std::swap(a, b);
        if (op == OP_SUB) op = OP_SUBR;
    }
    View vr, va, vb;
    ZK_CHECK_ARG(make_view(r, &vr) && make_view(a, &va) && make_view(b, &vb));
    ZK_CHECK_ARG(r.len >= upper);
    if (upper == 0) return cudaSuccess;
    binary_kernel<<<grid_for(upper, 256), 256, 0, stream>>>(vr, va, vb, len, upper, op);
    return cudaGetLastError();
}

extern "C" cudaError_t poly_add(PolyPtr r, ConstPolyPtr a, ConstPolyPtr b, cudaStream_t stream) {
    return binary_op(r, a, b, OP_ADD, stream);
}
extern "C" cudaError_t poly_sub(PolyPtr r, ConstPolyPtr a, ConstPolyPtr b, cudaStream_t stream) {
    return binary_op(r, a, b, OP_SUB, stream);
}
extern "C" cudaError_t poly_mul(PolyPtr r, ConstPolyPtr a, ConstPolyPtr b, cudaStream_t stream) {
    return binary_op(r, a, b, OP_MUL, stream);
}
extern "C" cudaError_t zkp_poly_square(PolyPtr r, ConstPolyPtr a, cudaStream_t stream) {
    return binary_op(r, a, a, OP_SQR, stream);
}

static cudaError_t fill(PolyPtr t, u32 kind, bool coef, cudaStream_t stream) {
    View v;
    ZK_CHECK_ARG(make_view(t, &v));
    if (v.len == 0) return cudaSuccess;
    fill_kernel<<<grid_for(v.len, 256), 256, 0, stream>>>(v, v.len, kind, coef);
    return cudaGetLastError();
}
extern "C" cudaError_t poly_one_lagrange(PolyPtr target, cudaStream_t stream) { return fill(target, 1, false, stream); }
extern "C" cudaError_t poly_one_coef(PolyPtr target, cudaStream_t stream) { return fill(target, 1, true, stream); }
extern "C" cudaError_t poly_zero(PolyPtr target, cudaStream_t stream) { return fill(target, 0, true, stream); }

extern "C" cudaError_t inv_scalar(unsigned int *target, cudaStream_t stream) {
    ZK_CHECK_ARG(target != nullptr);
    scalar_kernel<<<1, 32, 0, stream>>>(target, 0, 0);
    return cudaGetLastError();
}
extern "C" cudaError_t scalar_pow(unsigned int *target, unsigned long long exp, cudaStream_t stream) {
    ZK_CHECK_ARG(target != nullptr);
    scalar_kernel<<<1, 32, 0, stream>>>(target, exp, 1);
    return cudaGetLastError();
}

// ---- poly_eval: temp = powers (2 per level) + chunk-result arrays
extern "C" cudaError_t poly_eval(void *temp_buf, unsigned long *temp_buf_size, ConstPolyPtr poly, unsigned int *res,
                                 const unsigned int *x, cudaStream_t stream) {
    const u64 n = poly.len;
    std::vector<u64> lv = level_sizes(n, CHUNK);
    const u32 levels = (u32)lv.size() + 1;
    size_t need = al((size_t)levels * 2 * 32);
    for (u64 m : lv) need += al(m * 32);
    if (temp_buf == nullptr) {
        ZK_CHECK_ARG(temp_buf_size != nullptr);
        *temp_buf_size = need;
        return cudaSuccess;
    }
    ZK_CHECK_ARG(res != nullptr && x != nullptr);
    if (temp_buf_size) ZK_CHECK_ARG(*temp_buf_size >= need);
    View v;
    ZK_CHECK_ARG(make_view(poly, &v));
    if (n == 0) return cudaMemsetAsync(res, 0, 32, stream);
    char *base = reinterpret_cast<char *>(temp_buf);
    u32 *powers = reinterpret_cast<u32 *>(base);
    eval_powers_kernel<<<1, 32, 0, stream>>>(x, levels, powers);
    size_t off = al((size_t)levels * 2 * 32);
    View in = v;
    u64 m = n;
    for (u32 k = 0; k < levels; k++) {
        u32 *out = (k + 1 < levels) ? reinterpret_cast<u32 *>(base + off) : res;
        const u32 chunk = chunk_at(k, CHUNK);
        const u64 threads = (m + chunk - 1) / chunk;
        const u32 grid = (u32)((threads + BLOCK - 1) / BLOCK);
        if (k == 0)
            eval_level_kernel<<<grid, BLOCK, 0, stream>>>(in, m, powers, out);
        else
            eval_small_kernel<<<grid, BLOCK, 0, stream>>>(in, m, powers + 2 * k * 8, chunk, out);
        ZK_TRY(cudaGetLastError());
        if (k + 1 < levels) {
            in = plain_view(out, threads);
            off += al(threads * 32);
            m = threads;
        }
    }
    return cudaSuccess;
}

// ---- batched_invert: temp = prefix arrays + chunk-product arrays per level
extern "C" cudaError_t batched_invert(void *temp_buffer, unsigned long *buffer_size, PolyPtr poly,
                                      cudaStream_t stream) {
    const u64 n = poly.len;
    std::vector<u64> lv = level_sizes(n, SWEEP);
    size_t need = al(n * 32);
    for (u64 m : lv) need += 2 * al(m * 32);
    need += al(SWEEP * 32);
    if (temp_buffer == nullptr) {
        ZK_CHECK_ARG(buffer_size != nullptr);
        *buffer_size = need;
        return cudaSuccess;
    }
    View v;
    ZK_CHECK_ARG(make_view(poly, &v));
    if (n == 0) return cudaSuccess;
    char *base = reinterpret_cast<char *>(temp_buffer);
    // level k data: level 0 = poly; level k>0 = tot array of level k-1
    std::vector<View> data;
    std::vector<u32 *> prefix;
    std::vector<u64> size;
    data.push_back(v);
    size.push_back(n);
    size_t off = 0;
    prefix.push_back(reinterpret_cast<u32 *>(base + off));
    off += al(n * 32);
    for (u64 m : lv) {
        data.push_back(plain_view(base + off, m));
        off += al(m * 32);
        prefix.push_back(reinterpret_cast<u32 *>(base + off));
        off += al(m * 32);
        size.push_back(m);
    }
    // the top array: product of the last level's chunks (one value)
    u32 *top = reinterpret_cast<u32 *>(base + off);
    const size_t L = data.size();
    for (size_t k = 0; k < L; k++) {
        const u64 m = size[k];
        const u64 threads = (m + chunk_at(k, SWEEP) - 1) / chunk_at(k, SWEEP);
        u32 *tot = (k + 1 < L) ? data[k + 1].base : top;
        prod_up_kernel<<<(u32)((threads + BLOCK - 1) / BLOCK), BLOCK, 0, stream>>>(data[k], m, prefix[k], tot, k == 0,
                                                                                  chunk_at(k, SWEEP));
        ZK_TRY(cudaGetLastError());
    }
    inv_top_kernel<<<1, 32, 0, stream>>>(top, 1);
    ZK_TRY(cudaGetLastError());
    for (size_t k = L; k-- > 0;) {
        const u64 m = size[k];
        const u64 threads = (m + chunk_at(k, SWEEP) - 1) / chunk_at(k, SWEEP);
        const u32 *inv_tot = (k + 1 < L) ? data[k + 1].base : top;
        inv_down_kernel<<<(u32)((threads + BLOCK - 1) / BLOCK), BLOCK, 0, stream>>>(data[k], m, prefix[k], inv_tot,
                                                                                   chunk_at(k, SWEEP));
        ZK_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

// ---- scan_mul: inclusive product scan in place; temp = chunk-product arrays
extern "C" cudaError_t scan_mul(void *temp_buffer, unsigned long *buffer_size, PolyPtr target, cudaStream_t stream) {
    const u64 n = target.len;
    std::vector<u64> lv = level_sizes(n, SWEEP);
    size_t need = al(32);
    for (u64 m : lv) need += al(m * 32);
    if (temp_buffer == nullptr) {
        ZK_CHECK_ARG(buffer_size != nullptr);
        *buffer_size = need;
        return cudaSuccess;
    }
    View v;
    ZK_CHECK_ARG(make_view(target, &v));
    if (n == 0) return cudaSuccess;
    char *base = reinterpret_cast<char *>(temp_buffer);
    std::vector<View> data{v};
    std::vector<u64> size{n};
    size_t off = 0;
    for (u64 m : lv) {
        data.push_back(plain_view(base + off, m));
        off += al(m * 32);
        size.push_back(m);
    }
    const size_t L = data.size();
    for (size_t k = 0; k + 1 < L; k++) {
        const u64 threads = (size[k] + chunk_at(k, SWEEP) - 1) / chunk_at(k, SWEEP);
        prod_up_kernel<<<(u32)((threads + BLOCK - 1) / BLOCK), BLOCK, 0, stream>>>(data[k], size[k], nullptr,
                                                                                  data[k + 1].base, false,
                                                                                  chunk_at(k, SWEEP));
        ZK_TRY(cudaGetLastError());
    }
    for (size_t k = L; k-- > 0;) {
        const u64 threads = (size[k] + chunk_at(k, SWEEP) - 1) / chunk_at(k, SWEEP);
        const u32 *above = (k + 1 < L) ? data[k + 1].base : nullptr;
        scan_down_kernel<<<(u32)((threads + BLOCK - 1) / BLOCK), BLOCK, 0, stream>>>(data[k], size[k], above,
                                                                                    chunk_at(k, SWEEP));
        ZK_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

// ---- kate_division: q = (p - p(b)) / (X - b), length 2^log_p.
// Chunk carries are themselves a kate division (of the chunk-local values by b^CHUNK), so the
// levels recurse: level k+1 holds the chunk-local values of level k, and its quotient gives
// the carries of level k.
extern "C" cudaError_t kate_division(void *temp_buf, unsigned long *temp_buf_size, unsigned int log_p, ConstPolyPtr p,
                                     const unsigned int *b, PolyPtr q, cudaStream_t stream) {
    const u64 n = 1ull << log_p;
    std::vector<u64> lv = level_sizes(n, SWEEP);
    size_t need = al((lv.size() + 1) * 32);
    for (u64 m : lv) need += 2 * al(m * 32);
    if (temp_buf == nullptr) {
        ZK_CHECK_ARG(temp_buf_size != nullptr);
        *temp_buf_size = need;
        return cudaSuccess;
    }
    ZK_CHECK_ARG(p.len == n && q.len == n && b != nullptr);
    View vp, vq;
    ZK_CHECK_ARG(make_view(p, &vp) && make_view(q, &vq));
    char *base = reinterpret_cast<char *>(temp_buf);
    const size_t L = lv.size() + 1;
    std::vector<View> P{vp}, Q{vq};
    std::vector<const u32 *> Bs{b};
    std::vector<u64> size{n};
    u32 *bases = reinterpret_cast<u32 *>(base);
    size_t off = al(L * 32);
    for (size_t k = 0; k < lv.size(); k++) {
        P.push_back(plain_view(base + off, lv[k]));
        off += al(lv[k] * 32);
        Q.push_back(plain_view(base + off, lv[k]));
        off += al(lv[k] * 32);
        size.push_back(lv[k]);
        pow_chunk_kernel<<<1, 32, 0, stream>>>(Bs.back(), chunk_at(k, SWEEP), bases + k * 8);
        Bs.push_back(bases + k * 8);
    }
    // up-sweeps: P[k+1][t] = chunk-local value of level k at chunk t's start
    for (size_t k = 0; k + 1 < L; k++) {
        const u64 chunks = (size[k] + chunk_at(k, SWEEP) - 1) / chunk_at(k, SWEEP);
        kate_up_kernel<<<(u32)((chunks + BLOCK - 1) / BLOCK), BLOCK, 0, stream>>>(P[k], size[k], Bs[k],
                                                                                 P[k + 1].base, chunk_at(k, SWEEP));
        ZK_TRY(cudaGetLastError());
    }
    kate_small_kernel<<<1, 32, 0, stream>>>(P[L - 1], Q[L - 1], size[L - 1], Bs[L - 1]);
    ZK_TRY(cudaGetLastError());
    for (size_t k = L - 1; k-- > 0;) {
        const u64 chunks = (size[k] + chunk_at(k, SWEEP) - 1) / chunk_at(k, SWEEP);
        kate_down_kernel<<<(u32)((chunks + BLOCK - 1) / BLOCK), BLOCK, 0, stream>>>(P[k], Q[k], size[k], Bs[k],
                                                                                   Q[k + 1].base, chunk_at(k, SWEEP));
        ZK_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}
#include "permute.cuh"
