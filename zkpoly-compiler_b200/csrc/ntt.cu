// libntt.so: in-place natural-order NTT over BN254 Fr for sm_100a.
//
// Replaces the reference's SSIP kernels (core/src/ntt/src/ssip_ntt.cuh:10-566,
// recompute_ntt.cuh:23-438) behind the same C ABI (core/src/ntt/src/ntt.h:5-16).
//
// Algorithm (n = 2^L).  The index bits are split into digits of at most 12 bits, top digit
// first.  Pass p takes every "pencil" of 2^D elements that differ only in digit p (bits
// [lo, lo + D)), runs a radix-2 DIF sub-transform on it in shared memory (its output lands
// bit-reversed inside the digit), and, when lower digits remain, multiplies element k of the
// sub-transform by the four-step twist w_N^(c*k), where c is the pencil's value of the lower
// digits and N = 2^(lo + D).  After the last digit the whole vector is in bit-reversed order;
// a final in-place permutation pass swaps i <-> rev(i).  For L <= 12 one CTA does the whole
// transform and writes natural order directly.
//
// Every pass reads and writes the same pencil, so all passes run in place on the caller's
// buffer with no scratch memory.  Intermediate values stay in [0, 2m) (lazy Montgomery);
// the last transform pass stores canonical values.
//
// Shared memory holds the pencil as 8 word planes (element e, word w at w*S + swz(e)) and the
// 2^(D-1) sub-transform roots the same way; both swizzles keep a warp's 32 accesses on 32
// different banks for every butterfly span.
#include <cuda_runtime.h>
#include <atomic>
#include <cstring>
#include <vector>

#include "../../include/ntt.h"
#include "common.cuh"
#include "host_field.h"

namespace zk {
namespace ntt {

constexpr u32 MAX_D = 12;
constexpr u32 MAX_THREADS = 1024;

enum Flags : u32 {
    F_TWIST = 1u,          // multiply by the four-step twist after the sub-transform
    F_NATURAL = 2u,        // single-pass plan: store in natural order
    F_CANON = 4u,          // store canonical values (last transform pass)
    F_PRESHIFT = 8u,       // multiply x[i] by shift^i on load (pass 0 only)
    F_POSTSCALE = 16u,     // multiply by *scale on the final store
    F_RECOMPUTE = 32u,     // derive roots from omegas[] instead of a table
    F_SRC = 64u,           // pass 0 reads from src (zero beyond src_len), writes to v
};

struct PassArgs {
    View v;                 // data (in place)
    View src;               // optional source of pass 0 (coset LDE)
    const u32 *tw;          // [w^0 .. w^(n/2-1)] (table mode)
    const u32 *omegas;      // [w^(2^i)] (recompute mode)
    const u32 *shift;       // coset shift (Montgomery) or null
    const u32 *scale;       // post-scale or null
    const u32 *shoup;       // register passes: Shoup twiddle table (16 words per root) or null
    u32 L, D, lo, flags;
    u64 src_len;
};

ZK_DI u32 swz(u32 e) { return e ^ (((e >> 5) & 1u) * 31u); }
ZK_DI u32 swt(u32 x) { return x ^ (((x >> 5) ^ (x >> 10)) & 31u); }

ZK_DI Fr sm_load(const u32 *base, u32 stride, u32 pos) {
    Fr r;
#pragma unroll
    for (int w = 0; w < 8; w++) r.v[w] = base[w * stride + pos];
    return r;
}
ZK_DI void sm_store(u32 *base, u32 stride, u32 pos, const Fr &x) {
#pragma unroll
    for (int w = 0; w < 8; w++) base[w * stride + pos] = x.v[w];
}

// w^e for a 64-bit exponent from the n/2 root table (w^(n/2) = -1)
ZK_DI Fr table_root(const u32 *tw, u64 e, u32 L) {
    const u64 half = 1ull << (L - 1);
    if (e < half) return Fr::load_nc(tw + e * 8);
    Fr w = Fr::load_nc(tw + (e - half) * 8);
    return Fr::neg(w);
}

// w^e from omegas[i] = w^(2^i) (recompute mode): one multiply per set bit
ZK_DI Fr omega_pow(const u32 *omegas, u64 e) {
    Fr r = Fr::one();
    int i = 0;
    while (e) {
        if (e & 1) r = Fr::mul(r, Fr::load_nc(omegas + i * 8));
        e >>= 1;
        i++;
    }
    return r;
}

__device__ __forceinline__ void pass_body(const PassArgs &a, const u64 P, u32 *sm) {
    const u32 D = a.D;
    const u32 S = 1u << D;
    const u32 H = S >> 1;
    u32 *data = sm;
    u32 *tws = sm + 8 * S;
    u32 *aux = tws + 8 * (H > 0 ? H : 1);  // 2 x 64 elements of shift tables (recompute twist)
    const u32 T = blockDim.x;
    const u32 tid = threadIdx.x;
    const u64 cmask = (1ull << a.lo) - 1;
    const u64 c = P & cmask;
    const u64 h = P >> a.lo;
    const u64 gbase = (h << (a.lo + D)) | c;
    const bool recompute = (a.flags & F_RECOMPUTE) != 0;

    // ---- sub-transform roots w_{2^D}^i, i < H
    if (!recompute) {
        for (u32 i = tid; i < H; i += T) {
            Fr w = Fr::load_nc(a.tw + ((u64)i << (a.L - D)) * 8);
            sm_store(tws, H, swt(i), w);
        }
    } else if (H > 0) {
        // two-level: w^i = w^(i & 63) * w^(64 * (i >> 6)); the 64 + H/64 seeds by pow
        const u32 lo_n = H < 64 ? H : 64;
        const u32 hi_n = H > 64 ? H / 64 : 1;
        for (u32 i = tid; i < lo_n + hi_n; i += T) {
            u64 e = i < lo_n ? (u64)i : (u64)(i - lo_n) * 64;
            Fr w = omega_pow(a.omegas, e << (a.L - D));
            sm_store(aux, 128, i, w);
        }
        __syncthreads();
        for (u32 i = tid; i < H; i += T) {
            Fr w = sm_load(aux, 128, i & 63);
            if (i >= 64) w = Fr::mul(w, sm_load(aux, 128, lo_n + (i >> 6)));
            sm_store(tws, H, swt(i), w);
        }
        __syncthreads();
    }

    // ---- coset shift tables (pass 0): shift^(c + r*2^lo) = (shift^c * G^(r&63)) * G^(64*(r>>6))
    const bool preshift = (a.flags & F_PRESHIFT) != 0;
    if (preshift) {
        for (u32 i = tid; i < 128; i += T) {
            Fr g = Fr::load_nc(a.shift);
            Fr G = g;
            for (u32 k = 0; k < a.lo; k++) G = Fr::mul(G, G);
            Fr w;
            if (i < 64) {
                w = Fr::mul(Fr::pow_u64(g, c), Fr::pow_u64(G, i));
            } else {
                w = Fr::pow_u64(G, (u64)(i - 64) * 64);
            }
            sm_store(aux, 128, i, w);
        }
        __syncthreads();
    }

    // ---- load the pencil
    const bool from_src = (a.flags & F_SRC) != 0;
    for (u32 r = tid; r < S; r += T) {
        const u64 gi = gbase + ((u64)r << a.lo);
        Fr x;
        if (from_src) {
            x = gi < a.src_len ? Fr::load(a.src.at(gi)) : Fr::zero();
        } else {
            x = Fr::load(a.v.at(gi));
        }
        if (preshift) {
            x = Fr::mul(x, sm_load(aux, 128, r & 63));
            if (r >= 64) x = Fr::mul(x, sm_load(aux, 128, 64 + (r >> 6)));
        }
        sm_store(data, S, swz(r), x);
    }
    __syncthreads();

    // ---- radix-2 DIF stages, span 2^b
    for (int b = (int)D - 1; b >= 0; b--) {
        const u32 hh = 1u << b;
        for (u32 j = tid; j < H; j += T) {
            const u32 e0 = ((j >> b) << (b + 1)) | (j & (hh - 1));
            const u32 e1 = e0 + hh;
            const u32 p0 = swz(e0), p1 = swz(e1);
            Fr x0 = sm_load(data, S, p0);
            Fr x1 = sm_load(data, S, p1);
            Fr s = Fr::add(x0, x1);
            Fr d = Fr::sub(x0, x1);
            if (b > 0) {
                const u32 ti = (j & (hh - 1)) << (D - 1 - b);
                d = Fr::mul(d, sm_load(tws, H, swt(ti)));
            }
            sm_store(data, S, p0, s);
            sm_store(data, S, p1, d);
        }
        __syncthreads();
    }

    // ---- twist (recompute mode: per-CTA tables of (w_N^c)^k)
    const bool twist = (a.flags & F_TWIST) != 0;
    if (twist && recompute) {
        // base = w_N^c with w_N = w^(2^(L-lo-D)); tables base^(k & 63), base^(64 * (k >> 6))
        for (u32 i = tid; i < 128; i += T) {
            Fr base = omega_pow(a.omegas, c << (a.L - a.lo - D));
            Fr w = i < 64 ? Fr::pow_u64(base, i) : Fr::pow_u64(base, (u64)(i - 64) * 64);
            sm_store(aux, 128, i, w);
        }
        __syncthreads();
    }

    const bool natural = (a.flags & F_NATURAL) != 0;
    const bool canon = (a.flags & F_CANON) != 0;
    const bool postscale = (a.flags & F_POSTSCALE) != 0;
    Fr scale;
    if (postscale) scale = Fr::load_nc(a.scale);
    for (u32 q = tid; q < S; q += T) {
        // natural: thread writes global position q, which holds smem position rev(q)
        const u32 s = natural ? (__brev(q) >> (32 - D)) : q;
        Fr x = sm_load(data, S, swz(s));
        if (twist) {
            const u32 k = __brev(s) >> (32 - D);  // natural output index of position s
            if (c != 0 && k != 0) {
                Fr w;
                if (recompute) {
                    w = sm_load(aux, 128, k & 63);
                    if (k >= 64) w = Fr::mul(w, sm_load(aux, 128, 64 + (k >> 6)));
                } else {
                    const u64 e = ((u64)c * k) << (a.L - a.lo - D);
                    w = table_root(a.tw, e, a.L);
                }
                x = Fr::mul(x, w);
            }
        }
        if (postscale) x = Fr::mul(x, scale);
        if (canon) x = x.canonical();
        const u64 gi = gbase + ((u64)q << a.lo);
        x.store(a.v.at(gi));
    }
}

__global__ void __launch_bounds__(MAX_THREADS, 1) ntt_pass_kernel(PassArgs a) {
    extern __shared__ u32 sm[];
    pass_body(a, (u64)blockIdx.y * gridDim.x + blockIdx.x, sm);
}

// Batched form: one persistent launch runs the same pass of many transforms.  Work item w is
// pencil w - first[t] of task t, where first[] is the exclusive prefix of the tasks' pencil
// counts (first[ntasks] = total); each CTA walks items w = blockIdx.x, + gridDim.x, ...
__global__ void __launch_bounds__(MAX_THREADS, 1) ntt_batch_pass_kernel(const PassArgs *args, const u64 *first,
                                                                       u32 ntasks) {
    extern __shared__ u32 sm[];
    const u64 total = first[ntasks];
    for (u64 w = blockIdx.x; w < total; w += gridDim.x) {
        u32 lo = 0, hi = ntasks;  // largest t with first[t] <= w
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) / 2;
            if (first[mid] <= w) lo = mid; else hi = mid;
        }
        pass_body(args[lo], w - first[lo], sm);
        __syncthreads();  // the next item reuses shared memory
    }
}

// ------------------------------------------------------------------ register pass (D <= 6)
// The same pass as pass_body written as the global radix-2 DIF stages it equals (the four-step
// twist of pass_body is folded into the stage twiddles): stage s pairs i and i + 2^s and
// multiplies the difference by w^((i mod 2^s) * 2^(L-1-s)), read from the caller's root
// table.  A pencil of 2^D elements lives in the registers of g = 2^(D-1) lanes, two elements
// per lane: lane l starts with local indices l and l + g, so the first stage is a butterfly
// inside the lane.  Before each later stage (local bit k) the lane bit k and the register bit
// trade places through one shuffle of one element per lane, bringing the stage's partners
// into the same lane; after the last stage lane l holds local indices 2l and 2l + 1.  A lane
// group works on P pencils (1 or 2); with two, they differ only in their top index bits where
// there are any, so both use the same twiddle and a twiddle load feeds two products.  No
// shared memory and no block barrier; every element is one 32-byte sector in and out.
// SH: the twiddle product is Shoup's (Fr::mul_shoup) from a table of (w^e plain,
// floor(w^e 2^256 / m)) pairs, 64 bytes per root, built by shoup_table_kernel from the
// Montgomery table; the results are the same values.
constexpr u32 WARP_MAX_D = 6;

ZK_DI void lane_swap(Fr &a, Fr &b, u32 lane, u32 k) {
    const bool hi = (lane >> k) & 1u;
    Fr send = hi ? a : b;
#pragma unroll
    for (int w = 0; w < 8; w++) send.v[w] = __shfl_xor_sync(0xffffffffu, send.v[w], 1u << k);
    if (hi) a = send; else b = send;
}

template <u32 D, u32 P, bool SH>
__global__ void __launch_bounds__(256) ntt_warp_pass_kernel(PassArgs a) {
    constexpr u32 g = 1u << (D - 1);  // lanes per pencil group
    const u32 lo = a.lo, L = a.L;
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 grp = t >> (D - 1);
    const u32 l = (u32)t & (g - 1);
    const u32 lane = threadIdx.x & 31;
    // P pencils per lane group: q = grp + j * 2^(L-D-1) (they differ in the top index bit)
    const u64 half = 1ull << (L - D - 1);
    const u64 cmask = (1ull << lo) - 1;
    u64 base[P], c[P];
#pragma unroll
    for (u32 j = 0; j < P; j++) {
        const u64 q = grp + (j ? half : 0);
        c[j] = q & cmask;
        base[j] = ((q >> lo) << (lo + D)) | c[j];
    }
    const bool shared_tw = P == 1 || c[0] == c[P - 1];
    Fr x0[P], x1[P];
#pragma unroll
    for (u32 j = 0; j < P; j++) {
        x0[j] = Fr::load(a.v.at(base[j] + ((u64)l << lo)));
        x1[j] = Fr::load(a.v.at(base[j] + ((u64)(l + g) << lo)));
    }
#pragma unroll
    for (int k = (int)D - 1; k >= 0; k--) {
        if (k < (int)D - 1) {
#pragma unroll
            for (u32 j = 0; j < P; j++) lane_swap(x0[j], x1[j], lane, (u32)k);
        }
        const u64 low = (u64)(l & ((1u << k) - 1)) << lo;
        const u32 sh = L - 1 - lo - (u32)k;
        Fr w, ws;
#pragma unroll
        for (u32 j = 0; j < P; j++) {
            const u64 e = (low | c[j]) << sh;
            Fr s = Fr::add(x0[j], x1[j]);
            Fr d = Fr::sub(x0[j], x1[j]);
            if (e != 0) {
                if (SH) {
                    if (j == 0 || !shared_tw) {
                        w = Fr::load_nc(a.shoup + e * 16);
                        ws = Fr::load_nc(a.shoup + e * 16 + 8);
                    }
                    d = Fr::mul_shoup(d, w, ws);
                } else {
                    if (j == 0 || !shared_tw) w = Fr::load_nc(a.tw + e * 8);
                    d = Fr::mul(d, w);
                }
            }
            x0[j] = s;
            x1[j] = d;
        }
    }
    const bool canon = (a.flags & F_CANON) != 0;
    const bool postscale = (a.flags & F_POSTSCALE) != 0;
    Fr scale;
    if (postscale) scale = Fr::load_nc(a.scale);
#pragma unroll
    for (u32 j = 0; j < P; j++) {
        Fr y0 = x0[j], y1 = x1[j];
        if (postscale) {
            y0 = Fr::mul(y0, scale);
            y1 = Fr::mul(y1, scale);
        }
        if (canon) {
            y0 = y0.canonical();
            y1 = y1.canonical();
        }
        y0.store(a.v.at(base[j] + ((u64)(2 * l) << lo)));
        y1.store(a.v.at(base[j] + ((u64)(2 * l + 1) << lo)));
    }
}

#ifndef ZK_NTT_WARP_PENCILS
#define ZK_NTT_WARP_PENCILS 1  // pencils per lane group in the register pass (1 or 2)
#endif

// CTA size of the register passes per transform size, set by the tuner through
// zkp_ntt_set_block (0 = 128)
std::atomic<u32> g_warp_block[29];

template <u32 P, bool SH>
cudaError_t launch_warp_pass(const PassArgs &a, cudaStream_t stream) {
    // two elements of P pencils per thread; CTAs of 128 threads by default: at 52 registers
    // (the Shoup variant) 9 of them fit an SM, 36 warps, against 4 CTAs of 256 (32 warps), 5 %
    // faster.  The kernel keeps __launch_bounds__(256): with a bound of 128 the compiler takes
    // 58 registers and the occupancy gain is gone.
    const u64 threads = 1ull << (a.L - 1 - (P == 2 ? 1 : 0));
    const u32 tuned = a.L < 29 ? g_warp_block[a.L].load(std::memory_order_relaxed) : 0;
    const u32 want = tuned ? tuned : 128;
    const u32 block = (u32)(threads < want ? threads : want);
    const u32 grid = (u32)(threads / block);
    switch (a.D) {
        case 1: ntt_warp_pass_kernel<1, P, SH><<<grid, block, 0, stream>>>(a); break;
        case 2: ntt_warp_pass_kernel<2, P, SH><<<grid, block, 0, stream>>>(a); break;
        case 3: ntt_warp_pass_kernel<3, P, SH><<<grid, block, 0, stream>>>(a); break;
        case 4: ntt_warp_pass_kernel<4, P, SH><<<grid, block, 0, stream>>>(a); break;
        case 5: ntt_warp_pass_kernel<5, P, SH><<<grid, block, 0, stream>>>(a); break;
        default: ntt_warp_pass_kernel<6, P, SH><<<grid, block, 0, stream>>>(a); break;
    }
    return cudaGetLastError();
}

// Shoup table entry e = (w^e plain, floor(w^e 2^256 / m)) from the Montgomery table entry e
__global__ void __launch_bounds__(256) shoup_table_kernel(const u32 *tw, u64 count, u32 *out) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += stride) {
        Fr w, ws;
        Fr::mul_shoup_table_entry(Fr::load_nc(tw + e * 8), &w, &ws);
        w.store(out + e * 16);
        ws.store(out + e * 16 + 8);
    }
}

// batched in-place bit reversal: element w of the concatenation belongs to task t
__global__ void __launch_bounds__(256) bitrev_batch_kernel(const View *views, const u32 *logs, const u64 *first,
                                                          u32 ntasks) {
    const u64 total = first[ntasks];
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += stride) {
        u32 lo = 0, hi = ntasks;
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) / 2;
            if (first[mid] <= w) lo = mid; else hi = mid;
        }
        const u64 i = w - first[lo];
        const u32 L = logs[lo];
        const u64 j = __brevll(i) >> (64 - L);
        if (i < j) {
            const View &v = views[lo];
            u32 *pi = v.at(i), *pj = v.at(j);
            Fr x = Fr::load(pi), y = Fr::load(pj);
            y.store(pi);
            x.store(pj);
        }
    }
}

// in-place bit-reversal permutation of L index bits
__global__ void __launch_bounds__(256) bitrev_kernel(View v, u32 L, u64 n) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 j = __brevll(i) >> (64 - L);
        if (i < j) {
            u32 *pi = v.at(i), *pj = v.at(j);
            Fr a = Fr::load(pi), b = Fr::load(pj);
            b.store(pi);
            a.store(pj);
        }
    }
}

// Tiled in-place bit reversal for L >= 2 * BR_T.  An index is (a, m, b): a the top BR_T bits,
// b the low BR_T bits, m the L - 2 BR_T middle bits, and rev(a, m, b) = (rev b, rev m, rev a).
// CTA m (m <= rev m) owns tiles m and rev m (every (a, b) of that middle value), reads both
// into shared memory row by row (a row is 2^BR_T consecutive elements) and writes element (a, b)
// of one tile to (rev b, rev a) of the other, again row by row, so every global access is a
// run of 1 KB.  Shared memory holds 8 word planes per tile; element (a, b) sits at
// a * 32 + (b ^ a), which keeps both the row writes and the column reads on 32 banks.
constexpr u32 BR_T = 5;
constexpr u32 BR_TILE = 1u << (2 * BR_T);  // elements per tile

__global__ void __launch_bounds__(256) bitrev_tiled_kernel(View v, u32 L) {
    extern __shared__ u32 br_sm[];  // 2 tiles x 8 planes x BR_TILE words
    const u32 M = L - 2 * BR_T;
    const u32 m = blockIdx.x;
    const u32 mr = M ? (__brev(m) >> (32 - M)) : 0u;
    if (mr < m) return;  // the pair is handled by CTA mr
    const u32 ntile = mr == m ? 1 : 2;
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const u32 mid[2] = {m, mr};
    for (u32 t = 0; t < ntile; t++) {
        u32 *tile = br_sm + t * 8 * BR_TILE;
        for (u32 a = warp; a < 32; a += nwarp) {
            const u64 i = ((u64)a << (L - BR_T)) | ((u64)mid[t] << BR_T) | lane;
            Fr x = Fr::load(v.at(i));
            const u32 pos = a * 32 + (lane ^ a);
#pragma unroll
            for (int w = 0; w < 8; w++) tile[w * BR_TILE + pos] = x.v[w];
        }
    }
    __syncthreads();
    for (u32 t = 0; t < ntile; t++) {
        // destination tile mid[t] receives the other tile (itself when the pair is one tile)
        const u32 *src = br_sm + (ntile == 2 ? 1 - t : 0) * 8 * BR_TILE;
        for (u32 ao = warp; ao < 32; ao += nwarp) {
            // element (ao, lane) of the destination = element (rev lane, rev ao) of the source
            const u32 a = __brev(lane) >> 27, b = __brev(ao) >> 27;
            const u32 pos = a * 32 + (b ^ a);
            Fr x;
#pragma unroll
            for (int w = 0; w < 8; w++) x.v[w] = src[w * BR_TILE + pos];
            const u64 i = ((u64)ao << (L - BR_T)) | ((u64)mid[t] << BR_T) | lane;
            x.store(v.at(i));
        }
    }
}

constexpr size_t BR_SMEM = 2 * 8 * BR_TILE * sizeof(u32);  // 64 KiB

// The last register pass fused with the tiled bit reversal (L >= 2 BR_T, last digit D <= BR_T,
// table mode).  The last pass's pencils (2^D consecutive elements, lo = 0) lie inside the rows
// of 2^BR_T elements the tiled permutation moves, so CTA m (m <= rev m) loads the rows of tiles
// m and rev m, runs the last pass's radix-2 stages on each row in registers (16 lanes a row,
// two elements a lane, the register pass's lane swaps and twiddles), stores the canonical
// results into shared memory and writes them back permuted as bitrev_tiled_kernel does.  The
// vector is read and written once for both steps instead of twice.
template <u32 D, bool SH>
__global__ void __launch_bounds__(512) ntt_last_bitrev_kernel(PassArgs a) {
    extern __shared__ u32 br_sm[];  // 2 tiles x 8 planes x BR_TILE words
    const u32 L = a.L;
    const u32 M = L - 2 * BR_T;
    const u32 m = blockIdx.x;
    const u32 mr = M ? (__brev(m) >> (32 - M)) : 0u;
    if (mr < m) return;  // the pair is handled by CTA mr
    const u32 ntile = mr == m ? 1 : 2;
    constexpr u32 g = 1u << (D - 1);             // lanes per pencil
    const u32 lane = threadIdx.x & 31;
    const u32 u = threadIdx.x & 15;              // lane within the row
    const u32 j = u >> (D - 1), l = u & (g - 1);  // pencil within the row, lane within the pencil
    const bool postscale = (a.flags & F_POSTSCALE) != 0;
    Fr scale;
    if (postscale) scale = Fr::load_nc(a.scale);
    for (u32 r = threadIdx.x >> 4; r < 32 * ntile; r += blockDim.x >> 4) {
        const u32 t = r >> BR_T, ar = r & 31;    // tile, top bits of the row
        const u64 base = ((u64)ar << (L - BR_T)) | ((u64)(t ? mr : m) << BR_T) | ((u64)j << D);
        Fr x0 = Fr::load(a.v.at(base + l));
        Fr x1 = Fr::load(a.v.at(base + l + g));
#pragma unroll
        for (int k = (int)D - 1; k >= 0; k--) {
            if (k < (int)D - 1) lane_swap(x0, x1, lane, (u32)k);
            const u64 e = (u64)(l & ((1u << k) - 1)) << (L - 1 - (u32)k);
            Fr s = Fr::add(x0, x1);
            Fr d = Fr::sub(x0, x1);
            if (e != 0) {
                if (SH) d = Fr::mul_shoup(d, Fr::load_nc(a.shoup + e * 16), Fr::load_nc(a.shoup + e * 16 + 8));
                else d = Fr::mul(d, Fr::load_nc(a.tw + e * 8));
            }
            x0 = s;
            x1 = d;
        }
        if (postscale) {
            x0 = Fr::mul(x0, scale);
            x1 = Fr::mul(x1, scale);
        }
        x0 = x0.canonical();
        x1 = x1.canonical();
        // local outputs 2l and 2l + 1 of pencil j are row elements b0 and b0 + 1
        u32 *tile = br_sm + t * 8 * BR_TILE;
        const u32 b0 = (j << D) + 2 * l;
        const u32 p0 = ar * 32 + (b0 ^ ar), p1 = ar * 32 + ((b0 + 1) ^ ar);
#pragma unroll
        for (int w = 0; w < 8; w++) {
            tile[w * BR_TILE + p0] = x0.v[w];
            tile[w * BR_TILE + p1] = x1.v[w];
        }
    }
    __syncthreads();
    const u32 warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (u32 t = 0; t < ntile; t++) {
        const u32 *src = br_sm + (ntile == 2 ? 1 - t : 0) * 8 * BR_TILE;
        for (u32 ao = warp; ao < 32; ao += nwarp) {
            const u32 ra = __brev(lane) >> 27, rb = __brev(ao) >> 27;
            const u32 pos = ra * 32 + (rb ^ ra);
            Fr x;
#pragma unroll
            for (int w = 0; w < 8; w++) x.v[w] = src[w * BR_TILE + pos];
            const u64 i = ((u64)ao << (L - BR_T)) | ((u64)(t ? mr : m) << BR_T) | lane;
            x.store(a.v.at(i));
        }
    }
}

// Coset preparation for large table-mode transforms: v[i] = x[i] * shift^i, with x the source view (zero
// beyond src_len: the zero-extension of a coset LDE) or v itself, so that the transform then
// runs the tuned register passes; folding the shift into a shared-memory first pass (which must
// build per-pencil shift tables) made a 2^22 -> 2^24 coset LDE 5.9 ms against 3.4 ms for the
// plain transform.  Warp w owns elements [w * 32 C, (w + 1) * 32 C) and lane l the elements
// base + l + 32 k: it raises the shift to base + l once (square-and-multiply) and then steps by
// shift^32, so a carried element costs two products and every access is coalesced.
constexpr u32 PREP_C = 64;
// From this size the separate pass wins (2^20 -> 2^22: 0.98 against 1.40 ms; 2^22 -> 2^24: 3.80
// against 5.89 ms); below it the shifted wide first pass is faster (2^14 -> 2^16: 0.16 against
// 0.18 ms)
constexpr u32 PREP_MIN_L = 20;
__global__ void __launch_bounds__(256) coset_prep_kernel(View v, View src, u64 src_len, bool has_src,
                                                         const u32 *shift, u64 n) {
    const u64 warp = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 lane = threadIdx.x & 31;
    const u64 base = warp * 32 * PREP_C;
    if (base >= n) return;
    const u64 live = has_src ? (src_len < n ? src_len : n) : n;  // elements that carry a value
    Fr s, step;
    if (shift && base < live) {
        const Fr g = Fr::load(shift);
        s = Fr::pow_u64(g, base + lane);
        step = Fr::pow_u64(g, 32);
    }
    for (u32 k = 0; k < PREP_C; k++) {
        const u64 i = base + lane + 32ull * k;
        if (i >= n) break;
        Fr x = Fr::zero();
        if (i < live) {
            x = Fr::load(has_src ? src.at(i) : v.at(i));
            if (shift) {
                x = Fr::mul(x, s);
                s = Fr::mul(s, step);
            }
            x = x.canonical();
        }
        x.store(v.at(i));
    }
}

__global__ void __launch_bounds__(256) distribute_powers_kernel(View v, const u32 *powers, u64 pn, u64 n) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 k = pn >= n ? i : ((pn & (pn - 1)) == 0 ? (i & (pn - 1)) : i % pn);
        u32 *p = v.at(i);
        Fr x = Fr::mul(Fr::load(p), Fr::load_nc(powers + k * 8)).canonical();
        x.store(p);
    }
}

// table[i] = w^i for i < len; each thread seeds w^(64 t) and walks 64 steps
__global__ void __launch_bounds__(256) powers_kernel(u32 *out, const u32 *unit, u64 len) {
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * 64;
    if (start >= len) return;
    Fr w = Fr::load(unit);
    Fr x = Fr::pow_u64(w, start);
    const u64 end = start + 64 < len ? start + 64 : len;
    for (u64 i = start; i < end; i++) {
        x.canonical().store(out + i * 8);
        x = Fr::mul(x, w);
    }
}

// ------------------------------------------------------------------ host plan
struct Plan {
    u32 np;
    u32 D[8];  // up to ceil(28 / 4) passes
    u32 lo[8];
};

// Per-size cap on the digit width (the sub-transform size 2^D of a pass), set by the tuner
// through zkp_ntt_set_max_digit; 0 means MAX_D.  A smaller cap means more passes but smaller
// CTAs, several of which share an SM (one loads or stores while another computes).
std::atomic<u32> g_max_digit[29];

inline u32 digit_cap(u32 L) {
    const u32 d = L < 29 ? g_max_digit[L].load(std::memory_order_relaxed) : 0;
    return d ? d : MAX_D;
}

// Balanced split of L bits into passes of at most `cap` bits, top digit first, written into
// p starting at pass `first` with the digits below bit `top`.
inline void split_digits(Plan &p, u32 first, u32 L, u32 cap) {
    const u32 np = (L + cap - 1) / cap;
    const u32 base = L / np, extra = L % np;
    u32 rem = L;
    for (u32 i = 0; i < np; i++) {
        p.D[first + i] = base + (i < extra ? 1 : 0);
        rem -= p.D[first + i];
        p.lo[first + i] = rem;
    }
    p.np = first + np;
}

// Plan for 2^L elements.  The tuned digit cap applies to plain table-mode transforms.  A
// transform whose first pass multiplies by a coset shift or reads a shorter source keeps that
// pass at up to MAX_D bits: the first pass builds per-pencil shift tables, and the cost of
// that set-up grows with the number of pencils.  Recompute mode (roots rebuilt per pencil) and
// the batched form (one shared-memory pencil kernel for every pass) ignore the cap.
inline Plan make_plan(u32 L, bool wide_first = false, bool ignore_cap = false) {
    Plan p{};
    const u32 cap = ignore_cap ? MAX_D : digit_cap(L);
    const u32 first_cap = wide_first ? (cap > MAX_D ? cap : MAX_D) : cap;
    if (L <= first_cap) {
        p.np = 1;
        p.D[0] = L;
        p.lo[0] = 0;
        return p;
    }
    if (!wide_first || first_cap == cap) {
        split_digits(p, 0, L, cap);
        return p;
    }
    p.D[0] = first_cap;
    p.lo[0] = L - first_cap;
    split_digits(p, 1, L - first_cap, cap);
    return p;
}

std::atomic<uint64_t> g_attr_done{0};
std::atomic<uint64_t> g_batch_attr_done{0};
std::atomic<uint64_t> g_br_attr_done{0};
std::atomic<uint64_t> g_lbr_attr_done[BR_T + 1][2];

inline size_t pass_smem(u32 D) {
    const size_t S = 1u << D, H = S > 1 ? S / 2 : 1;
    return (8 * S + 8 * H + 8 * 128) * sizeof(u32);
}

// The register pass handles table-mode passes of at most 2^6-point pencils without a source,
// coset shift or natural-order store (pass_body does those), on at least 2^7 elements so that
// every warp is full.
inline bool warp_pass_ok(const PassArgs &a) {
    return a.D >= 1 && a.D <= WARP_MAX_D && a.L >= 7 &&
           (a.flags & (F_RECOMPUTE | F_PRESHIFT | F_SRC | F_NATURAL)) == 0;
}

cudaError_t launch_pass(const PassArgs &a, cudaStream_t stream) {
    if (warp_pass_ok(a)) {
        if (a.shoup) return launch_warp_pass<ZK_NTT_WARP_PENCILS, true>(a, stream);
        return launch_warp_pass<ZK_NTT_WARP_PENCILS, false>(a, stream);
    }
    ZK_TRY(ensure_smem_attr(ntt_pass_kernel, (int)pass_smem(MAX_D), g_attr_done));
    const u64 pencils = 1ull << (a.L - a.D);
    const u32 H = (1u << a.D) >> 1;
    const u32 threads = H == 0 ? 1 : (H < MAX_THREADS ? H : MAX_THREADS);
    dim3 grid;
    if (pencils <= 65535ull * 1024) {
        grid.x = (u32)(pencils < 65535 ? pencils : 65535);
        grid.y = (u32)((pencils + grid.x - 1) / grid.x);
        if ((u64)grid.x * grid.y != pencils) {
            // pencils is a power of two, so choose x as a power of two too
            u32 gx = 1;
            while ((u64)gx * 2 <= pencils && gx * 2 <= 32768) gx *= 2;
            grid.x = gx;
            grid.y = (u32)(pencils / gx);
        }
    } else {
        return cudaErrorInvalidValue;
    }
    ntt_pass_kernel<<<grid, threads, pass_smem(a.D), stream>>>(a);
    return cudaGetLastError();
}

// The last pass and the permutation in one kernel when the last pass is a register pass of at
// most 2^BR_T points on at least 2^(2 BR_T) elements.
inline bool fuse_last(const Plan &plan, u32 L, bool recompute) {
    return plan.np > 1 && L >= 2 * BR_T && !recompute && plan.D[plan.np - 1] <= BR_T;
}

template <u32 D, bool SH>
cudaError_t launch_last_bitrev_d(const PassArgs &a, cudaStream_t stream) {
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<D, SH>, (int)BR_SMEM, g_lbr_attr_done[D][SH ? 1 : 0]));
    ntt_last_bitrev_kernel<D, SH><<<1u << (a.L - 2 * BR_T), 512, BR_SMEM, stream>>>(a);
    return cudaGetLastError();
}

template <bool SH>
cudaError_t launch_last_bitrev(const PassArgs &a, cudaStream_t stream) {
    switch (a.D) {
        case 1: return launch_last_bitrev_d<1, SH>(a, stream);
        case 2: return launch_last_bitrev_d<2, SH>(a, stream);
        case 3: return launch_last_bitrev_d<3, SH>(a, stream);
        case 4: return launch_last_bitrev_d<4, SH>(a, stream);
        default: return launch_last_bitrev_d<5, SH>(a, stream);
    }
}

// the shared-memory limits of every kernel run() may launch, set ahead of a stream capture
inline cudaError_t prepare_run_attrs() {
    ZK_TRY(ensure_smem_attr(ntt_pass_kernel, (int)pass_smem(MAX_D), g_attr_done));
    ZK_TRY(ensure_smem_attr(bitrev_tiled_kernel, (int)BR_SMEM, g_br_attr_done));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<1, false>, (int)BR_SMEM, g_lbr_attr_done[1][0]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<2, false>, (int)BR_SMEM, g_lbr_attr_done[2][0]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<3, false>, (int)BR_SMEM, g_lbr_attr_done[3][0]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<4, false>, (int)BR_SMEM, g_lbr_attr_done[4][0]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<5, false>, (int)BR_SMEM, g_lbr_attr_done[5][0]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<1, true>, (int)BR_SMEM, g_lbr_attr_done[1][1]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<2, true>, (int)BR_SMEM, g_lbr_attr_done[2][1]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<3, true>, (int)BR_SMEM, g_lbr_attr_done[3][1]));
    ZK_TRY(ensure_smem_attr(ntt_last_bitrev_kernel<4, true>, (int)BR_SMEM, g_lbr_attr_done[4][1]));
    return ensure_smem_attr(ntt_last_bitrev_kernel<5, true>, (int)BR_SMEM, g_lbr_attr_done[5][1]);
}

// Runs the full plan.  src (if non-null) is the pass-0 source for the coset LDE.
cudaError_t run(const View &v, const View *src, u64 src_len, u32 L, const u32 *tw, const u32 *omegas,
                const u32 *shift, const u32 *scale, cudaStream_t stream, const u32 *shoup = nullptr) {
    profiler().begin(stream);
    if (omegas == nullptr && (shift != nullptr || src != nullptr) && L >= PREP_MIN_L) {
        // a multi-pass table-mode plan: shift and zero-extend in one elementwise pass, then the
        // plain transform in place
        const u64 n = 1ull << L;
        const u64 warps = (n + 32ull * PREP_C - 1) / (32ull * PREP_C);
        coset_prep_kernel<<<(u32)((warps * 32 + 255) / 256), 256, 0, stream>>>(v, src ? *src : View{}, src_len,
                                                                               src != nullptr, shift, n);
        ZK_TRY(cudaGetLastError());
        profiler().mark("ntt_prep", stream);
        shift = nullptr;
        src = nullptr;
        src_len = 0;
    }
    const Plan plan = make_plan(L, shift != nullptr || src != nullptr, omegas != nullptr);
    const bool fused_tail = fuse_last(plan, L, omegas != nullptr);
    for (u32 p = 0; p < plan.np; p++) {
        PassArgs a{};
        a.v = v;
        if (src) a.src = *src;
        a.tw = tw;
        a.omegas = omegas;
        a.shift = shift;
        a.scale = scale;
        a.shoup = shoup;
        a.L = L;
        a.D = plan.D[p];
        a.lo = plan.lo[p];
        a.src_len = src_len;
        u32 f = 0;
        if (a.lo > 0) f |= F_TWIST;
        if (plan.np == 1) f |= F_NATURAL;
        if (p + 1 == plan.np) {
            f |= F_CANON;
            if (scale) f |= F_POSTSCALE;
        }
        if (p == 0 && shift) f |= F_PRESHIFT;
        if (p == 0 && src) f |= F_SRC;
        if (omegas) f |= F_RECOMPUTE;
        a.flags = f;
        if (fused_tail && p + 1 == plan.np) {
            ZK_TRY(shoup ? launch_last_bitrev<true>(a, stream) : launch_last_bitrev<false>(a, stream));
            profiler().mark("ntt_pass", stream);
            return cudaSuccess;
        }
        ZK_TRY(launch_pass(a, stream));
        profiler().mark("ntt_pass", stream);
    }
    if (plan.np > 1) {
        const u64 n = 1ull << L;
        if (L >= 2 * BR_T) {
            ZK_TRY(ensure_smem_attr(bitrev_tiled_kernel, (int)BR_SMEM, g_br_attr_done));
            bitrev_tiled_kernel<<<1u << (L - 2 * BR_T), 256, BR_SMEM, stream>>>(v, L);
        } else {
            const u64 blocks = (n / 2 + 255) / 256;
            const u32 grid = (u32)(blocks < (u64)num_sms() * 16 ? blocks : (u64)num_sms() * 16);
            bitrev_kernel<<<grid, 256, 0, stream>>>(v, L, n);
        }
        ZK_TRY(cudaGetLastError());
        profiler().mark("bitrev", stream);
    }
    return cudaSuccess;
}

}  // namespace ntt
}  // namespace zk

using namespace zk;

ZK_DEFINE_PROFILER_API(zkp_ntt)

extern "C" cudaError_t ssip_ntt(PolyPtr x, const unsigned int *twiddle, unsigned int log_len, cudaStream_t stream,
                                const unsigned int, const unsigned int) {
    if (log_len == 0) return cudaSuccess;
    ZK_CHECK_ARG(log_len <= 28 && twiddle != nullptr);
    ZK_CHECK_ARG(x.len == (1ull << log_len));
    View v;
    ZK_CHECK_ARG(make_view(x, &v));
    return ntt::run(v, nullptr, 0, log_len, twiddle, nullptr, nullptr, nullptr, stream);
}

extern "C" cudaError_t zkp_ntt_ex(PolyPtr x, const unsigned int *twiddle, unsigned int log_len,
                                  const unsigned int *shift_d, const unsigned int *scale_d, cudaStream_t stream) {
    return zkp_ntt_ex_shoup(x, twiddle, nullptr, log_len, shift_d, scale_d, stream);
}

extern "C" cudaError_t zkp_ntt_ex_shoup(PolyPtr x, const unsigned int *twiddle, const unsigned int *shoup_d,
                                        unsigned int log_len, const unsigned int *shift_d,
                                        const unsigned int *scale_d, cudaStream_t stream) {
    ZK_CHECK_ARG(log_len <= 28 && twiddle != nullptr);
    ZK_CHECK_ARG(x.len == (1ull << log_len));
    ZK_CHECK_ARG((reinterpret_cast<uintptr_t>(shoup_d) & 15) == 0);
    View v;
    ZK_CHECK_ARG(make_view(x, &v));
    if (log_len == 0) {
        // a length-1 transform is the identity, but shift^0 = 1 and the scale still apply
        if (!scale_d) return cudaSuccess;
        return distribute_powers(x, scale_d, 1, stream);
    }
    return ntt::run(v, nullptr, 0, log_len, twiddle, nullptr, shift_d, scale_d, stream, shoup_d);
}

extern "C" cudaError_t zkp_coset_lde(PolyPtr out, ConstPolyPtr in, const unsigned int *twiddle, unsigned int log_in,
                                     unsigned int log_out, const unsigned int *shift_d, cudaStream_t stream) {
    return zkp_coset_lde_shoup(out, in, twiddle, nullptr, log_in, log_out, shift_d, stream);
}

extern "C" cudaError_t zkp_coset_lde_shoup(PolyPtr out, ConstPolyPtr in, const unsigned int *twiddle,
                                           const unsigned int *shoup_d, unsigned int log_in, unsigned int log_out,
                                           const unsigned int *shift_d, cudaStream_t stream) {
    ZK_CHECK_ARG(log_out <= 28 && log_in <= log_out && log_out >= 1 && twiddle != nullptr);
    ZK_CHECK_ARG(out.len == (1ull << log_out) && in.len == (1ull << log_in));
    ZK_CHECK_ARG((reinterpret_cast<uintptr_t>(shoup_d) & 15) == 0);
    View vo, vi;
    ZK_CHECK_ARG(make_view(out, &vo) && make_view(in, &vi));
    return ntt::run(vo, &vi, in.len, log_out, twiddle, nullptr, shift_d, nullptr, stream, shoup_d);
}

// Shoup-product throughput probe (the twiddle product of the register passes): every thread
// runs two independent chains of `iters` products x = x * w by fixed factors.
__global__ void __launch_bounds__(256) shoup_probe_kernel(u32 iters, u32 *out) {
    const u32 tid = blockIdx.x * blockDim.x + threadIdx.x;
    Fr x, y, ys, u, v, vs;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        x.v[k] = (tid + 1) * 0x9e3779b9u + k * 0x85ebca6bu;
        y.v[k] = (tid + 7) * 0xc2b2ae35u + k * 0x27d4eb2fu;
        u.v[k] = x.v[k] ^ 0x165667b1u;
        v.v[k] = y.v[k] ^ 0xd3a2646cu;
        ys.v[k] = y.v[k] * 0x7feb352du;
        vs.v[k] = v.v[k] * 0x846ca68bu;
    }
    x.v[7] &= 0x1fffffffu;  // below the modulus
    y.v[7] &= 0x1fffffffu;
    u.v[7] &= 0x1fffffffu;
    v.v[7] &= 0x1fffffffu;
    for (u32 i = 0; i < iters; i++) {
        x = Fr::mul_shoup(x, y, ys);
        u = Fr::mul_shoup(u, v, vs);
    }
    Fr::add(x, u).store(out + (u64)tid * 8);
}

// blocks x 256 threads x iters x 2 Shoup products; out_d holds blocks * 256 * 8 words
extern "C" cudaError_t zkp_ntt_shoup_probe(unsigned int blocks, unsigned int iters, unsigned int *out_d,
                                           cudaStream_t stream) {
    shoup_probe_kernel<<<blocks, 256, 0, stream>>>(iters, out_d);
    return cudaGetLastError();
}

extern "C" cudaError_t zkp_ntt_shoup_table(const unsigned int *twiddle_d, unsigned int log_len, unsigned int *table_d,
                                           cudaStream_t stream) {
    ZK_CHECK_ARG(log_len >= 1 && log_len <= 28 && twiddle_d != nullptr && table_d != nullptr);
    ZK_CHECK_ARG((reinterpret_cast<uintptr_t>(twiddle_d) & 15) == 0 && (reinterpret_cast<uintptr_t>(table_d) & 15) == 0);
    const u64 count = 1ull << (log_len - 1);
    const u64 blocks = (count + 255) / 256;
    const u32 grid = (u32)(blocks < (u64)num_sms() * 8 ? blocks : (u64)num_sms() * 8);
    ntt::shoup_table_kernel<<<grid, 256, 0, stream>>>(twiddle_d, count, table_d);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ batched form
// Tasks of at least 2^solo_log points run their own tuned plan (register passes, Shoup
// twiddles when given) instead of the shared persistent pencil launches, which use the
// shared-memory pass for every pass.
namespace zk {
namespace ntt {
std::atomic<u32> g_batch_solo_log{16};
}  // namespace ntt
}  // namespace zk

struct ZkpNttBatchPlan {
    struct Solo {
        View v;
        u32 L;
        const u32 *tw, *shift, *scale, *shoup;
    };
    struct Phase {
        ntt::PassArgs *args;
        u64 *first;
        u32 count;
        size_t smem;
        u32 threads;
        u32 grid;
    };
    int device = 0;
    std::vector<Phase> phases;
    View *br_views = nullptr;
    u32 *br_logs = nullptr;
    u64 *br_first = nullptr;
    u32 br_count = 0;
    u64 br_total = 0;
    std::vector<Solo> solo;
    void *mem = nullptr;
};

extern "C" cudaError_t zkp_ntt_batch_plan_create(const ZkpNttTask *tasks, unsigned int ntasks,
                                                 ZkpNttBatchPlan **out) {
    ZK_CHECK_ARG(out != nullptr && (ntasks == 0 || tasks != nullptr));
    auto *plan = new ZkpNttBatchPlan();
    cudaGetDevice(&plan->device);
    // host images of every phase's tables, then one device allocation
    std::vector<std::vector<ntt::PassArgs>> args;
    std::vector<std::vector<u64>> firsts;
    std::vector<View> br_views;
    std::vector<u32> br_logs;
    std::vector<u64> br_first{0};
    const u32 solo_log = ntt::g_batch_solo_log.load(std::memory_order_relaxed);
    for (u32 t = 0; t < ntasks; t++) {
        const ZkpNttTask &task = tasks[t];
        const u32 L = task.log_len;
        View v;
        if (L == 0 || L > 28 || task.x.len != (1ull << L) || task.twiddle == nullptr || !make_view(task.x, &v) ||
            (reinterpret_cast<uintptr_t>(task.shoup_d) & 15) != 0) {
            delete plan;
            return cudaErrorInvalidValue;
        }
        if (solo_log != 0 && L >= solo_log) {
            plan->solo.push_back({v, L, task.twiddle, task.shift_d, task.scale_d, task.shoup_d});
            continue;
        }
        const ntt::Plan p = ntt::make_plan(L, task.shift_d != nullptr, /*ignore_cap=*/true);
        for (u32 ph = 0; ph < p.np; ph++) {
            if (args.size() <= ph) {
                args.emplace_back();
                firsts.emplace_back(1, 0);
            }
            ntt::PassArgs a{};
            a.v = v;
            a.tw = task.twiddle;
            a.shift = task.shift_d;
            a.scale = task.scale_d;
            a.L = L;
            a.D = p.D[ph];
            a.lo = p.lo[ph];
            u32 f = 0;
            if (a.lo > 0) f |= ntt::F_TWIST;
            if (p.np == 1) f |= ntt::F_NATURAL;
            if (ph + 1 == p.np) {
                f |= ntt::F_CANON;
                if (task.scale_d) f |= ntt::F_POSTSCALE;
            }
            if (ph == 0 && task.shift_d) f |= ntt::F_PRESHIFT;
            a.flags = f;
            args[ph].push_back(a);
            firsts[ph].push_back(firsts[ph].back() + (1ull << (L - a.D)));
        }
        if (p.np > 1) {
            br_views.push_back(v);
            br_logs.push_back(L);
            br_first.push_back(br_first.back() + (1ull << L));
        }
    }
    size_t bytes = 0;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    for (size_t ph = 0; ph < args.size(); ph++)
        bytes += al(args[ph].size() * sizeof(ntt::PassArgs)) + al(firsts[ph].size() * sizeof(u64));
    bytes += al(br_views.size() * sizeof(View) + 16) + al(br_logs.size() * 4 + 16) + al(br_first.size() * 8);
    cudaError_t err = cudaMalloc(&plan->mem, bytes ? bytes : 256);
    if (err != cudaSuccess) {
        delete plan;
        return err;
    }
    char *base = reinterpret_cast<char *>(plan->mem);
    size_t off = 0;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, plan->device);
    err = ensure_smem_attr(ntt::ntt_batch_pass_kernel, (int)ntt::pass_smem(ntt::MAX_D), ntt::g_batch_attr_done);
    // the solo tasks' kernels get their shared-memory limits now, outside any stream capture
    if (err == cudaSuccess && !plan->solo.empty()) err = ntt::prepare_run_attrs();
    for (size_t ph = 0; ph < args.size() && err == cudaSuccess; ph++) {
        ZkpNttBatchPlan::Phase P{};
        P.args = reinterpret_cast<ntt::PassArgs *>(base + off);
        off += al(args[ph].size() * sizeof(ntt::PassArgs));
        P.first = reinterpret_cast<u64 *>(base + off);
        off += al(firsts[ph].size() * sizeof(u64));
        P.count = (u32)args[ph].size();
        u32 maxD = 1;
        for (auto &a : args[ph]) maxD = a.D > maxD ? a.D : maxD;
        P.smem = ntt::pass_smem(maxD);
        const u32 H = (1u << maxD) >> 1;
        P.threads = H < ntt::MAX_THREADS ? (H ? H : 1) : ntt::MAX_THREADS;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ntt::ntt_batch_pass_kernel, (int)P.threads, P.smem);
        if (per_sm < 1) per_sm = 1;
        const u64 total = firsts[ph].back();
        const u64 cap = (u64)num_sms() * per_sm;
        P.grid = (u32)(total < cap ? total : cap);
        err = cudaMemcpy(P.args, args[ph].data(), args[ph].size() * sizeof(ntt::PassArgs), cudaMemcpyHostToDevice);
        if (err == cudaSuccess)
            err = cudaMemcpy(P.first, firsts[ph].data(), firsts[ph].size() * sizeof(u64), cudaMemcpyHostToDevice);
        plan->phases.push_back(P);
    }
    if (err == cudaSuccess && !br_views.empty()) {
        plan->br_views = reinterpret_cast<View *>(base + off);
        off += al(br_views.size() * sizeof(View) + 16);
        plan->br_logs = reinterpret_cast<u32 *>(base + off);
        off += al(br_logs.size() * 4 + 16);
        plan->br_first = reinterpret_cast<u64 *>(base + off);
        plan->br_count = (u32)br_views.size();
        plan->br_total = br_first.back();
        err = cudaMemcpy(plan->br_views, br_views.data(), br_views.size() * sizeof(View), cudaMemcpyHostToDevice);
        if (err == cudaSuccess)
            err = cudaMemcpy(plan->br_logs, br_logs.data(), br_logs.size() * 4, cudaMemcpyHostToDevice);
        if (err == cudaSuccess)
            err = cudaMemcpy(plan->br_first, br_first.data(), br_first.size() * 8, cudaMemcpyHostToDevice);
    }
    if (err != cudaSuccess) {
        cudaFree(plan->mem);
        delete plan;
        return err;
    }
    *out = plan;
    return cudaSuccess;
}

// launches only (no allocation, no host copies), so a stream capture can record it
extern "C" cudaError_t zkp_ntt_batch_run(const ZkpNttBatchPlan *plan, cudaStream_t stream) {
    ZK_CHECK_ARG(plan != nullptr);
    for (const auto &P : plan->phases) {
        if (P.count == 0 || P.grid == 0) continue;
        ntt::ntt_batch_pass_kernel<<<P.grid, P.threads, P.smem, stream>>>(P.args, P.first, P.count);
        ZK_TRY(cudaGetLastError());
    }
    if (plan->br_count) {
        const u64 blocks = (plan->br_total / 2 + 255) / 256;
        const u32 grid = (u32)(blocks < (u64)num_sms() * 16 ? blocks : (u64)num_sms() * 16);
        ntt::bitrev_batch_kernel<<<grid, 256, 0, stream>>>(plan->br_views, plan->br_logs, plan->br_first,
                                                          plan->br_count);
        ZK_TRY(cudaGetLastError());
    }
    for (const auto &t : plan->solo)
        ZK_TRY(ntt::run(t.v, nullptr, 0, t.L, t.tw, nullptr, t.shift, t.scale, stream, t.shoup));
    return cudaSuccess;
}

extern "C" cudaError_t zkp_ntt_batch_set_solo_log(unsigned int log_len) {
    ZK_CHECK_ARG(log_len <= 29);
    ntt::g_batch_solo_log.store(log_len);
    return cudaSuccess;
}

extern "C" void zkp_ntt_batch_plan_destroy(ZkpNttBatchPlan *plan) {
    if (!plan) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(plan->device);
    cudaFree(plan->mem);
    cudaSetDevice(prev);
    delete plan;
}

extern "C" cudaError_t zkp_ntt_set_max_digit(unsigned int log_len, unsigned int max_digit) {
    ZK_CHECK_ARG(log_len <= 28 && (max_digit == 0 || (max_digit >= 4 && max_digit <= ntt::MAX_D)));
    if (log_len == 0) {
        for (u32 L = 0; L < 29; L++) ntt::g_max_digit[L].store(max_digit);
    } else {
        ntt::g_max_digit[log_len].store(max_digit);
    }
    return cudaSuccess;
}

extern "C" cudaError_t zkp_ntt_set_block(unsigned int log_len, unsigned int threads) {
    ZK_CHECK_ARG(log_len <= 28 && (threads == 0 || threads == 32 || threads == 64 || threads == 128 ||
                                   threads == 256));
    if (log_len == 0) {
        for (u32 L = 0; L < 29; L++) ntt::g_warp_block[L].store(threads);
    } else {
        ntt::g_warp_block[log_len].store(threads);
    }
    return cudaSuccess;
}

extern "C" unsigned int zkp_ntt_plan_digits(unsigned int log_len, unsigned int *digits, unsigned int max) {
    if (log_len == 0 || log_len > 28) return 0;
    const ntt::Plan p = ntt::make_plan(log_len);
    for (u32 i = 0; i < p.np && i < max && digits; i++) digits[i] = p.D[i];
    return p.np;
}

extern "C" unsigned int zkp_ntt_num_passes(unsigned int log_len) {
    ntt::Plan p = ntt::make_plan(log_len);
    if (ntt::fuse_last(p, log_len, false)) return p.np;  // the last pass also permutes
    return p.np + (p.np > 1 ? 1 : 0);
}

extern "C" cudaError_t recompute_ntt(PolyPtr x, const unsigned int *pq_d, unsigned int pq_deg,
                                     const unsigned int *omegas_d, unsigned int log_len, cudaStream_t stream,
                                     const unsigned int, const unsigned int) {
    (void)pq_d;
    (void)pq_deg;
    if (log_len == 0) return cudaSuccess;
    ZK_CHECK_ARG(log_len <= 28 && omegas_d != nullptr);
    ZK_CHECK_ARG(x.len == (1ull << log_len));
    View v;
    ZK_CHECK_ARG(make_view(x, &v));
    return ntt::run(v, nullptr, 0, log_len, nullptr, omegas_d, nullptr, nullptr, stream);
}

extern "C" cudaError_t distribute_powers(PolyPtr poly, const unsigned int *powers, unsigned long long power_num,
                                         cudaStream_t stream) {
    View v;
    ZK_CHECK_ARG(make_view(poly, &v));
    if (v.len == 0) return cudaSuccess;
    ZK_CHECK_ARG(powers != nullptr && power_num > 0);
    const u64 blocks = (v.len + 255) / 256;
    const u32 grid = (u32)(blocks < (u64)num_sms() * 32 ? blocks : (u64)num_sms() * 32);
    ntt::distribute_powers_kernel<<<grid, 256, 0, stream>>>(v, powers, power_num, v.len);
    return cudaGetLastError();
}

extern "C" cudaError_t zkp_ntt_roots_device(unsigned int *out_d, unsigned long long count, const unsigned int *unit_d,
                                            cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    ZK_CHECK_ARG(out_d != nullptr && unit_d != nullptr);
    const u64 threads = (count + 63) / 64;
    ntt::powers_kernel<<<(u32)((threads + 255) / 256), 256, 0, stream>>>(out_d, unit_d, count);
    return cudaGetLastError();
}

extern "C" cudaError_t ssip_precompute(unsigned int *twiddle, unsigned int len, const unsigned int *unit) {
    if (len == 0) return cudaSuccess;
    ZK_CHECK_ARG(twiddle != nullptr && unit != nullptr);
    // roots are generated on the device and copied to the caller's host table
    u32 *d_out = nullptr, *d_unit = nullptr;
    ZK_TRY(cudaMalloc(&d_out, (size_t)len * 32));
    cudaError_t err = cudaMalloc(&d_unit, 32);
    if (err == cudaSuccess) err = cudaMemcpy(d_unit, unit, 32, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        const u64 threads = ((u64)len + 63) / 64;
        ntt::powers_kernel<<<(u32)((threads + 255) / 256), 256>>>(d_out, d_unit, len);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(twiddle, d_out, (size_t)len * 32, cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    if (d_unit) cudaFree(d_unit);
    return err;
}

extern "C" void gen_pq_omegas(unsigned int *pq, unsigned int *omegas, unsigned int pq_deg, unsigned int len,
                              unsigned int *unit) {
    // precompute.cuh:89-113, byte for byte
    const zkh::Params &P = zkh::fr();
    const zkh::Fe u = zkh::load(unit);
    const size_t pq_len = (size_t)(1u << pq_deg >> 1);
    memset(pq, 0, pq_len * 32);
    zkh::store(pq, zkh::one(P));
    zkh::Fe tw = zkh::pow(P, u, (uint64_t)(len >> pq_deg));
    if (pq_deg > 1) {
        zkh::store(pq + 8, tw);
        zkh::Fe last = tw;
        for (size_t i = 2; i < pq_len; i++) {
            last = zkh::mul(P, last, tw);
            zkh::store(pq + i * 8, last);
        }
    }
    zkh::store(omegas, u);
    zkh::Fe last = u;
    for (int i = 1; i < 32; i++) {
        last = zkh::mul(P, last, last);
        zkh::store(omegas + i * 8, last);
    }
}
