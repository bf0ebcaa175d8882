// libmsm.so: Pippenger multi-scalar multiplication over BN254 G1 for sm_100a.
//
// Replaces the reference's MSM (core/src/msm/src/msm.cu:9-50, msm_impl.cuh:22-909) behind
// the same C ABI (core/src/msm/src/msm.h:4-11) and adds an asynchronous device-pointer entry
// for resident bases.  Result: sum_i s_i * P_i as a canonical affine Montgomery point,
// identity = (0, 0), exactly what the reference returns after to_affine (msm.cu:38).
//
// Pipeline (all on the device, no locks, no host arithmetic):
//   1. digits:   each scalar leaves Montgomery form (to_number, msm_impl.cuh:52), is cut into
//                W windows of c bits and recoded to signed digits in [-2^(c-1), 2^(c-1)]
//                (signed_digit, msm_impl.cuh:22-33); non-zero digits count into per-bucket
//                histograms.  With precomputed tables (reference MSMPrecompute,
//                msm_impl.cuh:776-828) logical window j*Wp + w maps to table j, window w.
//   2. scan:     exclusive prefix sum of the histograms gives every bucket's run.
//   3. scatter:  digits are recomputed and each (bucket id, point code = index | sign) record
//                lands in its bucket's run, so the records are sorted by (window, bucket) - a
//                counting sort (one launch per task of a batch).
//   4a. pairing rounds (large MSMs): each round adds neighbouring points of every bucket's list
//                in affine coordinates, all of a round's inverses from one inversion
//                (Montgomery's trick over a CTA-level product tree), roughly halving the lists.
//   4. accumulate: the (last) list is cut into equal chunks, one per thread; each thread walks
//                its chunk with mixed XYZZ additions.  Runs wholly inside a chunk are written
//                straight to their bucket; runs cut by a chunk boundary leave partial sums that
//                a fix-up pass joins (one thread per recorded chain).  Load balance does not
//                depend on the scalar distribution.
//   5. reduce:   per window sum_b b * S_b: short segments form their sums and running sums
//                (summation by parts), the segment sums are split by the bits of their
//                index into classes summed in parallel, and the classes are scaled by
//                doublings and added.
//   6. combine:  one thread folds the windows (c doublings each) and normalises to affine.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/msm.h"
#include "common.cuh"
#include "curve.cuh"

namespace zk {
namespace msm {

constexpr int SCALAR_BITS = 254;
constexpr u32 EMPTY = 0xffffffffu;
constexpr u32 MAX_TASKS = 32;

// One MSM of a batch.  A single MSM is a batch of one.
struct Task {
    const u32 *points;   // n_tables tables of n affine points
    const u32 *scalars;  // n Montgomery scalars
    u32 *result;         // 64-byte affine result
    u64 n;
    u64 stride;  // points between consecutive tables (>= n; tables may be longer than n)
    u32 n_tables;
    u32 c;    // window bits
    u32 W;    // logical windows = ceil(254 / c)
    u32 Wp;   // physical windows = ceil(W / n_tables)
    u32 B;    // buckets per window = 2^(c-1)
    u32 L;    // buckets per reduction segment
    u32 gbits;  // log2(B / L): bit classes of the segment index
    u32 parts;  // CTAs per class in the reduction
};

// The whole batch travels as a kernel parameter (no device copy, capturable in a graph).
// Every global index space is the concatenation of the tasks' spaces; *_first are the
// exclusive prefixes (entry ntasks is the total).
struct Batch {
    u32 ntasks;
    u32 K;  // entries per accumulation chunk
    Task task[MAX_TASKS];
    u64 sc_first[MAX_TASKS + 1];   // scalars
    u64 key_first[MAX_TASKS + 1];  // buckets (Wp * B per task)
    u64 seg_first[MAX_TASKS + 1];  // reduction segments (key count / L)
    u32 win_first[MAX_TASKS + 1];  // physical windows
    u32 ncls, nparts;              // largest class count / parts of any task (reduction grid)
    u32 rounds;                    // affine pairing rounds before the XYZZ walk (0 = none)
};

template <typename T>
ZK_DI u32 find_task(const T *first, u32 ntasks, T x) {
    u32 lo = 0, hi = ntasks;  // largest t with first[t] <= x
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (first[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

// CTAs per bit class in the bucket reduction (a power of two); scale_kernel and window_kernel
// fold up to 32 parts and 32 classes, one per lane
constexpr u32 MAX_PARTS = 32;

inline Task make_task(u64 n, u32 c, u32 n_tables) {
    Task t{};
    t.n = n;
    t.stride = n;
    t.c = c;
    t.W = (SCALAR_BITS + c - 1) / c;
    t.n_tables = n_tables;
    t.Wp = (t.W + n_tables - 1) / n_tables;
    t.B = 1u << (c - 1);
    // buckets per reduction segment: 4, or more for large windows so that the bit classes stay
    // small (8 at 2^19 buckets, 16 from 2^20); at least two segments per window
    t.L = t.B >= 8 ? 4 : t.B / 2;
    if (t.B >= (1u << 19)) t.L = t.B >= (1u << 20) ? 16 : 8;
    const u32 G = t.B / t.L;
    t.gbits = 31 - __builtin_clz(G);
    const u32 half = G / 2, per_cta = 256 * 8;  // about 8 additions per thread
    t.parts = half / per_cta < 1 ? 1 : (half / per_cta > MAX_PARTS ? MAX_PARTS : half / per_cta);
    return t;
}

// default window width for n points with one point table (a cost model in the spirit of
// core/src/msm/tuning/cost_model.py: n*W mixed adds vs 2*W*2^(c-1) bucket adds).  From 2^18 to
// 2^23 points the model is replaced by the width measured fastest on B200 with the pairing
// rounds (one table: 15 at 2^18, 2^20 and 2^22, 3-4 % ahead of the model's 16 and 17).
inline u32 default_window(u64 n) {
    if (n >= (1ull << 18) && n <= (1ull << 23)) return 15;
    u32 best = 8;
    double best_cost = 1e300;
    for (u32 c = 8; c <= 20; c++) {
        const double W = (double)((SCALAR_BITS + c - 1) / c);
        const double cost = (double)n * W * 10.0 + W * (double)(1u << (c - 1)) * 2.2 * 14.0 + W * c * 8.0 * 1000.0;
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

// CTA sizes of the stages whose thread count is free (each thread owns its own slots or chunk),
// set by the tuner through zkp_msm_set_block: pair_up, pair_down, accumulate (0 = 256)
enum BlockStage { BLK_PAIR_UP = 0, BLK_PAIR_DOWN = 1, BLK_ACCUMULATE = 2, BLK_STAGES = 3 };
inline std::atomic<u32> *block_settings() {
    static std::atomic<u32> b[BLK_STAGES];
    return b;
}
inline u32 block_for(BlockStage st) {
    const u32 v = block_settings()[st].load(std::memory_order_relaxed);
    return v ? v : 256u;
}

// Affine pairing rounds (stage 4a below): -1 chooses by size, else a fixed count.
constexpr u32 MAX_ROUNDS = 4;
constexpr u32 KA = 64;  // list elements per thread in a pairing round (at most KA / 2 pairs)
inline int &affine_rounds_setting() {
    static int r = -1;
    return r;
}
// measured on B200 (2^19..2^22 points, 15 tables): rounds pay from about 12 M digit entries
inline u32 auto_rounds(u64 entries) {
    if (entries >= (1ull << 26)) return 4;
    if (entries >= (1ull << 24)) return 3;
    return entries >= (3ull << 22) ? 2u : 0u;
}

// upper bounds of the list lengths: E_0 = live digits, E_{r+1} <= sum_b (m_b / 2 + 1) =
// E_r / 2 + nb (a bucket's run leaves at most one unpaired point at each end)
inline u64 next_list_bound(u64 e, u64 nb) {
    const u64 x = (e + 1) / 2 + nb;
    return x < e ? x : e;
}

// fills the prefixes and the chunk size; tasks[] must be set.  rounds < 0: the library
// setting (itself -1 = by size).
inline void finish_batch(Batch &b, int rounds = -1) {
    b.sc_first[0] = b.key_first[0] = b.seg_first[0] = 0;
    b.win_first[0] = 0;
    b.ncls = b.nparts = 1;
    u64 entries = 0;
    for (u32 t = 0; t < b.ntasks; t++) {
        const Task &k = b.task[t];
        b.sc_first[t + 1] = b.sc_first[t] + k.n;
        b.key_first[t + 1] = b.key_first[t] + (u64)k.Wp * k.B;
        b.seg_first[t + 1] = b.seg_first[t] + (u64)k.Wp * k.B / k.L;
        b.win_first[t + 1] = b.win_first[t] + k.Wp;
        b.ncls = b.ncls > k.gbits + 2 ? b.ncls : k.gbits + 2;
        b.nparts = b.nparts > k.parts ? b.nparts : k.parts;
        entries += k.n * k.W;
    }
    if (rounds < 0) rounds = affine_rounds_setting();
    b.rounds = rounds < 0 ? auto_rounds(entries) : (u32)(rounds > (int)MAX_ROUNDS ? MAX_ROUNDS : rounds);
    u64 walk = entries;
    for (u32 r = 0; r < b.rounds; r++) walk = next_list_bound(walk, b.key_first[b.ntasks]);
    entries = walk;
    // chunk so that roughly 4 waves of 384 threads per SM cover the walk's entries
    const u64 threads = (u64)num_sms() * 384 * 4;
    u64 k = (entries + threads - 1) / threads;
    if (k < 8) k = 8;
    if (k > 4096) k = 4096;
    b.K = (u32)k;
}

// ------------------------------------------------------------------ workspace layout
// Montgomery-trick tree over a round's thread totals: a CTA of TREE_CTA threads folds
// TREE_CTA * TREE_PER values per level, so two levels and the top cover 2^36 values
constexpr u32 TREE_CTA = 256, TREE_PER = 16;
constexpr u64 TREE_SPAN = (u64)TREE_CTA * TREE_PER;
constexpr u32 TREE_LEVELS = 3;

struct Layout {
    size_t counts, cursor, sorted_bucket, sorted_point, bucket_sums, part_pts, part_bucket, part_flag, long_list,
        chain_list,
        seg, cls, win, scan_sums, total;
    u64 nb, entries, chunks, segs, wins;
    // affine pairing rounds: list r + 1 (r < rounds) lives in buffer r % 2; starts[r] are the
    // bucket starts of list r (starts[0] = the counts region); thr[r] threads in round r
    u32 rounds;
    u64 emax[MAX_ROUNDS + 1], thr[MAX_ROUNDS];
    size_t starts[MAX_ROUNDS + 1], lst_bkt[2], lst_pts[2], prefix[MAX_ROUNDS], tvals;
    // per tree level: member prefixes, per-thread exclusive prefix / suffix products, and the
    // next level's values (the CTA products)
    size_t tree_pre[TREE_LEVELS + 1], tree_ex[TREE_LEVELS + 1], tree_sx[TREE_LEVELS + 1], tree_dat[TREE_LEVELS + 1];
};

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }


// digit records and bucket ids are indexed with 32-bit positions: a batch must stay below 2^32 of
// each (entry points refuse larger ones)
inline bool batch_fits(const Batch &b) {
    u64 entries = 0;
    for (u32 t = 0; t < b.ntasks; t++) entries += b.task[t].n * b.task[t].W;
    return entries < (1ull << 32) - 1 && b.key_first[b.ntasks] < (1ull << 32) - 1;
}

inline Layout make_layout(const Batch &b) {
    Layout l{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += align_up(bytes);
        return o;
    };
    l.nb = b.key_first[b.ntasks];
    l.entries = 0;
    for (u32 t = 0; t < b.ntasks; t++) l.entries += b.task[t].n * b.task[t].W;
    l.segs = b.seg_first[b.ntasks];
    l.wins = b.win_first[b.ntasks];
    l.rounds = b.rounds;
    l.emax[0] = l.entries;
    for (u32 r = 0; r < l.rounds; r++) {
        l.emax[r + 1] = next_list_bound(l.emax[r], l.nb);
        l.thr[r] = (l.emax[r] + KA - 1) / KA;
    }
    l.chunks = (l.emax[l.rounds] + b.K - 1) / b.K;
    l.counts = take((l.nb + 1) * 4);
    l.cursor = take((l.nb + 1) * 4);
    l.scan_sums = take(((l.nb + 1) / 4096 + 2) * 4);
    // list 0: one 8-byte record per digit (bucket id, point code), written by one store
    l.sorted_bucket = take(l.entries * 8);
    l.sorted_point = l.sorted_bucket + 4;
    if (l.rounds) {
        l.starts[0] = l.counts;
        for (u32 r = 1; r <= l.rounds; r++) l.starts[r] = take((l.nb + 1) * 4);
        for (u32 i = 0; i < 2 && i < l.rounds; i++) {
            l.lst_bkt[i] = take(l.emax[i + 1] * 4);
            l.lst_pts[i] = take(l.emax[i + 1] * 64);
        }
        // Prefix products (slot-major, KA / 2 slots a thread).  Round 0 keeps them in list
        // buffer 1, which round 1 fills only later; the later rounds in the sorted arrays,
        // which round 0 has consumed.  Either falls back to space of its own when too small.
        const u64 pre0 = l.thr[0] * (KA / 2) * 32;
        l.prefix[0] = (l.rounds >= 2 && pre0 <= l.emax[2] * 64) ? l.lst_pts[1] : take(pre0);
        if (l.rounds >= 2) {
            const u64 pre1 = l.thr[1] * (KA / 2) * 32;  // thr[r] <= thr[1] for r >= 1
            const size_t sorted_bytes = l.entries * 8;
            const size_t at1 = pre1 <= sorted_bytes ? l.sorted_bucket : take(pre1);
            for (u32 r = 1; r < l.rounds; r++) l.prefix[r] = at1;
        }
        l.tvals = take(l.thr[0] * 32);
        u64 m = l.thr[0];
        for (u32 k = 0; k <= TREE_LEVELS; k++) l.tree_pre[k] = l.tree_ex[k] = l.tree_sx[k] = l.tree_dat[k] = 0;
        for (u32 k = 0; k <= TREE_LEVELS; k++) {
            l.tree_pre[k] = take(m * 32);  // the top level uses only this one
            if (m <= TREE_SPAN) break;
            const u64 ctas = (m + TREE_SPAN - 1) / TREE_SPAN;
            l.tree_ex[k] = take(ctas * TREE_CTA * 32);
            l.tree_sx[k] = take(ctas * TREE_CTA * 32);
            m = ctas;
            l.tree_dat[k + 1] = take(m * 32);
        }
    }
    l.bucket_sums = take(l.nb * 128);
    l.part_pts = take(l.chunks * 2 * 128);
    l.part_bucket = take(l.chunks * 2 * 4);
    l.part_flag = take(l.chunks * 2 * 4);
    l.long_list = take((l.chunks + 1) * 4 + 4);  // long chain starts + a counter at the end
    l.chain_list = take((l.chunks + 1) * 4);     // chain starts + a counter at the end
    l.seg = take(2 * l.segs * 128);  // U_g then T_g
    l.cls = take(l.wins * b.ncls * b.nparts * 128);
    l.win = take(l.wins * 128);
    l.total = off;
    return l;
}

// canonical negation: q - y, with 0 kept
ZK_DI Fq neg_canonical(const Fq &y) { return Fq::sub_c(Fq::zero(), y); }

// ------------------------------------------------------------------ 1 + 3: digits
// signed c-bit digits of the canonical scalar, least significant window first
struct Digits {
    u32 limbs[8];
    u32 c;

    ZK_DI u32 raw(u32 w) const {
        const u32 bit = w * c;
        const u32 word = bit >> 5, sh = bit & 31;
        if (word >= 8) return 0;
        u64 v = limbs[word];
        if (word + 1 < 8) v |= (u64)limbs[word + 1] << 32;
        return (u32)(v >> sh) & ((1u << c) - 1);
    }
};

ZK_DI void load_digits(Digits &d, const u32 *scalar, u32 c) {
    Fr s = Fr::load(scalar);
    Fr num = s.to_number();
#pragma unroll
    for (int i = 0; i < 8; i++) d.limbs[i] = num.v[i];
    d.c = c;
}

// per (scalar, window) with a non-zero digit: f(table, local bucket key, negative).  Digits
// are signed in [-2^(c-1), 2^(c-1)]: a raw window value above 2^(c-1) becomes raw - 2^c with
// a carry into the next window (signed_digit, msm_impl.cuh:22-33).  254 is not a multiple of
// c for any c in [2, 24] except 2, so the top window never carries out.
template <typename F>
ZK_DI void for_each_digit(const Digits &d, const Task &k, F &&f) {
    u32 carry = 0;
    const u32 half = 1u << (k.c - 1);
    for (u32 w = 0; w < k.W; w++) {
        u32 raw = d.raw(w) + carry;
        bool neg = false;
        u32 mag;
        if (raw > half) {
            mag = (1u << k.c) - raw;
            neg = true;
            carry = 1;
        } else {
            mag = raw;
            carry = 0;
        }
        if (mag != 0) {
            const u32 table = w / k.Wp, pw = w % k.Wp;
            f(table, pw * k.B + mag - 1, neg);
        }
    }
}

__global__ void __launch_bounds__(256) count_kernel(const Batch b, u32 *counts) {
    const u64 total = b.sc_first[b.ntasks];
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const u32 t = find_task(b.sc_first, b.ntasks, g);
        const Task &k = b.task[t];
        const u64 i = g - b.sc_first[t];
        Digits d;
        load_digits(d, k.scalars + i * 8, k.c);
        u32 *cnt = counts + b.key_first[t];
        for_each_digit(d, k, [&](u32, u32 key, bool) { atomicAdd(cnt + key, 1u); });
    }
}

// Scalars [first, last) of the batch's concatenation (one launch per task, so that the
// records being written at any time fall into one task's buckets: with a whole batch at once the
// open write positions of millions of buckets overflow L2).
__global__ void __launch_bounds__(256) scatter_kernel(const Batch b, u32 *cursor, uint2 *records, u64 first,
                                                     u64 last) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 g = first + (u64)blockIdx.x * blockDim.x + threadIdx.x; g < last; g += stride) {
        const u32 t = find_task(b.sc_first, b.ntasks, g);
        const Task &k = b.task[t];
        const u64 i = g - b.sc_first[t];
        const u32 kb = (u32)b.key_first[t];
        Digits d;
        load_digits(d, k.scalars + i * 8, k.c);
        // records queue up QD at a time, so QD cursor atomics are in flight before the first of
        // their stores waits on a returned position; the queue keeps the digits' order
        constexpr u32 QD = 4;
        u32 qk[QD], qv[QD], nq = 0;
        auto flush = [&]() {
            u32 pos[QD];
#pragma unroll
            for (u32 q = 0; q < QD; q++)
                if (q < nq) pos[q] = atomicAdd(cursor + qk[q], 1u);
#pragma unroll
            for (u32 q = 0; q < QD; q++)
                if (q < nq) records[pos[q]] = make_uint2(qk[q], qv[q]);
            nq = 0;
        };
        for_each_digit(d, k, [&](u32 table, u32 key, bool neg) {
            const u32 id = kb + key, v = (u32)(table * k.stride + i) | (neg ? 0x80000000u : 0u);
#pragma unroll
            for (u32 q = 0; q < QD; q++)
                if (q == nq) {
                    qk[q] = id;
                    qv[q] = v;
                }
            if (++nq == QD) flush();
        });
        flush();
    }
}

// ------------------------------------------------------------------ 2: exclusive scan
// three-phase scan of u32 counts: block sums, scan of block sums, per-block scan + offset
constexpr u32 SCAN_BLOCK = 1024;
constexpr u32 SCAN_ITEMS = 4;

__device__ u32 block_exclusive_scan(u32 v, u32 *sm, u32 &total) {
    const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    u32 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (u32)o) x += y;
    }
    if (lane == 31) sm[wid] = x;
    __syncthreads();
    if (wid == 0) {
        u32 s = lane < (blockDim.x >> 5) ? sm[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (u32)o) s += y;
        }
        sm[lane] = s;
    }
    __syncthreads();
    const u32 prefix = (wid > 0 ? sm[wid - 1] : 0) + x - v;
    total = sm[(blockDim.x >> 5) - 1];
    __syncthreads();
    return prefix;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_reduce_kernel(const u32 *in, u64 n, u32 *block_sums) {
    __shared__ u32 sm[32];
    const u64 base = (u64)blockIdx.x * SCAN_BLOCK * SCAN_ITEMS + (u64)threadIdx.x * SCAN_ITEMS;
    u32 s = 0;
    for (u32 k = 0; k < SCAN_ITEMS; k++)
        if (base + k < n) s += in[base + k];
    u32 total;
    block_exclusive_scan(s, sm, total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_blocks_kernel(u32 *block_sums, u32 nblocks) {
    __shared__ u32 sm[32];
    u32 carry = 0;
    for (u32 base = 0; base < nblocks; base += SCAN_BLOCK) {
        const u32 i = base + threadIdx.x;
        const u32 v = i < nblocks ? block_sums[i] : 0;
        u32 total;
        const u32 p = block_exclusive_scan(v, sm, total);
        if (i < nblocks) block_sums[i] = p + carry;
        carry += total;
    }
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_apply_kernel(const u32 *in, u64 n, const u32 *block_sums,
                                                               u32 *out, u32 *out2) {
    __shared__ u32 sm[32];
    const u64 base = (u64)blockIdx.x * SCAN_BLOCK * SCAN_ITEMS + (u64)threadIdx.x * SCAN_ITEMS;
    u32 vals[SCAN_ITEMS];
    u32 s = 0;
    for (u32 k = 0; k < SCAN_ITEMS; k++) {
        vals[k] = base + k < n ? in[base + k] : 0;
        s += vals[k];
    }
    u32 total;
    u32 p = block_exclusive_scan(s, sm, total) + block_sums[blockIdx.x];
    for (u32 k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < n) {
            out[base + k] = p;
            out2[base + k] = p;
        }
        p += vals[k];
    }
}

// ------------------------------------------------------------------ 4: accumulation
ZK_DI G1A fetch_point(const u32 *points, u32 code) {
    const u32 idx = code & 0x7fffffffu;
    G1A p = G1A::load_nc(points + (u64)idx * 16);
    if (code & 0x80000000u) p = p.neg();
    return p;
}

// The sorted array (live entries: *live) is cut into chunks of K; one thread per chunk walks
// it with mixed additions.  A run of one bucket wholly inside the chunk is stored to its
// bucket; a run cut by a chunk edge leaves a partial: part_flag 1 = head run (continued from
// the previous chunk, ends here), 2 = head run that also continues into the next chunk,
// 3 = tail run (starts here, continues into the next).  Buckets of different tasks never
// share a key, so runs never span two tasks.
#ifndef ZK_ACC_MIN_BLOCKS
#define ZK_ACC_MIN_BLOCKS 2  // resident CTAs of 256 threads per SM the register budget targets
#endif
// CODES: the walk reads list 0 (8-byte records: bucket id, point code into the task tables;
// sorted_point = sorted_bucket + 1, stride 2 words); otherwise the last pairing round's list
// (bucket ids, and explicit points at their list positions).
template <bool CODES>
__global__ void __launch_bounds__(256, ZK_ACC_MIN_BLOCKS) accumulate_kernel(const Batch b, const u32 *sorted_bucket,
                                                           const u32 *sorted_point, const u32 *live,
                                                           u32 *bucket_sums, u32 *part_pts, u32 *part_bucket,
                                                           u32 *part_flag, u32 *chain_list, u32 *chain_count) {
    constexpr u32 S = CODES ? 2 : 1;  // words between consecutive bucket ids
    const u64 entries = *live;
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 start = t * b.K;
    if (start >= entries) return;
    const u64 end = start + b.K < entries ? start + b.K : entries;
    const bool from_prev = start > 0 && sorted_bucket[S * (start - 1)] == sorted_bucket[S * start];
    u64 run_start = start;
    u32 cur = sorted_bucket[S * start];
    const u32 *pts = CODES ? b.task[find_task(b.key_first, b.ntasks, (u64)cur)].points : sorted_point;
    G1X acc = G1X::from_affine(CODES ? fetch_point(pts, sorted_point[S * start])
                                     : G1A::load_nc(sorted_point + start * 16));
    // The next record's bucket, code and point address are read one iteration ahead; its point
    // is loaded when it is used.  (Keeping the point load itself one iteration ahead helped
    // while the Fq product was slower; with the paired product the 16 registers it holds cost
    // more: 16.0 vs 15.7 ms at 2^22.)
    u32 nbk = EMPTY, ncode = 0;
    const u32 *npts = pts;
    const u32 *naddr = pts;
    bool chain_start = false;  // a tail partial was written: a chain for the fix-up starts here
    if (start + 1 < end) {
        nbk = sorted_bucket[S * (start + 1)];
        if (CODES) {
            ncode = sorted_point[S * (start + 1)];
            if (nbk != cur) npts = b.task[find_task(b.key_first, b.ntasks, (u64)nbk)].points;
            naddr = npts + (u64)(ncode & 0x7fffffffu) * 16;
        } else {
            naddr = sorted_point + (start + 1) * 16;
        }
    }
    for (u64 p = start + 1; p <= end; p++) {
        const u32 bk = nbk, code = ncode;
        const u32 *bpts = npts;
        G1A pt;
        if (p < end) pt = G1A::load_nc(naddr);
        if (p + 1 < end) {
            nbk = sorted_bucket[S * (p + 1)];
            if (CODES) {
                ncode = sorted_point[S * (p + 1)];
                if (nbk != bk) npts = b.task[find_task(b.key_first, b.ntasks, (u64)nbk)].points;
                naddr = npts + (u64)(ncode & 0x7fffffffu) * 16;
            } else {
                naddr = sorted_point + (p + 1) * 16;
            }
        } else {
            nbk = EMPTY;
        }
        if (CODES && p < end && (code & 0x80000000u)) pt = pt.neg();
        if (p < end && bk == cur) {
            acc = g1_madd(acc, pt);
            continue;
        }
        const bool head = run_start == start && from_prev;
        const bool to_next = p == end && end < entries && sorted_bucket[S * end] == cur;
        if (!head && !to_next) {
            acc.store(bucket_sums + (u64)cur * 32);
        } else {
            const u64 slot = head ? 2 * t : 2 * t + 1;
            acc.store(part_pts + slot * 32);
            part_bucket[slot] = cur;
            part_flag[slot] = head ? (to_next ? 2u : 1u) : 3u;
            chain_start = chain_start || !head;
        }
        if (p < end) {
            cur = bk;
            run_start = p;
            pts = bpts;
            acc = G1X::from_affine(pt);
        }
    }
    // append this chunk to the fix-up's list of chain starts (one atomic per group of lanes
    // that arrive together), so that the fix-up runs dense threads
    const unsigned act = __activemask();
    const unsigned want = __ballot_sync(act, chain_start);
    if (want) {
        const u32 lane = threadIdx.x & 31, leader = __ffs(want) - 1;
        u32 base = 0;
        if (lane == leader) base = atomicAdd(chain_count, (u32)__popc(want));
        base = __shfl_sync(act, base, leader);
        if (chain_start) chain_list[base + __popc(want & ((1u << lane) - 1u))] = (u32)t;
    }
}

// Joins the partial sums of every run that crosses chunk boundaries.  A run's partials sit in
// consecutive chunks: the tail slot of its first chunk t0, then the head slots of the chunks
// after it.  One thread joins a short run; a run longer than SHORT_CHAIN chunks (a huge bucket:
// equal scalars, or a top window with very few bits) is handed to long_chain_kernel, where a
// whole CTA reduces it in parallel.
constexpr u32 SHORT_CHAIN = 32;

ZK_DI bool chain_member(const u32 *part_bucket, const u32 *part_flag, u64 u, u32 bucket) {
    const u32 f = part_flag[2 * u];
    return (f == 1u || f == 2u) && part_bucket[2 * u] == bucket;
}

// One thread per chain start recorded by the walk (chain_list, chain_count entries).
__global__ void __launch_bounds__(256) fixup_kernel(const u32 *live, u32 K, u32 *bucket_sums, const u32 *part_pts,
                                                   const u32 *part_bucket, const u32 *part_flag,
                                                   const u32 *chain_list, const u32 *chain_count, u32 *long_list,
                                                   u32 *long_count) {
    const u64 chunks = ((u64)*live + K - 1) / K;
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *chain_count) return;
    const u64 t = chain_list[i];
    const u64 slot = 2 * t + 1;
    const u32 bucket = part_bucket[slot];
    // a chain longer than SHORT_CHAIN goes to the CTA-wide pass
    const u64 probe = t + 1 + SHORT_CHAIN;
    if (probe < chunks && chain_member(part_bucket, part_flag, probe - 1, bucket) &&
        part_flag[2 * (probe - 1)] == 2u) {
        long_list[atomicAdd(long_count, 1u)] = (u32)t;
        return;
    }
    G1X acc = G1X::load(part_pts + slot * 32);
    for (u64 u = t + 1; u < chunks; u++) {
        if (!chain_member(part_bucket, part_flag, u, bucket)) break;
        acc = g1_add(acc, G1X::load(part_pts + 2 * u * 32));
        if (part_flag[2 * u] == 1u) break;
    }
    acc.store(bucket_sums + (u64)bucket * 32);
}

// one CTA per long chain (looping over the recorded list): strided partial sums, then a tree
__global__ void __launch_bounds__(128) long_chain_kernel(const u32 *live, u32 K, u32 *bucket_sums,
                                                        const u32 *part_pts, const u32 *part_bucket,
                                                        const u32 *part_flag, const u32 *long_list,
                                                        const u32 *long_count) {
    __shared__ u32 sm[128 * 32];
    const u64 chunks = ((u64)*live + K - 1) / K;
    const u32 nlong = *long_count;
    for (u32 item = blockIdx.x; item < nlong; item += gridDim.x) {
        const u64 t0 = long_list[item];
        const u32 bucket = part_bucket[2 * t0 + 1];
        G1X acc = threadIdx.x == 0 ? G1X::load(part_pts + (2 * t0 + 1) * 32) : G1X::identity();
        // members are the contiguous chunks t0+1 .. t1; each thread takes every blockDim-th
        for (u64 u = t0 + 1 + threadIdx.x; u < chunks; u += blockDim.x) {
            if (!chain_member(part_bucket, part_flag, u, bucket)) break;
            // a flag-1 head ends the chain, but threads strided past it stop at the next
            // non-member anyway; a member after an earlier flag-1 end cannot share the bucket id
            // because bucket ids are strictly increasing along the sorted array
            acc = g1_add(acc, G1X::load(part_pts + 2 * u * 32));
        }
        acc.store(sm + threadIdx.x * 32);
        __syncthreads();
        for (u32 stride = blockDim.x / 2; stride > 0; stride >>= 1) {
            if (threadIdx.x < stride) {
                G1X a = G1X::load(sm + threadIdx.x * 32);
                G1X b = G1X::load(sm + (threadIdx.x + stride) * 32);
                g1_add(a, b).store(sm + threadIdx.x * 32);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) G1X::load(sm).store(bucket_sums + (u64)bucket * 32);
        __syncthreads();
    }
}

// ------------------------------------------------------------------ 4a: affine pairing rounds
// Before the XYZZ walk, each round roughly halves every bucket's list: list positions 2k and
// 2k + 1 (pair slot k) holding two points of the same bucket are added in affine coordinates;
// a point whose slot partner belongs to another bucket (at most one at each end of a bucket's
// run) is carried unchanged.  Round r reads list r and writes list r + 1, in which bucket b
// starts at s'_b = sum_{b' < b} m'_b with m'_b = o + ceil((m_b - o) / 2), o = s_b mod 2, and
// the point from position e of bucket b lands at s'_b + (e - s_b + o) / 2.  Slot-major
// indexing (thread t takes slots t, t + T, t + 2T, ...) keeps every list access coalesced.
//
// An affine sum needs one inverse; a round shares one inversion among all its pairs by
// Montgomery's trick: each thread chains the denominators of its pairs (KA / 2 slots), a
// product tree over the thread totals ends in one inversion, and each thread then walks its
// slots backwards, recovering every denominator's inverse with two products.  A pair costs six
// products (three for the trick; the slope, its square, and the new y), against ten for the
// mixed XYZZ addition it replaces.  The bucket sums, and so the result, are the same.

// list r + 1's counts from list r's starts; entry nb is 0 (the scan's total)
__global__ void halve_counts_kernel(const u32 *starts, u64 nb, u32 *cnt) {
    const u64 b = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nb) return;
    u32 m = 0;
    if (b < nb) {
        const u32 s0 = starts[b], mb = starts[b + 1] - s0, o = s0 & 1u;
        m = mb == 0 ? 0u : o + ((mb - o + 1) >> 1);
    }
    cnt[b] = m;
}


// Address of the point at list position e, and its sign code.  CODES: list 0, whose entries
// are 8-byte records (bucket id, point code into the bucket's task tables: index | sign << 31;
// pts = the record array + 1 word); otherwise explicit 64-byte canonical affine points.
template <bool CODES>
ZK_DI const u32 *list_addr(const Batch &b, const u32 *pts, u64 e, u32 bucket, u32 &code) {
    if (CODES) {
        code = pts[2 * e];
        const u32 *tbl = b.task[find_task(b.key_first, b.ntasks, (u64)bucket)].points;
        return tbl + (u64)(code & 0x7fffffffu) * 16;
    }
    code = 0;
    return pts + e * 16;
}
ZK_DI G1A signed_point(const u32 *addr, u32 code) {
    G1A a = G1A::load_nc(addr);
    if (code & 0x80000000u) a.y = neg_canonical(a.y);
    return a;
}

// pair kinds: 0 general (d = x2 - x1), 1 doubling (d = 2 y1), 2 first is the identity (sum =
// second), 3 second is the identity (sum = first), 4 opposite points (sum = identity); kinds
// 2-4 use d = 1.  A point is the identity exactly when y == 0 (canonical); a valid point with
// x != 0 is never the identity, so x1 != x2 with both non-zero decides kind 0 from x alone.
ZK_DI bool general_by_x(const Fq &x1, const Fq &x2) { return !x1.is_zero() && !x2.is_zero() && !(x1 == x2); }
ZK_DI u32 pair_kind(const G1A &a, const G1A &c) {
    if (general_by_x(a.x, c.x)) return 0;
    if (a.y.is_zero()) return 2;
    if (c.y.is_zero()) return 3;
    if (!(a.x == c.x)) return 0;
    return a.y == c.y ? 1u : 4u;
}
ZK_DI Fq pair_den(const G1A &a, const G1A &c, u32 kind) {
    if (kind == 0) return Fq::sub(c.x, a.x);
    if (kind == 1) return Fq::dbl(a.y);
    return Fq::one();
}
ZK_DI G1A pair_sum(const G1A &a, const G1A &c, u32 kind, const Fq &inv) {
    if (kind == 2) return c;
    if (kind == 3) return a;
    G1A r;
    if (kind == 4) {
        r.x = Fq::zero();
        r.y = Fq::zero();
        return r;
    }
    Fq lam;
    if (kind == 0) {
        lam = fmul(Fq::sub(c.y, a.y), inv);
    } else {
        const Fq x2 = fsqr(a.x);
        lam = fmul(Fq::add(Fq::dbl(x2), x2), inv);
    }
    const Fq x3 = Fq::sub(Fq::sub(fsqr(lam), a.x), c.x);
    r.y = Fq::sub(fmul(lam, Fq::sub(a.x, x3)), a.y).canonical();
    r.x = x3.canonical();
    return r;
}

// Up pass: for each of the thread's pair slots that holds a pair, store the product of the
// thread's earlier denominators (slot-major, prefix[k T + t]) and chain this one; tot[t] is
// the product of all of them (1 when the thread has none).
template <bool CODES>
__global__ void __launch_bounds__(256) pair_up_kernel(const Batch b, const u32 *bkt, const u32 *pts,
                                                     const u32 *starts, u64 nb, u64 nthr, u32 *prefix, u32 *tot) {
    constexpr u32 S = CODES ? 2 : 1;  // words between consecutive bucket ids
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nthr) return;
    const u64 E = starts[nb];
    Fq acc = Fq::one();
    for (u32 k = 0; k < KA / 2; k++) {
        const u64 e0 = 2 * (t + (u64)k * nthr);
        if (e0 + 1 >= E) break;
        const u32 b0 = bkt[S * e0];
        if (bkt[S * (e0 + 1)] != b0) continue;
        u32 c0, c1;
        const u32 *a0 = list_addr<CODES>(b, pts, e0, b0, c0);
        const u32 *a1 = list_addr<CODES>(b, pts, e0 + 1, b0, c1);
        const Fq x1 = Fq::load_nc(a0), x2 = Fq::load_nc(a1);
        Fq d;
        if (general_by_x(x1, x2)) {
            d = Fq::sub(x2, x1);
        } else {
            const G1A pa = signed_point(a0, c0), pc = signed_point(a1, c1);
            d = pair_den(pa, pc, pair_kind(pa, pc));
        }
        acc.canonical().store(prefix + ((u64)k * nthr + t) * 8);
        acc = fmul(acc, d);
    }
    acc.canonical().store(tot + t * 8);
}

// Down pass: with inv_tot[t] the inverse of the thread's product, walk the slots backwards
// (d^-1 = acc * prefix, then acc *= d), add the pairs, carry the singles, write list r + 1.
template <bool CODES>
__global__ void __launch_bounds__(256, 3) pair_down_kernel(const Batch b, const u32 *bkt, const u32 *pts,
                                                          const u32 *starts, const u32 *starts_next, u64 nb,
                                                          u64 nthr, const u32 *prefix, const u32 *inv_tot,
                                                          u32 *out_bkt, u32 *out_pts) {
    constexpr u32 S = CODES ? 2 : 1;  // words between consecutive bucket ids
    const u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nthr) return;
    const u64 E = starts[nb];
    Fq acc = Fq::load(inv_tot + t * 8);
    for (u32 k = KA / 2; k-- > 0;) {
        const u64 e0 = 2 * (t + (u64)k * nthr);
        if (e0 >= E) continue;
        const u32 b0 = bkt[S * e0];
        const u32 b1 = e0 + 1 < E ? bkt[S * (e0 + 1)] : EMPTY;
        u32 c0;
        const u32 *a0 = list_addr<CODES>(b, pts, e0, b0, c0);
        G1A r = signed_point(a0, c0);
        if (b1 == b0) {
            u32 c1;
            const u32 *a1 = list_addr<CODES>(b, pts, e0 + 1, b0, c1);
            const G1A c = signed_point(a1, c1);
            const u32 kind = pair_kind(r, c);
            const Fq d = pair_den(r, c, kind);
            const Fq inv = fmul(acc, Fq::load(prefix + ((u64)k * nthr + t) * 8));
            acc = fmul(acc, d);
            r = pair_sum(r, c, kind, inv);
        } else if (b1 != EMPTY) {
            // the slot's second point starts the next bucket: carried on its own
            u32 c1;
            const u32 *a1 = list_addr<CODES>(b, pts, e0 + 1, b1, c1);
            const u32 s1 = starts[b1];
            const u64 q1 = starts_next[b1] + ((e0 + 1 - s1 + (s1 & 1u)) >> 1);
            signed_point(a1, c1).store(out_pts + q1 * 16);
            out_bkt[q1] = b1;
        }
        const u32 s0 = starts[b0];
        const u64 q0 = starts_next[b0] + ((e0 - s0 + (s0 & 1u)) >> 1);
        r.store(out_pts + q0 * 16);
        out_bkt[q0] = b0;
    }
}

// Montgomery's trick over a plain array of non-zero Fq values (the thread totals), in place.
// A CTA takes TREE_SPAN values: thread j folds the values base + j + TREE_CTA k (k <
// TREE_PER) into running prefixes and a product p_j; shared-memory scans give every thread the
// products E_j of the threads before it and S_j of those after it, so p_j^-1 = P^-1 E_j S_j
// with P the CTA's product.  tree_up_kernel hands P to the next level; tree_top_kernel (one
// CTA, at most TREE_SPAN values) inverts its P once and resolves its members; tree_down_kernel
// resolves a level's members from the inverses of its CTA products.

// exclusive product scan over the CTA's threads, forward (reverse = false) or backward
ZK_DI Fq cta_exclusive_product(const Fq &v, u32 *sm, bool reverse) {
    const u32 j = reverse ? TREE_CTA - 1 - threadIdx.x : threadIdx.x;
    Fq x = v;
    for (u32 d = 1; d < TREE_CTA; d <<= 1) {
        x.store(sm + j * 8);
        __syncthreads();
        const Fq y = j >= d ? Fq::load(sm + (j - d) * 8) : Fq::one();
        __syncthreads();
        x = fmul(x, y);
    }
    // x = inclusive product; shift by one
    x.store(sm + j * 8);
    __syncthreads();
    const Fq r = j > 0 ? Fq::load(sm + (j - 1) * 8) : Fq::one();
    __syncthreads();
    return r;
}

// thread's member fold: pre[i] = product of its earlier members, returns the product
ZK_DI Fq tree_fold(const u32 *vals, u64 n, u64 base, u32 *pre) {
    Fq acc = Fq::one();
    for (u32 k = 0; k < TREE_PER; k++) {
        const u64 i = base + threadIdx.x + (u64)k * TREE_CTA;
        if (i >= n) break;
        acc.canonical().store(pre + i * 8);
        acc = fmul(acc, Fq::load(vals + i * 8));
    }
    return acc;
}

// members from the inverse of the thread's product, walking backwards
ZK_DI void tree_resolve(u32 *vals, u64 n, u64 base, const u32 *pre, Fq inv) {
    for (u32 k = TREE_PER; k-- > 0;) {
        const u64 i = base + threadIdx.x + (u64)k * TREE_CTA;
        if (i >= n) continue;
        const Fq v = Fq::load(vals + i * 8);
        fmul(inv, Fq::load(pre + i * 8)).canonical().store(vals + i * 8);
        inv = fmul(inv, v);
    }
}

__global__ void __launch_bounds__(TREE_CTA) tree_up_kernel(const u32 *vals, u64 n, u32 *pre, u32 *ex, u32 *sx,
                                                          u32 *tot) {
    __shared__ __align__(16) u32 sm[TREE_CTA * 8];
    const u64 base = (u64)blockIdx.x * TREE_SPAN;
    const Fq p = tree_fold(vals, n, base, pre);
    const Fq e = cta_exclusive_product(p, sm, false);
    const Fq f = cta_exclusive_product(p, sm, true);
    const u64 slot = (u64)blockIdx.x * TREE_CTA + threadIdx.x;
    e.canonical().store(ex + slot * 8);
    f.canonical().store(sx + slot * 8);
    if (threadIdx.x == TREE_CTA - 1) fmul(e, p).canonical().store(tot + (u64)blockIdx.x * 8);
}

__global__ void __launch_bounds__(TREE_CTA) tree_top_kernel(u32 *vals, u64 n, u32 *pre) {
    __shared__ __align__(16) u32 sm[TREE_CTA * 8];
    const Fq p = tree_fold(vals, n, 0, pre);
    const Fq e = cta_exclusive_product(p, sm, false);
    const Fq f = cta_exclusive_product(p, sm, true);
    if (threadIdx.x == TREE_CTA - 1) inv_binary<FqParams>(fmul(e, p)).store(sm);
    __syncthreads();
    const Fq inv_all = Fq::load(sm);
    tree_resolve(vals, n, 0, pre, fmul(inv_all, fmul(e, f)));
}

__global__ void __launch_bounds__(TREE_CTA) tree_down_kernel(u32 *vals, u64 n, const u32 *pre, const u32 *ex,
                                                            const u32 *sx, const u32 *inv_tot) {
    const u64 base = (u64)blockIdx.x * TREE_SPAN;
    const u64 slot = (u64)blockIdx.x * TREE_CTA + threadIdx.x;
    const Fq inv = fmul(Fq::load(inv_tot + (u64)blockIdx.x * 8), fmul(Fq::load(ex + slot * 8), Fq::load(sx + slot * 8)));
    tree_resolve(vals, n, base, pre, inv);
}

// ------------------------------------------------------------------ 5: bucket reduction
// A physical window's value is sum_j (j + 1) S_j over its B buckets.  With segments of L
// buckets (g < G = B / L), U_g = the segment's sum and T_g = sum_i (i + 1) S_{gL+i}, the value
// is  sum_g T_g + L * sum_g g U_g,  and  sum_g g U_g = sum_k 2^k X_k  with X_k the sum of the
// U_g whose index g has bit k set.  segment_kernel forms U_g and T_g (2L additions per
// thread); class_kernel sums every class (each X_k, and the T_g in two halves) in parallel
// parts; scale_kernel joins each class's parts and scales X_k by 2^k * L with doublings, and
// window_kernel adds the classes.  Every chain of dependent additions stays short, so a window of 2^16 buckets is
// reduced by tens of thousands of threads instead of a few thousand long ones.
__global__ void __launch_bounds__(128) segment_kernel(const Batch b, const u32 *bucket_sums, u32 *seg_u,
                                                     u32 *seg_t) {
    const u64 s = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.seg_first[b.ntasks]) return;
    const u32 t = find_task(b.seg_first, b.ntasks, s);
    const Task &k = b.task[t];
    const u64 sl = s - b.seg_first[t];
    const u32 *base = bucket_sums + (b.key_first[t] + sl * k.L) * 32;
    G1X run = G1X::identity(), acc = G1X::identity();
    for (int j = (int)k.L - 1; j >= 0; j--) {
        run = g1_add(run, G1X::load(base + (u64)j * 32));
        acc = g1_add(acc, run);
    }
    run.store(seg_u + s * 32);
    acc.store(seg_t + s * 32);
}

// sum of the CTA's per-thread points (256 threads) into sm[0]
ZK_DI void cta_tree_sum(u32 *sm, const G1X &mine) {
    mine.store(sm + threadIdx.x * 32);
    __syncthreads();
    for (u32 stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride) {
            G1X x = G1X::load(sm + threadIdx.x * 32);
            G1X y = G1X::load(sm + (threadIdx.x + stride) * 32);
            g1_add(x, y).store(sm + threadIdx.x * 32);
        }
        __syncthreads();
    }
}

// grid (windows, classes, parts): class k < gbits sums U_g over the g with bit k set; classes
// gbits and gbits + 1 sum T_g over the lower and upper half of g.  Each class has G/2 items,
// split into `parts` equal ranges, one CTA each.
__global__ void __launch_bounds__(256) class_kernel(const Batch b, const u32 *seg_u, const u32 *seg_t,
                                                   u32 *cls_out) {
    __shared__ u32 sm[256 * 32];
    const u32 wg = blockIdx.x, cls = blockIdx.y, part = blockIdx.z;
    const u32 t = find_task(b.win_first, b.ntasks, wg);
    const Task &k = b.task[t];
    if (cls >= k.gbits + 2 || part >= k.parts) return;  // the whole CTA leaves together
    const u64 G = k.B / k.L, half = G / 2;
    const u64 seg0 = b.seg_first[t] + (u64)(wg - b.win_first[t]) * G;
    const u64 per = half / k.parts;
    const u64 m0 = (u64)part * per;
    const bool is_t = cls >= k.gbits;
    const u32 *src = is_t ? seg_t : seg_u;
    G1X acc = G1X::identity();
    for (u64 m = m0 + threadIdx.x; m < m0 + per; m += blockDim.x) {
        const u64 g = is_t ? m + (u64)(cls - k.gbits) * half
                           : ((m >> cls) << (cls + 1)) | (1ull << cls) | (m & ((1ull << cls) - 1));
        acc = g1_add(acc, G1X::load(src + (seg0 + g) * 32));
    }
    cta_tree_sum(sm, acc);
    if (threadIdx.x == 0) G1X::load(sm).store(cls_out + (((u64)wg * b.ncls + cls) * b.nparts + part) * 32);
}

// Classes to window values in two launches of single warps, so that the work spreads over as
// many SMs as there are classes.  scale_kernel, one warp per (window, class): one part per lane
// (at most 32 parts, a power of two) summed by a shuffle tree of additions; every lane then
// holds the class sum X_k and the warp scales it by 2^k L with warp-wide doublings (each
// doubling's independent products side by side, g1_dbl_warp), the longest dependent chain of
// the reduction (up to 18 doublings); the result replaces part 0 of the class.  window_kernel,
// one warp per window: one class per lane (at most 32), summed by a shuffle tree.
ZK_DI G1X g1x_shfl_down(const G1X &p, u32 d) {
    G1X r;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        r.x.v[w] = __shfl_down_sync(0xffffffffu, p.x.v[w], d);
        r.y.v[w] = __shfl_down_sync(0xffffffffu, p.y.v[w], d);
        r.zz.v[w] = __shfl_down_sync(0xffffffffu, p.zz.v[w], d);
        r.zzz.v[w] = __shfl_down_sync(0xffffffffu, p.zzz.v[w], d);
    }
    return r;
}
ZK_DI G1X g1x_bcast(const G1X &p, int src) {
    G1X r;
    r.x = lane_bcast(p.x, src);
    r.y = lane_bcast(p.y, src);
    r.zz = lane_bcast(p.zz, src);
    r.zzz = lane_bcast(p.zzz, src);
    return r;
}

// grid (windows, classes), 32 threads
__global__ void __launch_bounds__(32) scale_kernel(const Batch b, u32 *cls_out) {
    const u32 wg = blockIdx.x, cl = blockIdx.y, lane = threadIdx.x;
    const u32 t = find_task(b.win_first, b.ntasks, wg);
    const Task &k = b.task[t];
    if (cl >= k.gbits + 2) return;  // the whole warp leaves together
    const u32 P = k.parts;
    u32 *base = cls_out + ((u64)wg * b.ncls + cl) * b.nparts * 32;
    G1X v = lane < P ? G1X::load(base + (u64)lane * 32) : G1X::identity();
    for (u32 d = P >> 1; d > 0; d >>= 1) v = g1_add(v, g1x_shfl_down(v, d));
    if (cl < k.gbits) {
        v = g1x_bcast(v, 0);
        const u32 dbls = cl + (31 - __clz(k.L));  // 2^cl * L
        for (u32 i = 0; i < dbls; i++) v = g1_dbl_warp(v);
    }
    if (lane == 0) v.store(base);
}

// one warp per physical window: the sum of its classes' scaled values
__global__ void __launch_bounds__(32) window_kernel(const Batch b, const u32 *cls_out, u32 *win_out) {
    const u32 wg = blockIdx.x, lane = threadIdx.x;
    const u32 t = find_task(b.win_first, b.ntasks, wg);
    const Task &k = b.task[t];
    const u32 ncls = k.gbits + 2;
    G1X v = lane < ncls ? G1X::load(cls_out + ((u64)wg * b.ncls + lane) * b.nparts * 32) : G1X::identity();
    const u32 span = 1u << (32 - __clz(ncls - 1));  // ncls >= 2 rounded up to a power of two
    for (u32 d = span >> 1; d > 0; d >>= 1) v = g1_add(v, g1x_shfl_down(v, d));
    if (lane == 0) v.store(win_out + (u64)wg * 32);
}

// ------------------------------------------------------------------ 6: window combination
// one warp per task (one CTA of 32 threads): Horner over the physical windows (c doublings
// each).  Without precomputed tables that is a serial chain of (Wp - 1) c doublings (240 at
// c = 15, 17 windows), so the warp computes each doubling's and addition's independent
// products side by side (g1_dbl_warp / g1_add_warp: 1.2 ms -> 0.4 ms at 2^22); lane 0 then
// normalises to affine.
__global__ void __launch_bounds__(32) combine_kernel(const Batch b, const u32 *win_out) {
    const u32 t = blockIdx.x;
    if (t >= b.ntasks) return;
    const Task &k = b.task[t];
    const u32 *w = win_out + (u64)b.win_first[t] * 32;
    G1X acc = G1X::load(w + (u64)(k.Wp - 1) * 32);
    for (int i = (int)k.Wp - 2; i >= 0; i--) {
        for (u32 d = 0; d < k.c; d++) acc = g1_dbl_warp(acc);
        acc = g1_add_warp(acc, G1X::load(w + (u64)i * 32));
    }
    if (threadIdx.x == 0) g1_to_affine(acc).store(k.result);
}

__global__ void zero_results_kernel(const Batch b) {
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.ntasks || b.task[t].n != 0) return;
    for (int i = 0; i < 16; i++) b.task[t].result[i] = 0;
}

// ------------------------------------------------------------------ precompute tables
// table j = 2^(j * Wp * c) * P, affine (MSMPrecompute::run, msm_impl.cuh:776-800)
__global__ void __launch_bounds__(128) precompute_kernel(const u32 *src, u32 *dst, u64 n, u32 shift_bits) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    G1X p = G1X::from_affine(G1A::load(src + i * 16));
    for (u32 k = 0; k < shift_bits; k++) p = g1_dbl(p);
    g1_to_affine(p).store(dst + i * 16);
}

__global__ void add_points_kernel(u32 *acc_affine, const u32 *other_affine) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    G1X a = G1X::from_affine(G1A::load(acc_affine));
    a = g1_madd(a, G1A::load(other_affine));
    g1_to_affine(a).store(acc_affine);
}

// ------------------------------------------------------------------ driver
inline u32 grid_for(u64 items, u32 block, u32 per_sm = 8) {
    const u64 b = (items + block - 1) / block;
    const u64 cap = (u64)num_sms() * per_sm;
    return (u32)(b < cap ? (b == 0 ? 1 : b) : cap);
}

// Runs a batch of MSMs whose points / scalars are on the device; `ws` holds the layout
// regions.  Launches only: no allocation, no host copy.
// points_ready (optional): the first kernel that reads the points (the first pairing round, or
// the accumulation) waits for it, so a host-to-device copy of the points can overlap the
// digit sort.  scalars_read (optional): recorded once the scalars have
// been read (after the scatter), so the caller may overwrite them.
cudaError_t run_batch(const Batch &b, const Layout &l, char *ws, cudaStream_t stream,
                      cudaEvent_t points_ready = nullptr, cudaEvent_t scalars_read = nullptr) {
    u32 *counts = reinterpret_cast<u32 *>(ws + l.counts);
    u32 *cursor = reinterpret_cast<u32 *>(ws + l.cursor);
    u32 *sb = reinterpret_cast<u32 *>(ws + l.sorted_bucket);
    u32 *sp = reinterpret_cast<u32 *>(ws + l.sorted_point);
    u32 *bs = reinterpret_cast<u32 *>(ws + l.bucket_sums);
    u32 *pp = reinterpret_cast<u32 *>(ws + l.part_pts);
    u32 *pb = reinterpret_cast<u32 *>(ws + l.part_bucket);
    u32 *pf = reinterpret_cast<u32 *>(ws + l.part_flag);
    u32 *longs = reinterpret_cast<u32 *>(ws + l.long_list);
    u32 *nlong = longs + l.chunks + 1;
    u32 *chains = reinterpret_cast<u32 *>(ws + l.chain_list);
    u32 *nchain = chains + l.chunks;
    u32 *seg = reinterpret_cast<u32 *>(ws + l.seg);
    u32 *cls = reinterpret_cast<u32 *>(ws + l.cls);
    u32 *win = reinterpret_cast<u32 *>(ws + l.win);
    const u64 nb = l.nb;
    auto at = [&](size_t off) { return reinterpret_cast<u32 *>(ws + off); };
    // exclusive scan of items counters in[] into out[] (and out2[])
    auto scan = [&](const u32 *in, u64 items, u32 *out, u32 *out2) -> cudaError_t {
        const u32 nblocks = (u32)((items + SCAN_BLOCK * SCAN_ITEMS - 1) / (SCAN_BLOCK * SCAN_ITEMS));
        u32 *block_sums = at(l.scan_sums);
        scan_reduce_kernel<<<nblocks, SCAN_BLOCK, 0, stream>>>(in, items, block_sums);
        scan_blocks_kernel<<<1, SCAN_BLOCK, 0, stream>>>(block_sums, nblocks);
        scan_apply_kernel<<<nblocks, SCAN_BLOCK, 0, stream>>>(in, items, block_sums, out, out2);
        return cudaGetLastError();
    };

    StageProfiler &prof = profiler();
    prof.begin(stream);
    ZK_TRY(cudaMemsetAsync(counts, 0, (nb + 1) * 4, stream));
    ZK_TRY(cudaMemsetAsync(bs, 0, nb * 128, stream));
    ZK_TRY(cudaMemsetAsync(pf, 0, l.chunks * 2 * 4, stream));
    ZK_TRY(cudaMemsetAsync(nlong, 0, 4, stream));
    ZK_TRY(cudaMemsetAsync(nchain, 0, 4, stream));
    prof.mark("memset", stream);
    const u64 scalars = b.sc_first[b.ntasks];
    if (scalars) {
        count_kernel<<<grid_for(scalars, 256), 256, 0, stream>>>(b, counts);
        ZK_TRY(cudaGetLastError());
    }
    prof.mark("count", stream);
    // exclusive scan of the nb + 1 counters: cursor[k] = first slot of bucket k, and
    // counts[nb] becomes the number of live (non-zero digit) entries
    ZK_TRY(scan(counts, nb + 1, cursor, counts));
    prof.mark("scan", stream);
    for (u32 t = 0; t < b.ntasks; t++) {
        const u64 first = b.sc_first[t], last = b.sc_first[t + 1];
        if (last == first) continue;
        scatter_kernel<<<grid_for(last - first, 256), 256, 0, stream>>>(b, cursor, reinterpret_cast<uint2 *>(sb),
                                                                         first, last);
        ZK_TRY(cudaGetLastError());
    }
    prof.mark("scatter", stream);
    if (scalars_read) ZK_TRY(cudaEventRecord(scalars_read, stream));
    if (points_ready) ZK_TRY(cudaStreamWaitEvent(stream, points_ready, 0));
    const u32 *live = counts + nb;
    const u32 *walk_bkt = sb, *walk_pts = sp;
    static const char *const kUp[MAX_ROUNDS] = {"pair_up0", "pair_up1", "pair_up2", "pair_up3"};
    static const char *const kTree[MAX_ROUNDS] = {"pair_tree0", "pair_tree1", "pair_tree2", "pair_tree3"};
    static const char *const kDown[MAX_ROUNDS] = {"pair_down0", "pair_down1", "pair_down2", "pair_down3"};
    for (u32 r = 0; r < l.rounds; r++) {
        // list r + 1's bucket starts
        const u32 *st = at(l.starts[r]);
        u32 *st_next = at(l.starts[r + 1]);
        halve_counts_kernel<<<(u32)((nb + 256) / 256), 256, 0, stream>>>(st, nb, cursor);
        ZK_TRY(cudaGetLastError());
        ZK_TRY(scan(cursor, nb + 1, st_next, st_next));
        // Montgomery's trick over the round's pairs
        const u64 T = l.thr[r];
        const u32 bu = block_for(BLK_PAIR_UP), bd = block_for(BLK_PAIR_DOWN);
        const u32 grid = (u32)((T + bu - 1) / bu), grid_d = (u32)((T + bd - 1) / bd);
        u32 *prefix = at(l.prefix[r]), *tv = at(l.tvals);
        u32 *out_bkt = at(l.lst_bkt[r % 2]), *out_pts = at(l.lst_pts[r % 2]);
        if (r == 0)
            pair_up_kernel<true><<<grid, bu, 0, stream>>>(b, walk_bkt, walk_pts, st, nb, T, prefix, tv);
        else
            pair_up_kernel<false><<<grid, bu, 0, stream>>>(b, walk_bkt, walk_pts, st, nb, T, prefix, tv);
        ZK_TRY(cudaGetLastError());
        prof.mark(kUp[r], stream);
        // batched inverse of the T thread totals (levels as laid out for round 0's count)
        {
            u64 sizes[TREE_LEVELS + 1];
            u32 *dat[TREE_LEVELS + 1];
            u32 L = 0;
            sizes[0] = T;
            dat[0] = tv;
            while (sizes[L] > TREE_SPAN) {
                if (L == TREE_LEVELS) return cudaErrorInvalidValue;  // beyond the laid-out levels
                const u64 ctas = (sizes[L] + TREE_SPAN - 1) / TREE_SPAN;
                tree_up_kernel<<<(u32)ctas, TREE_CTA, 0, stream>>>(dat[L], sizes[L], at(l.tree_pre[L]),
                                                                   at(l.tree_ex[L]), at(l.tree_sx[L]),
                                                                   at(l.tree_dat[L + 1]));
                ZK_TRY(cudaGetLastError());
                dat[L + 1] = at(l.tree_dat[L + 1]);
                sizes[L + 1] = ctas;
                L++;
            }
            tree_top_kernel<<<1, TREE_CTA, 0, stream>>>(dat[L], sizes[L], at(l.tree_pre[L]));
            ZK_TRY(cudaGetLastError());
            for (u32 k = L; k-- > 0;) {
                tree_down_kernel<<<(u32)sizes[k + 1], TREE_CTA, 0, stream>>>(dat[k], sizes[k], at(l.tree_pre[k]),
                                                                             at(l.tree_ex[k]), at(l.tree_sx[k]),
                                                                             dat[k + 1]);
                ZK_TRY(cudaGetLastError());
            }
        }
        prof.mark(kTree[r], stream);
        if (r == 0)
            pair_down_kernel<true><<<grid_d, bd, 0, stream>>>(b, walk_bkt, walk_pts, st, st_next, nb, T, prefix,
                                                              tv, out_bkt, out_pts);
        else
            pair_down_kernel<false><<<grid_d, bd, 0, stream>>>(b, walk_bkt, walk_pts, st, st_next, nb, T, prefix,
                                                               tv, out_bkt, out_pts);
        ZK_TRY(cudaGetLastError());
        prof.mark(kDown[r], stream);
        walk_bkt = out_bkt;
        walk_pts = out_pts;
        live = st_next + nb;
    }
    if (l.chunks) {
        const u32 ba = block_for(BLK_ACCUMULATE);
        const u32 ga = (u32)((l.chunks + ba - 1) / ba);
        if (l.rounds)
            accumulate_kernel<false><<<ga, ba, 0, stream>>>(b, walk_bkt, walk_pts, live, bs, pp, pb, pf, chains,
                                                            nchain);
        else
            accumulate_kernel<true><<<ga, ba, 0, stream>>>(b, sb, sp, live, bs, pp, pb, pf, chains, nchain);
        ZK_TRY(cudaGetLastError());
    }
    prof.mark("accumulate", stream);
    if (l.chunks) {
        fixup_kernel<<<(u32)((l.chunks + 255) / 256), 256, 0, stream>>>(live, b.K, bs, pp, pb, pf, chains, nchain,
                                                                        longs, nlong);
        ZK_TRY(cudaGetLastError());
        long_chain_kernel<<<num_sms() * 2, 128, 0, stream>>>(live, b.K, bs, pp, pb, pf, longs, nlong);
        ZK_TRY(cudaGetLastError());
    }
    prof.mark("fixup", stream);
    if (l.segs) {
        segment_kernel<<<(u32)((l.segs + 127) / 128), 128, 0, stream>>>(b, bs, seg, seg + l.segs * 32);
        ZK_TRY(cudaGetLastError());
    }
    prof.mark("segment", stream);
    if (l.wins) {
        class_kernel<<<dim3((u32)l.wins, b.ncls, b.nparts), 256, 0, stream>>>(b, seg, seg + l.segs * 32, cls);
        ZK_TRY(cudaGetLastError());
        prof.mark("classes", stream);
        scale_kernel<<<dim3((u32)l.wins, b.ncls), 32, 0, stream>>>(b, cls);
        ZK_TRY(cudaGetLastError());
        window_kernel<<<(u32)l.wins, 32, 0, stream>>>(b, cls, win);
        ZK_TRY(cudaGetLastError());
    }
    prof.mark("window_sum", stream);
    combine_kernel<<<b.ntasks, 32, 0, stream>>>(b, win);
    zero_results_kernel<<<(b.ntasks + 31) / 32, 32, 0, stream>>>(b);
    ZK_TRY(cudaGetLastError());
    prof.mark("combine", stream);
    return cudaSuccess;
}

// ------------------------------------------------------------------ library configuration
// The reference builds one libmsm_<curve>_<s>_<target_windows>_<debug>.so per configuration
// (core/src/msm.rs:100-111) with the number of precomputed point tables fixed at compile time
// (msm.cuh:53-69).  This library reads the same fields from its own file name when it is
// installed under such a name, so a caller passes exactly as many tables as it would to the
// reference; under any other name there is one table and the window is chosen per call.
struct LibConfig {
    u32 window = 0;  // 0 = choose per call
    u32 target_windows = 0;
};

inline LibConfig lib_config() {
    static LibConfig cfg;
    static std::once_flag once;
    std::call_once(once, [] {
        Dl_info info;
        if (dladdr(reinterpret_cast<void *>(&lib_config), &info) && info.dli_fname) {
            std::string name(info.dli_fname);
            auto slash = name.find_last_of('/');
            if (slash != std::string::npos) name = name.substr(slash + 1);
            unsigned s = 0, tw = 0;
            char curve[32] = {0}, dbg[16] = {0};
            if (sscanf(name.c_str(), "libmsm_%31[a-z0-9]_%u_%u_%15[a-z]", curve, &s, &tw, dbg) == 4 && s >= 2 &&
                s <= 24 && tw >= 1) {
                cfg.window = s;
                cfg.target_windows = tw;
            }
        }
    });
    return cfg;
}

inline void resolve(u64 n, u32 window, u32 n_tables_hint, u32 *c, u32 *n_tables) {
    LibConfig lc = lib_config();
    u32 cc = window ? window : (lc.window ? lc.window : default_window(n));
    u32 W = (SCALAR_BITS + cc - 1) / cc;
    u32 nt = 1;
    if (n_tables_hint) {
        nt = n_tables_hint;
    } else if (lc.target_windows) {
        u32 nw = W < lc.target_windows ? W : lc.target_windows;
        nt = (W + nw - 1) / nw;
    }
    *c = cc;
    *n_tables = nt;
}

inline Batch single(const u32 *points, u32 n_tables, const u32 *scalars, u64 n, u32 c, u32 *result,
                    int rounds = -1) {
    Batch b{};
    b.ntasks = 1;
    b.task[0] = make_task(n, c, n_tables);
    b.task[0].points = points;
    b.task[0].scalars = scalars;
    b.task[0].result = result;
    finish_batch(b, rounds);
    return b;
}

}  // namespace msm
}  // namespace zk

using namespace zk;

ZK_DEFINE_PROFILER_API(zkp_msm)

// Integer-multiply throughput probe for the roofline denominator: every thread runs `iters`
// rounds of 8 independent 32-bit multiply-add chains (mad.lo), 16 IMAD per round with the
// chains' high halves.  out[tid] keeps the chains live.
__global__ void __launch_bounds__(256) imad_probe_kernel(u32 iters, u32 seed, u32 *out) {
    u32 a[8], b = seed | 1u;
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + threadIdx.x * 8 + k;
    for (u32 i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(b), "r"(a[(k + 1) & 7]));
            asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(b), "r"(a[(k + 3) & 7]));
        }
    }
    u32 s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s ^= a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// launches the probe: blocks x 256 threads x iters x 16 IMAD instructions
extern "C" cudaError_t zkp_imad_probe(unsigned int blocks, unsigned int iters, unsigned int *out_d,
                                      cudaStream_t stream) {
    imad_probe_kernel<<<blocks, 256, 0, stream>>>(iters, 0x9e3779b9u, out_d);
    return cudaGetLastError();
}

// Montgomery-product throughput probe for the field-product roofline: every thread runs two
// independent chains of `iters` Fq products (x = x * y) from values derived from its index.
__global__ void __launch_bounds__(256) mont_probe_kernel(u32 iters, u32 *out) {
    const u32 tid = blockIdx.x * blockDim.x + threadIdx.x;
    Fq x, y, u, v;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        x.v[k] = (tid + 1) * 0x9e3779b9u + k * 0x85ebca6bu;
        y.v[k] = (tid + 7) * 0xc2b2ae35u + k * 0x27d4eb2fu;
        u.v[k] = x.v[k] ^ 0x165667b1u;
        v.v[k] = y.v[k] ^ 0xd3a2646cu;
    }
    x.v[7] &= 0x1fffffffu;  // below the modulus
    y.v[7] &= 0x1fffffffu;
    u.v[7] &= 0x1fffffffu;
    v.v[7] &= 0x1fffffffu;
    for (u32 i = 0; i < iters; i++) {
        x = Fq::mul(x, y);
        u = Fq::mul(u, v);
    }
    Fq::add(x, u).store(out + (u64)tid * 8);
}

// blocks x 256 threads x iters x 2 Fq products; out_d holds blocks * 256 * 8 words
extern "C" cudaError_t zkp_mont_probe(unsigned int blocks, unsigned int iters, unsigned int *out_d,
                                      cudaStream_t stream) {
    mont_probe_kernel<<<blocks, 256, 0, stream>>>(iters, out_d);
    return cudaGetLastError();
}

extern "C" unsigned int zkp_msm_default_window(unsigned long long n) { return msm::default_window(n); }

// pairing rounds an MSM of n points with this window and table count runs under the current
// setting
extern "C" unsigned int zkp_msm_rounds_for(unsigned long long n, unsigned int window, unsigned int n_tables) {
    u32 c, nt;
    msm::resolve(n ? n : 1, window, n_tables, &c, &nt);
    return msm::single(nullptr, nt, nullptr, n, c, nullptr).rounds;
}

// affine pairing rounds for MSMs planned after this call: -1 = by size (the default), else
// 0..4.  Workspace sizes depend on it, so size queries and runs must see the same setting.
extern "C" cudaError_t zkp_msm_set_block(unsigned int stage, unsigned int threads) {
    ZK_CHECK_ARG(stage < msm::BLK_STAGES && (threads == 0 || threads == 64 || threads == 128 || threads == 256));
    msm::block_settings()[stage].store(threads);
    return cudaSuccess;
}

extern "C" cudaError_t zkp_msm_set_affine_rounds(int rounds) {
    ZK_CHECK_ARG(rounds >= -1 && rounds <= (int)msm::MAX_ROUNDS);
    msm::affine_rounds_setting() = rounds;
    return cudaSuccess;
}

extern "C" unsigned long long zkp_msm_workspace_size(unsigned long long n, unsigned int window, unsigned int n_tables) {
    u32 c, nt;
    msm::resolve(n, window, n_tables, &c, &nt);
    return msm::make_layout(msm::single(nullptr, nt, nullptr, n, c, nullptr)).total;
}

extern "C" cudaError_t zkp_msm_device(void *workspace_d, unsigned long long workspace_bytes,
                                      const unsigned int *points_d, unsigned int n_tables,
                                      const unsigned int *scalars_d, unsigned long long n, unsigned int window,
                                      unsigned int *result_d, cudaStream_t stream) {
    ZK_CHECK_ARG(result_d != nullptr);
    if (n == 0) return cudaMemsetAsync(result_d, 0, 64, stream);
    ZK_CHECK_ARG(points_d != nullptr && scalars_d != nullptr && workspace_d != nullptr);
    u32 c, nt;
    msm::resolve(n, window, n_tables, &c, &nt);
    ZK_CHECK_ARG(c >= 2 && c <= 24 && nt >= 1);
    ZK_CHECK_ARG(n * nt < (1ull << 31));
    const msm::Batch b = msm::single(points_d, nt, scalars_d, n, c, result_d);
    ZK_CHECK_ARG(msm::batch_fits(b));
    const msm::Layout l = msm::make_layout(b);
    ZK_CHECK_ARG(workspace_bytes >= l.total);
    return msm::run_batch(b, l, reinterpret_cast<char *>(workspace_d), stream);
}

// batches of more than MAX_TASKS are not split here; the caller chunks them
static cudaError_t build_batch(const ZkpMsmTask *tasks, unsigned int ntasks, msm::Batch *out) {
    ZK_CHECK_ARG(ntasks >= 1 && ntasks <= msm::MAX_TASKS && tasks != nullptr);
    msm::Batch b{};
    b.ntasks = ntasks;
    for (u32 t = 0; t < ntasks; t++) {
        const ZkpMsmTask &k = tasks[t];
        u32 c, nt;
        msm::resolve(k.n ? k.n : 1, k.window, k.n_tables, &c, &nt);
        const u64 stride = k.table_stride ? k.table_stride : k.n;
        ZK_CHECK_ARG(c >= 2 && c <= 24 && nt >= 1 && stride >= k.n && stride * nt < (1ull << 31) && k.result_d != nullptr);
        ZK_CHECK_ARG(k.n == 0 || (k.points_d != nullptr && k.scalars_d != nullptr));
        b.task[t] = msm::make_task(k.n, c, nt);
        b.task[t].stride = stride;
        b.task[t].points = k.points_d;
        b.task[t].scalars = k.scalars_d;
        b.task[t].result = k.result_d;
    }
    msm::finish_batch(b);
    ZK_CHECK_ARG(msm::batch_fits(b));
    *out = b;
    return cudaSuccess;
}

extern "C" unsigned long long zkp_msm_batch_workspace_size(const ZkpMsmTask *tasks, unsigned int ntasks) {
    msm::Batch b;
    if (build_batch(tasks, ntasks, &b) != cudaSuccess) return 0;
    return msm::make_layout(b).total;
}

extern "C" cudaError_t zkp_msm_batch(const ZkpMsmTask *tasks, unsigned int ntasks, void *workspace_d,
                                     unsigned long long workspace_bytes, cudaStream_t stream) {
    msm::Batch b;
    ZK_TRY(build_batch(tasks, ntasks, &b));
    const msm::Layout l = msm::make_layout(b);
    ZK_CHECK_ARG(workspace_d != nullptr && workspace_bytes >= l.total);
    return msm::run_batch(b, l, reinterpret_cast<char *>(workspace_d), stream);
}

extern "C" cudaError_t zkp_msm_precompute_device(unsigned int *tables_d, unsigned long long n, unsigned int window,
                                                 unsigned int n_tables, cudaStream_t stream) {
    ZK_CHECK_ARG(tables_d != nullptr && n_tables >= 1 && window >= 2 && window <= 24);
    const u32 W = (msm::SCALAR_BITS + window - 1) / window;
    const u32 Wp = (W + n_tables - 1) / n_tables;
    for (u32 j = 1; j < n_tables; j++) {
        msm::precompute_kernel<<<(u32)((n + 127) / 128), 128, 0, stream>>>(tables_d + (j - 1) * n * 16,
                                                                           tables_d + j * n * 16, n, Wp * window);
        ZK_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

// device layout of one card's buffer for the reference ABI: points | scalars | result | batch ws
// A card's buffer: the point tables, two scalar buffers (batch b uses buffer b % 2, so the next
// batch's copy overlaps this batch's work), the result and the MSM workspace.
struct CardLayout {
    size_t points, scalars[2], result, ws, total;
    msm::Batch batch[2];
    msm::Layout l;
};

static CardLayout card_layout(u64 cnt, u32 c, u32 nt, char *base) {
    CardLayout cl{};
    size_t off = 0;
    cl.points = off;
    off += msm::align_up(cnt * nt * 64);
    for (int i = 0; i < 2; i++) {
        cl.scalars[i] = off;
        off += msm::align_up(cnt * 32);
    }
    cl.result = off;
    off += 256;
    cl.ws = off;
    u32 *pts = base ? reinterpret_cast<u32 *>(base + cl.points) : nullptr;
    u32 *res = base ? reinterpret_cast<u32 *>(base + cl.result) : nullptr;
    for (int i = 0; i < 2; i++) {
        u32 *sc = base ? reinterpret_cast<u32 *>(base + cl.scalars[i]) : nullptr;
        cl.batch[i] = msm::single(pts, nt, sc, cnt, c, res);
    }
    cl.l = msm::make_layout(cl.batch[0]);
    cl.total = off + cl.l.total;
    return cl;
}

extern "C" cudaError_t msm(void *const *buffers, unsigned long *buffer_sizes, unsigned long long len,
                           unsigned int batch_per_run, unsigned int parts, unsigned int stage_scalers,
                           unsigned int stage_points, unsigned int num_cards, const unsigned int *cards,
                           unsigned int const *const *h_points, unsigned int batches,
                           unsigned int const *const *h_scaler_batch, unsigned int *const *h_result) {
    (void)batch_per_run;
    (void)parts;
    (void)stage_scalers;
    (void)stage_points;
    ZK_CHECK_ARG(num_cards >= 1 && cards != nullptr && len > 0);
    u32 c, nt;
    msm::resolve(len / num_cards + 1, 0, 0, &c, &nt);
    {
        const u64 per_card = len / num_cards + 1;  // 32-bit record positions and point codes
        ZK_CHECK_ARG(per_card * ((msm::SCALAR_BITS + c - 1) / c) < (1ull << 32) - 1 && per_card * nt < (1ull << 31));
    }
    // card k takes points [k*len/num_cards, (k+1)*len/num_cards)
    auto slice = [&](u32 k, u64 *lo, u64 *cnt) {
        *lo = len * k / num_cards;
        *cnt = len * (k + 1) / num_cards - *lo;
    };
    if (buffers == nullptr) {
        ZK_CHECK_ARG(buffer_sizes != nullptr);
        for (u32 k = 0; k < num_cards; k++) {
            u64 lo, cnt;
            slice(k, &lo, &cnt);
            buffer_sizes[k] = card_layout(cnt ? cnt : 1, c, nt, nullptr).total;
        }
        return cudaSuccess;
    }
    ZK_CHECK_ARG(h_points != nullptr && (batches == 0 || (h_scaler_batch != nullptr && h_result != nullptr)));
    int prev_dev = 0;
    ZK_TRY(cudaGetDevice(&prev_dev));
    std::vector<std::vector<u32>> partial(num_cards, std::vector<u32>((size_t)batches * 16, 0));
    cudaError_t err = cudaSuccess;
    for (u32 k = 0; k < num_cards && err == cudaSuccess; k++) {
        u64 lo, cnt;
        slice(k, &lo, &cnt);
        if (cnt == 0) continue;
        err = cudaSetDevice((int)cards[k]);
        if (err != cudaSuccess) break;
        char *base = reinterpret_cast<char *>(buffers[k]);
        CardLayout cl = card_layout(cnt, c, nt, base);
        u32 *d_points = reinterpret_cast<u32 *>(base + cl.points);
        u32 *d_result = reinterpret_cast<u32 *>(base + cl.result);
        // Copies run on their own stream in the order scalars 0, points, scalars 1, 2, ...; the
        // compute stream sorts batch 0's digits while the points arrive, and batch b + 1's
        // scalars arrive while batch b is accumulated.
        cudaStream_t st = cudaStreamPerThread, cs = nullptr;
        cudaEvent_t pts_ready = nullptr, copied[2] = {nullptr, nullptr}, read[2] = {nullptr, nullptr};
        err = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&pts_ready, cudaEventDisableTiming);
        for (int i = 0; i < 2 && err == cudaSuccess; i++) {
            err = cudaEventCreateWithFlags(&copied[i], cudaEventDisableTiming);
            if (err == cudaSuccess) err = cudaEventCreateWithFlags(&read[i], cudaEventDisableTiming);
        }
        // the copy stream starts after any work the caller queued on the compute stream
        if (err == cudaSuccess) err = cudaEventRecord(read[0], st);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(cs, read[0], 0);
        auto copy_scalars = [&](u32 b) {
            const int i = b & 1;
            cudaError_t e = cudaSuccess;
            if (b >= 2) e = cudaStreamWaitEvent(cs, read[i], 0);  // batch b - 2 is done with the buffer
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(base + cl.scalars[i], h_scaler_batch[b] + lo * 8, cnt * 32,
                                    cudaMemcpyHostToDevice, cs);
            if (e == cudaSuccess) e = cudaEventRecord(copied[i], cs);
            return e;
        };
        if (batches > 0 && err == cudaSuccess) err = copy_scalars(0);
        for (u32 j = 0; j < nt && err == cudaSuccess; j++)
            err = cudaMemcpyAsync(d_points + j * cnt * 16, h_points[j] + lo * 16, cnt * 64, cudaMemcpyHostToDevice, cs);
        if (err == cudaSuccess) err = cudaEventRecord(pts_ready, cs);
        for (u32 b = 1; b < batches && b < 2 && err == cudaSuccess; b++) err = copy_scalars(b);
        for (u32 b = 0; b < batches && err == cudaSuccess; b++) {
            const int i = b & 1;
            err = cudaStreamWaitEvent(st, copied[i], 0);
            if (err == cudaSuccess)
                err = msm::run_batch(cl.batch[i], cl.l, base + cl.ws, st, b == 0 ? pts_ready : nullptr, read[i]);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(partial[k].data() + b * 16, d_result, 64, cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess && b + 2 < batches) err = copy_scalars(b + 2);
        }
        if (batches == 0 && err == cudaSuccess) err = cudaStreamWaitEvent(st, pts_ready, 0);
        if (err == cudaSuccess) err = cudaStreamSynchronize(st);
        if (cs) {
            cudaStreamSynchronize(cs);
            cudaStreamDestroy(cs);
        }
        if (pts_ready) cudaEventDestroy(pts_ready);
        for (int i = 0; i < 2; i++) {
            if (copied[i]) cudaEventDestroy(copied[i]);
            if (read[i]) cudaEventDestroy(read[i]);
        }
    }
    // add the other cards' affine partials on the first card (msm_impl.cuh:902-907 does this
    // on the host; here it is one device addition per card)
    if (err == cudaSuccess && num_cards > 1) {
        err = cudaSetDevice((int)cards[0]);
        u64 lo0, cnt0;
        slice(0, &lo0, &cnt0);
        char *base0 = reinterpret_cast<char *>(buffers[0]);
        CardLayout cl0 = card_layout(cnt0 ? cnt0 : 1, c, nt, base0);
        u32 *acc = reinterpret_cast<u32 *>(base0 + cl0.result);
        u32 *other = acc + 16;  // the 256-byte result slot holds a second point
        for (u32 b = 0; b < batches && err == cudaSuccess; b++) {
            err = cudaMemcpy(acc, partial[0].data() + b * 16, 64, cudaMemcpyHostToDevice);
            for (u32 k = 1; k < num_cards && err == cudaSuccess; k++) {
                err = cudaMemcpy(other, partial[k].data() + b * 16, 64, cudaMemcpyHostToDevice);
                if (err == cudaSuccess) {
                    msm::add_points_kernel<<<1, 32>>>(acc, other);
                    err = cudaGetLastError();
                }
            }
            if (err == cudaSuccess) err = cudaMemcpy(partial[0].data() + b * 16, acc, 64, cudaMemcpyDeviceToHost);
        }
    }
    if (err == cudaSuccess)
        for (u32 b = 0; b < batches; b++) memcpy(h_result[b], partial[0].data() + b * 16, 64);
    cudaSetDevice(prev_dev);
    return err;
}

extern "C" cudaError_t msm_precompute(unsigned long long len, unsigned int *const *h_points, unsigned int max_cards) {
    (void)max_cards;
    u32 c, nt;
    msm::resolve(len, 0, 0, &c, &nt);
    if (nt <= 1) return cudaSuccess;
    ZK_CHECK_ARG(h_points != nullptr && len > 0);
    u32 *d = nullptr;
    ZK_TRY(cudaMalloc(&d, (size_t)len * nt * 64));
    cudaError_t err = cudaMemcpy(d, h_points[0], len * 64, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = zkp_msm_precompute_device(d, len, c, nt, 0);
    for (u32 j = 1; j < nt && err == cudaSuccess; j++)
        err = cudaMemcpy(h_points[j], d + (u64)j * len * 16, len * 64, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return err;
}

// ------------------------------------------------------------------ allocation-free entry
// Some callers cannot allocate device memory: a plugin whose host application hands it only
// input and output buffers and owns every allocator, or a serving loop that must never call
// cudaMalloc because it synchronises the whole device.  For them zkp_msm_device_noalloc runs
// the same MSM with its workspace in this fixed array instead of a caller buffer.  The array
// lives in the library image, so every GPU that loads the library holds it until the process
// exits.
static constexpr unsigned long long kNoAllocScratchBytes = 64ull << 20;  // 64 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host code must not use `g_noalloc_scratch` as a device address (on the host it names a
// stand-in).  The array's real address belongs to a CUDA context, not to a device: a host that
// makes its own driver-API context current, or a cudaDeviceReset, brings a new context with its
// own copy of the array.  So the address is looked up with the calling context current and
// cached under that context's unique id (cuCtxGetId ids are never reused within a process).
using CtxGetCurrentFn = int (*)(void **ctx);
using CtxGetIdFn = int (*)(void *ctx, unsigned long long *id);

struct NoAllocEntry {
    unsigned long long ctx_id;
    void *ptr;
};
static std::mutex g_noalloc_mu;
static NoAllocEntry g_noalloc_cache[64];
static unsigned g_noalloc_used = 0, g_noalloc_next = 0;

static cudaError_t current_context_id(unsigned long long *id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    if (!get_current || !get_id) return cudaErrorNotSupported;
    void *ctx = nullptr;
    if (get_current(&ctx) != 0) return cudaErrorDeviceUninitialized;
    if (!ctx) {
        // no context current yet on this thread: the runtime's own rule applies, the current
        // device's primary context (cudaSetDevice initialises it and makes it current)
        int dev = 0;
        ZK_TRY(cudaGetDevice(&dev));
        ZK_TRY(cudaSetDevice(dev));
        if (get_current(&ctx) != 0 || !ctx) return cudaErrorDeviceUninitialized;
    }
    if (get_id(ctx, id) != 0) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}

static cudaError_t noalloc_scratch(cudaStream_t stream, void **out) {
    unsigned long long id = 0;
    ZK_TRY(current_context_id(&id));
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    for (unsigned i = 0; i < g_noalloc_used; i++)
        if (g_noalloc_cache[i].ctx_id == id) {
            *out = g_noalloc_cache[i].ptr;
            return cudaSuccess;
        }
    // first call in this context: the lookup is not a stream operation, so it is not made
    // while the stream is being captured into a graph
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    ZK_TRY(cudaStreamIsCapturing(stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) return cudaErrorStreamCaptureUnsupported;
    void *p = nullptr;
    ZK_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    // a full cache (64 live contexts) replaces its entries in turn
    unsigned slot = g_noalloc_used < 64 ? g_noalloc_used++ : (g_noalloc_next++ % 64);
    g_noalloc_cache[slot] = {id, p};
    *out = p;
    return cudaSuccess;
}

extern "C" unsigned long long zkp_msm_noalloc_capacity(void) { return kNoAllocScratchBytes; }

extern "C" cudaError_t zkp_msm_device_noalloc(const unsigned int *points_d, unsigned int n_tables,
                                              const unsigned int *scalars_d, unsigned long long n,
                                              unsigned int window, unsigned int *result_d, cudaStream_t stream) {
    ZK_CHECK_ARG(result_d != nullptr);
    if (n == 0) return cudaMemsetAsync(result_d, 0, 64, stream);
    ZK_CHECK_ARG(points_d != nullptr && scalars_d != nullptr);
    u32 c, nt;
    msm::resolve(n, window, n_tables, &c, &nt);
    ZK_CHECK_ARG(c >= 2 && c <= 24 && nt >= 1);
    ZK_CHECK_ARG(n * nt < (1ull << 31));
    // no pairing rounds: their lists would not fit the fixed scratch
    const msm::Batch b = msm::single(points_d, nt, scalars_d, n, c, result_d, 0);
    ZK_CHECK_ARG(msm::batch_fits(b));
    const msm::Layout l = msm::make_layout(b);
    // larger problems do not fit the fixed scratch: refuse instead of overrunning it
    if (l.total > kNoAllocScratchBytes) return cudaErrorInvalidValue;
    void *scratch = nullptr;
    ZK_TRY(noalloc_scratch(stream, &scratch));
    return msm::run_batch(b, l, reinterpret_cast<char *>(scratch), stream);
}
