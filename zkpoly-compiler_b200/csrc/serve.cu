// libzkp_runtime.so: continuous-batching request loop for prover-shaped programs (one GPU).
//
// Host-side structure (the reference's scheduler, scheduler/src/scheduler.rs:255-426, admits
// whole programs by CPU-memory "versions" and runs one card per request; here admission is by
// planned HBM footprint and requests share the GPU):
//   - Arena: one device allocation carved by a first-fit free list with coalescing (the
//     device-resident memory pool); a request's buffers are one contiguous block.
//   - Scheduler thread: pops pending requests in arrival order while a slot (stream) is free
//     and the request's footprint fits in the arena (with a short look-ahead so a small request
//     can pass a large one that is waiting for memory), launches the program asynchronously on
//     the slot's stream, records an event, and polls the events of running requests; on
//     completion it copies the tiny results, frees the block and wakes waiters.
//   - Device work of different requests overlaps because every request has its own stream;
//     nothing inside a program synchronises the host.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/msm.h"
#include "../../include/ntt.h"
#include "../../include/poly.h"
#include "../../include/zkp_gen.h"
#include "../../include/zkp_runtime.h"
#include "host_field.h"

namespace {

using u32 = uint32_t;
using u64 = uint64_t;

inline size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

// ------------------------------------------------------------------ device arena
class Arena {
   public:
    cudaError_t init(size_t bytes) {
        size_ = al(bytes);
        cudaError_t e = cudaMalloc(&base_, size_);
        if (e != cudaSuccess) return e;
        free_[0] = size_;
        return cudaSuccess;
    }
    ~Arena() {
        if (base_) cudaFree(base_);
    }
    // first fit; returns offset or SIZE_MAX
    size_t alloc(size_t bytes) {
        bytes = al(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                size_t off = it->first, sz = it->second;
                free_.erase(it);
                if (sz > bytes) free_[off + bytes] = sz - bytes;
                used_ += bytes;
                peak_ = std::max(peak_, used_);
                return off;
            }
        }
        return SIZE_MAX;
    }
    void release(size_t off, size_t bytes) {
        bytes = al(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    char *ptr(size_t off) const { return reinterpret_cast<char *>(base_) + off; }
    size_t size() const { return size_; }
    size_t peak() const { return peak_; }

   private:
    void *base_ = nullptr;
    size_t size_ = 0, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;
};

// per-size constants resident for the server's lifetime
struct SizeConsts {
    u32 *inv_tw = nullptr;   // inverse roots, 2^(k-1) entries
    u32 *fwd_tw = nullptr;   // forward roots of the extended size, 2^(k+ext-1) entries
    u32 *inv_sh = nullptr;   // Shoup tables of the two (16 words per root)
    u32 *fwd_sh = nullptr;
    u32 *ninv = nullptr;     // n^-1
    u32 *zh_inv = nullptr;   // 2^ext values of 1/Z_H on the coset
};

// buffer plan of one request (offsets inside its arena block)
struct Plan {
    size_t a, b, c, z, e, q, x, args, results, msm_ws, eval_tmp0, eval_tmp1, total;
    unsigned long msm_ws_bytes, eval_bytes;
};

struct Request {
    long long ticket;
    ZkpProverRequest req;
    ZkpProverResult res;
    size_t off = SIZE_MAX, bytes = 0;
    int slot = -1;
    bool done = false;
    cudaStream_t stream = nullptr;  // the slot's stream of the request's priority class
    bool large = false;             // counted against the policy's large-request limit
    // a request of a compiled program (null for the built-in prover program)
    const ZkpProgram *prog = nullptr;
    std::vector<const void *> inputs;
    void *results = nullptr;
};

using FusedFn = cudaError_t (*)(const ConstPolyPtr *, const PolyPtr *, unsigned long long, bool, void *, cudaStream_t);

}  // namespace

struct ZkpProgram {
    std::vector<ZkpProgOp> ops;
    u64 device_bytes = 0, host_bytes = 0, result_extent = 0;
    std::vector<ZkpProgOut> outs;
    std::vector<u64> input_bytes;
    long long live = 0;     // requests submitted and not yet completed (under the server mutex)
    bool orphaned = false;  // destroyed while requests were live: freed by the last one
};

struct ZkpServer {
    ZkpServeConfig cfg{};
    int device = 0;
    std::vector<ZkpServeTableSet> sets;  // by ascending max_k

    const ZkpServeTableSet &set_for(u32 k) const {
        for (const auto &t : sets)
            if (k <= t.max_k) return t;
        return sets.back();
    }
    Arena arena;
    std::vector<SizeConsts> consts;  // index k
    u32 *shift = nullptr;            // coset shift 7 (Montgomery)
    void *fused_lib = nullptr;
    FusedFn fused = nullptr;

    struct Slot {
        cudaStream_t stream = nullptr;     // normal priority
        cudaStream_t stream_hi = nullptr;  // high priority (requests of at least priority_bytes)
        cudaEvent_t done = nullptr;
        u32 *host = nullptr;    // pinned: results (4*16 + 2*8 words) + PolyPtr staging
        char *prog_host = nullptr;  // pinned host block of compiled-program requests
        size_t prog_host_bytes = 0;
        Request *req = nullptr;
    };
    std::vector<Slot> slots;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;
    std::unordered_map<long long, Request *> all;
    long long next_ticket = 0;
    bool stop = false;
    std::thread worker;
    std::chrono::steady_clock::time_point t0;
    ZkpServeStats stats{};
    u64 inflight = 0;
    ZkpServePolicy policy{};  // priorities and the large-request limit (all 0: off)
    u64 large_inflight = 0;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

PolyPtr pp(u32 *p, u64 len) { return PolyPtr{p, len, 0, 0, len}; }
ConstPolyPtr cp(const u32 *p, u64 len, u64 rotate = 0) { return ConstPolyPtr{p, len, rotate, 0, len}; }

bool plan_request(ZkpServer *s, u32 k, Plan *p) {
    const u64 n = 1ull << k, N = 1ull << (k + s->cfg.ext_log);
    size_t off = 0;
    auto take = [&](size_t b) {
        size_t o = off;
        off += al(b);
        return o;
    };
    p->a = take(n * 32);
    p->b = take(n * 32);
    p->c = take(n * 32);
    p->z = take(N * 32);
    p->e = take(N * 32);
    p->q = take(N * 32);
    p->x = take(32);
    p->args = take(8 * sizeof(PolyPtr));
    p->results = take(4 * 64 + 2 * 32);
    ZkpMsmTask t[4];
    const ZkpServeTableSet &ts = s->set_for(k);
    for (int i = 0; i < 4; i++)
        t[i] = ZkpMsmTask{ts.tables_d, ts.n_tables, ts.tables_d /*sizes only*/, n, ts.window,
                          reinterpret_cast<u32 *>(16), ts.rows};
    p->msm_ws_bytes = (unsigned long)zkp_msm_batch_workspace_size(t, 4);
    if (p->msm_ws_bytes == 0) return false;
    p->msm_ws = take(p->msm_ws_bytes);
    unsigned long ev = 0;
    if (poly_eval(nullptr, &ev, cp(nullptr, n), nullptr, nullptr, nullptr) != cudaSuccess) return false;
    p->eval_bytes = ev;
    p->eval_tmp0 = take(ev);
    p->eval_tmp1 = take(ev);
    p->total = off;
    return true;
}

// the program of one request, launched asynchronously on `st`
cudaError_t launch_program(ZkpServer *s, Request *r, ZkpServer::Slot &slot) {
    const u32 k = r->req.k, ext = s->cfg.ext_log;
    const u64 n = 1ull << k, N = 1ull << (k + ext);
    Plan p;
    plan_request(s, k, &p);
    char *base = s->arena.ptr(r->off);
    auto P = [&](size_t off) { return reinterpret_cast<u32 *>(base + off); };
    cudaStream_t st = r->stream;
    const SizeConsts &sc = s->consts[k];
    const u64 seed = r->req.seed * 8;
#define RUN(x)                                   \
    do {                                         \
        cudaError_t e__ = (x);                   \
        if (e__ != cudaSuccess) return e__;      \
    } while (0)
    if (r->req.inject_fault == 2) return cudaErrorLaunchFailure;  // host-side injected failure
    // inputs (seeded, generated on the device)
    RUN(zkp_gen_fr(seed + 0, 0, n, P(p.a), st));
    RUN(zkp_gen_fr(seed + 1, 0, n, P(p.b), st));
    RUN(zkp_gen_fr(seed + 2, 0, n, P(p.c), st));
    RUN(zkp_gen_fr(seed + 3, 0, N, P(p.z), st));
    RUN(zkp_gen_fr(seed + 4, 0, 1, P(p.x), st));
    // three INTTs (n^-1 fused into the last pass)
    RUN(zkp_ntt_ex_shoup(pp(P(p.a), n), sc.inv_tw, sc.inv_sh, k, nullptr, sc.ninv, st));
    RUN(zkp_ntt_ex_shoup(pp(P(p.b), n), sc.inv_tw, sc.inv_sh, k, nullptr, sc.ninv, st));
    RUN(zkp_ntt_ex_shoup(pp(P(p.c), n), sc.inv_tw, sc.inv_sh, k, nullptr, sc.ninv, st));
    // coset NTT of c on the extended domain
    RUN(zkp_coset_lde_shoup(pp(P(p.e), N), cp(P(p.c), n), sc.fwd_tw, sc.fwd_sh, k, k + ext, s->shift, st));
    // fused quotient: vars = [e, e, e, z, z(wX), zh_inv], mut = [q]
    PolyPtr *stage = reinterpret_cast<PolyPtr *>(slot.host + 96);
    stage[0] = pp(P(p.e), N);
    stage[1] = pp(P(p.e), N);
    stage[2] = pp(P(p.e), N);
    stage[3] = pp(P(p.z), N);
    stage[4] = PolyPtr{P(p.z), N, N - (1ull << ext), 0, N};  // element i = z[(i + 2^ext) mod N]
    stage[5] = PolyPtr{sc.zh_inv, 1ull << ext, 0, 0, 1ull << ext};
    stage[6] = pp(P(p.q), N);
    RUN(cudaMemcpyAsync(P(p.args), stage, 7 * sizeof(PolyPtr), cudaMemcpyHostToDevice, st));
    const PolyPtr *dargs = reinterpret_cast<const PolyPtr *>(P(p.args));
    RUN(s->fused(reinterpret_cast<const ConstPolyPtr *>(dargs), dargs + 6, N, true, nullptr, st));
    // four MSMs over the resident bases of this size's table set in one batched launch set
    const ZkpServeTableSet &ts = s->set_for(k);
    const u32 nt = ts.n_tables, w = ts.window;
    ZkpMsmTask t[4] = {
        {ts.tables_d, nt, P(p.a), n, w, P(p.results) + 0, ts.rows},
        {ts.tables_d, nt, P(p.b), n, w, P(p.results) + 16, ts.rows},
        {ts.tables_d, nt, P(p.c), n, w, P(p.results) + 32, ts.rows},
        {ts.tables_d, nt, P(p.q), n, w, P(p.results) + 48, ts.rows},
    };
    RUN(zkp_msm_batch(t, 4, P(p.msm_ws), p.msm_ws_bytes, st));
    // two evaluations
    unsigned long eb = p.eval_bytes;
    RUN(poly_eval(P(p.eval_tmp0), &eb, cp(P(p.a), n), P(p.results) + 64, P(p.x), st));
    RUN(poly_eval(P(p.eval_tmp1), &eb, cp(P(p.b), n), P(p.results) + 72, P(p.x), st));
    RUN(cudaMemcpyAsync(slot.host, P(p.results), 4 * 64 + 2 * 32, cudaMemcpyDeviceToHost, st));
    RUN(cudaEventRecord(slot.done, st));
#undef RUN
    return cudaSuccess;
}

// ------------------------------------------------------------------ compiled programs
// Element size of view j of an op: buffers (temps, workspaces, argument buffers) count bytes,
// MSM results and COPY / ZERO of points 64 bytes, everything else a 32-byte field element.
u64 view_elem_bytes(const ZkpProgOp &op, u32 j) {
    switch (op.kind) {
        case ZKP_OP_COPY:
        case ZKP_OP_ZERO:
            return op.imm[0];
        case ZKP_OP_FUSED:
            return j >= 14 ? 1 : 32;
        case ZKP_OP_MSM:
            if (j == 15) return 1;
            return j >= op.imm[3] ? 64 : 32;
        case ZKP_OP_EVAL:
        case ZKP_OP_INVERT:
        case ZKP_OP_KATE:
        case ZKP_OP_SCAN:
            return j == 0 ? 1 : 32;
        default:
            return 32;
    }
}

bool view_well_formed(const ZkpProgView &v) {
    if (v.len == 0 && v.whole_len == 0) return true;
    return v.whole_len >= v.len && v.whole_len > 0 && v.offset < v.whole_len && v.rotate < v.whole_len;
}

// the op's views that must be present (kind-specific count)
u32 required_views(const ZkpProgOp &op) {
    switch (op.kind) {
        case ZKP_OP_COPY: return 2;
        case ZKP_OP_ZERO: return 1;
        case ZKP_OP_NTT: return 2;
        case ZKP_OP_NTT_RECOMPUTE: return 3;
        case ZKP_OP_DISTRIBUTE: return 2;
        case ZKP_OP_FUSED: return (u32)(op.imm[1] + op.imm[2]);
        case ZKP_OP_MSM: return (u32)(2 * op.imm[3]);
        case ZKP_OP_EVAL: return 4;
        case ZKP_OP_INVERT: return 2;
        case ZKP_OP_KATE: return 4;
        case ZKP_OP_SCAN: return 2;
        case ZKP_OP_ADD:
        case ZKP_OP_SUB: return 3;
        case ZKP_OP_ZERO_POLY:
        case ZKP_OP_ONE_LAGRANGE:
        case ZKP_OP_ONE_COEF:
        case ZKP_OP_SCALAR_INV:
        case ZKP_OP_SCALAR_POW: return 1;
        default: return ~0u;
    }
}

// a resolved view: element i at base + phys(i) * eb
struct RView {
    char *base;
    u64 len, start, whole;  // start = (offset - rotate) mod whole
    u64 phys(u64 i) const {
        const u64 p = start + i;
        return p >= whole ? p - whole : p;
    }
    PolyPtr poly() const {
        // PolyPtr with the same element order: a rotation becomes an offset on the whole array
        return PolyPtr{reinterpret_cast<u32 *>(base), len, 0, whole ? start : 0, whole ? whole : len};
    }
    ConstPolyPtr cpoly() const {
        return ConstPolyPtr{reinterpret_cast<const u32 *>(base), len, 0, whole ? start : 0, whole ? whole : len};
    }
    u32 *ptr() const { return reinterpret_cast<u32 *>(base); }
};

RView resolve(ZkpServer *s, const Request *r, const ZkpServer::Slot &slot, const ZkpProgView &v) {
    char *base = nullptr;
    switch (v.space) {
        case ZKP_SPACE_DEVICE: base = s->arena.ptr(r->off) + v.addr; break;
        case ZKP_SPACE_HOST: base = slot.prog_host + v.addr; break;
        case ZKP_SPACE_ABS: base = reinterpret_cast<char *>(v.addr); break;
        case ZKP_SPACE_INPUT: base = const_cast<char *>(static_cast<const char *>(r->inputs[v.index])) + v.addr; break;
        default: break;
    }
    RView out{base, v.len, 0, v.whole_len};
    if (v.whole_len) out.start = (v.offset + v.whole_len - v.rotate % v.whole_len) % v.whole_len;
    return out;
}

// element-order copy dst[i] <- src[i], i < len, split where either view wraps (at most 4
// copies; any direction: the addresses are unified)
cudaError_t copy_views(const RView &dst, const RView &src, u64 len, u64 eb, cudaStream_t st) {
    for (u64 i = 0; i < len;) {
        const u64 sp = src.phys(i), dp = dst.phys(i);
        const u64 seg = std::min(len - i, std::min(src.whole - sp, dst.whole - dp));
        cudaError_t e = cudaMemcpyAsync(dst.base + dp * eb, src.base + sp * eb, seg * eb, cudaMemcpyDefault, st);
        if (e != cudaSuccess) return e;
        i += seg;
    }
    return cudaSuccess;
}

cudaError_t zero_view(const RView &dst, u64 eb, cudaStream_t st) {
    for (u64 i = 0; i < dst.len;) {
        const u64 dp = dst.phys(i);
        const u64 seg = std::min(dst.len - i, dst.whole - dp);
        cudaError_t e = cudaMemsetAsync(dst.base + dp * eb, 0, seg * eb, st);
        if (e != cudaSuccess) return e;
        i += seg;
    }
    return cudaSuccess;
}

inline u32 log2_exact(u64 n) {
    u32 l = 0;
    while ((1ull << l) < n) l++;
    return l;
}

// runs the ops of a compiled program in order on the request's stream
cudaError_t launch_compiled(ZkpServer *s, Request *r, ZkpServer::Slot &slot) {
    cudaStream_t st = r->stream;
    if (r->req.inject_fault == 2) return cudaErrorLaunchFailure;
    for (const ZkpProgOp &op : r->prog->ops) {
        RView v[ZKP_PROG_MAX_VIEWS];
        for (u32 j = 0; j < ZKP_PROG_MAX_VIEWS; j++) v[j] = resolve(s, r, slot, op.v[j]);
        cudaError_t e = cudaSuccess;
        switch (op.kind) {
            case ZKP_OP_COPY:
                e = copy_views(v[0], v[1], v[0].len, op.imm[0], st);
                break;
            case ZKP_OP_ZERO:
                e = zero_view(v[0], op.imm[0], st);
                break;
            case ZKP_OP_NTT:
                e = op.imm[0] ? zkp_ntt_ex_shoup(v[0].poly(), v[1].ptr(), reinterpret_cast<const u32 *>(op.imm[0]),
                                                 log2_exact(v[0].len), nullptr, nullptr, st)
                              : zkp_ntt_ex(v[0].poly(), v[1].ptr(), log2_exact(v[0].len), nullptr, nullptr, st);
                break;
            case ZKP_OP_NTT_RECOMPUTE:
                e = recompute_ntt(v[0].poly(), v[1].ptr(), (u32)op.imm[0], v[2].ptr(), log2_exact(v[0].len), st, 8,
                                  8);
                break;
            case ZKP_OP_DISTRIBUTE:
                e = distribute_powers(v[0].poly(), v[1].ptr(), v[1].len, st);
                break;
            case ZKP_OP_FUSED: {
                const u32 nv = (u32)op.imm[1], nm = (u32)op.imm[2];
                // the PolyPtr arrays go through the request's pinned staging to its device
                // argument buffer, as the reference's wrapper copies them (fused_kernels.rs:165-172)
                PolyPtr *stage = reinterpret_cast<PolyPtr *>(v[15].base);
                for (u32 j = 0; j < nv + nm; j++) stage[j] = v[j].poly();
                e = cudaMemcpyAsync(v[14].base, stage, (nv + nm) * sizeof(PolyPtr), cudaMemcpyHostToDevice, st);
                if (e == cudaSuccess) {
                    const PolyPtr *d = reinterpret_cast<const PolyPtr *>(v[14].base);
                    auto fn = reinterpret_cast<FusedFn>(op.imm[0]);
                    e = fn(reinterpret_cast<const ConstPolyPtr *>(d), d + nv, op.imm[3], true, nullptr, st);
                }
                break;
            }
            case ZKP_OP_MSM: {
                const u32 m = (u32)op.imm[3];
                const u32 nt = (u32)(op.imm[1] & 0xffffu), w = (u32)(op.imm[1] >> 16);
                ZkpMsmTask t[32];
                for (u32 j = 0; j < m; j++)
                    t[j] = ZkpMsmTask{reinterpret_cast<const u32 *>(op.imm[0]), nt, v[j].ptr(), v[j].len, w,
                                      v[m + j].ptr(), op.imm[2]};
                e = zkp_msm_batch(t, m, v[15].base, v[15].len, st);
                break;
            }
            case ZKP_OP_EVAL: {
                unsigned long tb = (unsigned long)v[0].len;
                e = poly_eval(v[0].base, &tb, v[2].cpoly(), v[1].ptr(), v[3].ptr(), st);
                break;
            }
            case ZKP_OP_INVERT: {
                unsigned long tb = (unsigned long)v[0].len;
                e = batched_invert(v[0].base, &tb, v[1].poly(), st);
                break;
            }
            case ZKP_OP_KATE: {
                unsigned long tb = (unsigned long)v[0].len;
                e = kate_division(v[0].base, &tb, log2_exact(v[2].len), v[2].cpoly(), v[3].ptr(), v[1].poly(), st);
                break;
            }
            case ZKP_OP_SCAN: {
                unsigned long tb = (unsigned long)v[0].len;
                e = scan_mul(v[0].base, &tb, v[1].poly(), st);
                break;
            }
            case ZKP_OP_ADD: e = poly_add(v[0].poly(), v[1].cpoly(), v[2].cpoly(), st); break;
            case ZKP_OP_SUB: e = poly_sub(v[0].poly(), v[1].cpoly(), v[2].cpoly(), st); break;
            case ZKP_OP_ZERO_POLY: e = poly_zero(v[0].poly(), st); break;
            case ZKP_OP_ONE_LAGRANGE: e = poly_one_lagrange(v[0].poly(), st); break;
            case ZKP_OP_ONE_COEF: e = poly_one_coef(v[0].poly(), st); break;
            case ZKP_OP_SCALAR_INV: e = inv_scalar(v[0].ptr(), st); break;
            case ZKP_OP_SCALAR_POW: e = scalar_pow(v[0].ptr(), op.imm[0], st); break;
            default: e = cudaErrorInvalidValue; break;
        }
        if (e != cudaSuccess) return e;
    }
    return cudaEventRecord(slot.done, st);
}

void finish(ZkpServer *s, Request *r, int status) {
    if (r->prog) {  // called with the server mutex held
        auto *p = const_cast<ZkpProgram *>(r->prog);
        if (--p->live == 0 && p->orphaned) delete p;
        r->prog = nullptr;
    }
    r->res.status = status;
    r->res.done_s = s->now();
    r->done = true;
    if (status == 0)
        s->stats.completed++;
    else
        s->stats.failed++;
}

// a request of the class the policy limits; the class is fixed at admission (r->large)
bool is_large(const ZkpServer *s, Request *r) {
    if (r->slot < 0) r->large = s->policy.max_large_inflight && s->policy.large_bytes &&
                                r->bytes >= s->policy.large_bytes;
    return r->large;
}

void worker_loop(ZkpServer *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        bool progressed = false;
        // completions
        for (auto &slot : s->slots) {
            if (!slot.req) continue;
            cudaError_t q = cudaEventQuery(slot.done);
            if (q == cudaErrorNotReady) continue;
            Request *r = slot.req;
            if (q == cudaSuccess) {
                if (r->prog) {
                    for (const ZkpProgOut &o : r->prog->outs)
                        memcpy(static_cast<char *>(r->results) + o.result_offset, slot.prog_host + o.host_offset,
                               o.bytes);
                } else {
                    memcpy(r->res.msm, slot.host, sizeof(r->res.msm));
                    memcpy(r->res.evals, slot.host + 64, sizeof(r->res.evals));
                }
                finish(s, r, 0);
            } else {
                finish(s, r, -3);
            }
            s->arena.release(r->off, r->bytes);
            if (is_large(s, r)) s->large_inflight--;
            slot.req = nullptr;
            s->inflight--;
            progressed = true;
        }
        if (progressed) s->cv_done.notify_all();
        // admission: arrival order, look-ahead of 8 for a request that fits
        for (size_t idx = 0; idx < s->pending.size() && idx < 8;) {
            int free_slot = -1;
            for (size_t i = 0; i < s->slots.size(); i++)
                if (!s->slots[i].req) {
                    free_slot = (int)i;
                    break;
                }
            if (free_slot < 0) break;
            Request *r = s->pending[idx];
            if (r->req.inject_fault == 1) {  // host-side injected allocation refusal
                s->pending.erase(s->pending.begin() + idx);
                r->res.start_s = s->now();
                finish(s, r, -4);
                s->cv_done.notify_all();
                continue;
            }
            if (is_large(s, r) && s->large_inflight >= s->policy.max_large_inflight) {
                idx++;  // a large request waits for another to finish; smaller ones may pass
                continue;
            }
            size_t off = s->arena.alloc(r->bytes);
            if (off == SIZE_MAX) {
                idx++;
                continue;
            }
            s->pending.erase(s->pending.begin() + idx);
            r->off = off;
            r->slot = free_slot;
            r->res.start_s = s->now();
            auto &slot = s->slots[free_slot];
            slot.req = r;
            // large requests make up the latency tail: with the policy's priority_bytes set they
            // run on the slot's high-priority stream, so the blocks of requests admitted around
            // them queue behind theirs instead of sharing the SMs evenly
            r->stream = (s->policy.priority_bytes && r->bytes >= s->policy.priority_bytes) ? slot.stream_hi
                                                                                               : slot.stream;
            if (is_large(s, r)) s->large_inflight++;
            s->inflight++;
            s->stats.peak_inflight = std::max<u64>(s->stats.peak_inflight, s->inflight);
            s->stats.peak_bytes = s->arena.peak();
            cudaError_t e = cudaSuccess;
            if (r->prog && slot.prog_host_bytes < r->prog->host_bytes) {
                // the slot is idle (its last request completed), so its host block can grow
                if (slot.prog_host) cudaFreeHost(slot.prog_host);
                slot.prog_host = nullptr;
                slot.prog_host_bytes = 0;
                e = cudaMallocHost(reinterpret_cast<void **>(&slot.prog_host), r->prog->host_bytes);
                if (e == cudaSuccess) slot.prog_host_bytes = r->prog->host_bytes;
            }
            if (e == cudaSuccess) e = r->prog ? launch_compiled(s, r, slot) : launch_program(s, r, slot);
            if (e != cudaSuccess) {
                // the request fails alone: drain what was queued on its stream, release it
                cudaStreamSynchronize(r->stream);
                cudaGetLastError();
                s->arena.release(r->off, r->bytes);
                if (is_large(s, r)) s->large_inflight--;
                slot.req = nullptr;
                s->inflight--;
                finish(s, r, -3);
                s->cv_done.notify_all();
            }
        }
        if (s->stop && s->pending.empty() && s->inflight == 0) break;
        if (s->inflight > 0)
            s->cv_work.wait_for(lk, std::chrono::microseconds(50));
        else
            s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
    }
}

}  // namespace

extern "C" unsigned long long zkp_serve_footprint(const ZkpServer *s, unsigned int k) {
    Plan p;
    if (!plan_request(const_cast<ZkpServer *>(s), k, &p)) return 0;
    return p.total;
}

extern "C" cudaError_t zkp_serve_create(const ZkpServeConfig *cfg, const unsigned int *bases_d,
                                        unsigned long long n_bases, ZkpServer **out) {
    if (!cfg || !out || cfg->max_inflight == 0 || cfg->min_k < 1 || cfg->max_k > 26 || cfg->min_k > cfg->max_k ||
        cfg->ext_log < 1 || cfg->ext_log > 3 || cfg->n_sets > ZKP_SERVE_MAX_SETS)
        return cudaErrorInvalidValue;
    std::vector<ZkpServeTableSet> sets;
    if (cfg->n_sets == 0) {
        sets.push_back(ZkpServeTableSet{bases_d, n_bases, cfg->msm_window, cfg->msm_tables, cfg->max_k});
    } else {
        sets.assign(cfg->sets, cfg->sets + cfg->n_sets);
    }
    for (size_t i = 0; i < sets.size(); i++) {
        const ZkpServeTableSet &t = sets[i];
        const u32 kmax = t.max_k < cfg->max_k ? t.max_k : cfg->max_k;
        if (!t.tables_d || t.n_tables == 0 || (t.n_tables > 1 && t.window == 0) || t.rows < (1ull << kmax) ||
            (i > 0 && t.max_k <= sets[i - 1].max_k))
            return cudaErrorInvalidValue;
    }
    if (sets.back().max_k < cfg->max_k) return cudaErrorInvalidValue;
    auto *s = new ZkpServer();
    s->cfg = *cfg;
    s->t0 = std::chrono::steady_clock::now();
    cudaGetDevice(&s->device);
    s->sets = sets;
    // fused quotient kernel, generated next to this library (lib/fused/)
    Dl_info info;
    std::string dir = ".";
    if (dladdr(reinterpret_cast<void *>(&zkp_serve_create), &info) && info.dli_fname) {
        dir = info.dli_fname;
        dir = dir.substr(0, dir.find_last_of('/'));
    }
    s->fused_lib = dlopen((dir + "/fused/libzkp_quotient_z8.so").c_str(), RTLD_NOW | RTLD_LOCAL);
    if (s->fused_lib) s->fused = reinterpret_cast<FusedFn>(dlsym(s->fused_lib, "zkp_quotient_z8"));
    if (!s->fused) {
        delete s;
        return cudaErrorSharedObjectSymbolNotFound;
    }
    cudaError_t e = s->arena.init(cfg->hbm_bytes);
    // per-size constants
    const zkh::Params &F = zkh::fr();
    s->consts.resize(cfg->max_k + 1);
    u32 *tmp = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&tmp, 32);
    if (e == cudaSuccess) e = cudaMalloc(&s->shift, 32);
    if (e == cudaSuccess) {
        zkh::Fe g = zkh::from_u64(F, 7);
        e = cudaMemcpy(s->shift, g.l, 32, cudaMemcpyHostToDevice);
    }
    const u32 ext = cfg->ext_log;
    for (u32 k = cfg->min_k; k <= cfg->max_k && e == cudaSuccess; k++) {
        SizeConsts &c = s->consts[k];
        const u64 n = 1ull << k;
        e = cudaMalloc(&c.inv_tw, (n / 2) * 32);
        if (e == cudaSuccess) e = cudaMalloc(&c.fwd_tw, (n << ext) / 2 * 32);
        if (e == cudaSuccess) e = cudaMalloc(&c.inv_sh, (n / 2) * 64);
        if (e == cudaSuccess) e = cudaMalloc(&c.fwd_sh, (n << ext) / 2 * 64);
        if (e == cudaSuccess) e = cudaMalloc(&c.ninv, 32);
        if (e == cudaSuccess) e = cudaMalloc(&c.zh_inv, (32u << ext));
        if (e != cudaSuccess) break;
        zkh::Fe wi = zkh::fr_root_of_unity(k, true);
        e = cudaMemcpy(tmp, wi.l, 32, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = zkp_ntt_roots_device(c.inv_tw, n / 2, tmp, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        zkh::Fe wf = zkh::fr_root_of_unity(k + ext, false);
        if (e == cudaSuccess) e = cudaMemcpy(tmp, wf.l, 32, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = zkp_ntt_roots_device(c.fwd_tw, (n << ext) / 2, tmp, 0);
        if (e == cudaSuccess) e = zkp_ntt_shoup_table(c.inv_tw, k, c.inv_sh, 0);
        if (e == cudaSuccess) e = zkp_ntt_shoup_table(c.fwd_tw, k + ext, c.fwd_sh, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        zkh::Fe ninv = zkh::inv(F, zkh::from_u64(F, n));
        if (e == cudaSuccess) e = cudaMemcpy(c.ninv, ninv.l, 32, cudaMemcpyHostToDevice);
        // 1/Z_H at g w_(k+ext)^j, Z_H(X) = X^n - 1: (g^n w^(j n) - 1)^-1 for j < 2^ext
        std::vector<zkh::Fe> zh(1u << ext);
        zkh::Fe gn = zkh::pow(F, zkh::from_u64(F, 7), n);
        zkh::Fe wn = zkh::pow(F, wf, n);
        zkh::Fe acc = gn;
        for (u32 j = 0; j < (1u << ext); j++) {
            zkh::Fe d = acc;
            // d - 1 (canonical subtraction of the Montgomery one)
            zkh::Fe one = zkh::one(F);
            uint64_t t[4];
            if (zkh::sub4(t, d.l, one.l)) zkh::add4(t, t, F.p);
            memcpy(d.l, t, 32);
            zh[j] = zkh::inv(F, d);
            acc = zkh::mul(F, acc, wn);
        }
        if (e == cudaSuccess) e = cudaMemcpy(c.zh_inv, zh.data(), (32u << ext), cudaMemcpyHostToDevice);
    }
    if (tmp) cudaFree(tmp);
    int prio_low = 0, prio_high = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    s->slots.resize(cfg->max_inflight);
    for (auto &slot : s->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&slot.stream, cudaStreamNonBlocking, prio_low);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&slot.stream_hi, cudaStreamNonBlocking, prio_high);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost(&slot.host, 4096);
    }
    if (e != cudaSuccess) {
        zkp_serve_destroy(s);
        return e;
    }
    s->stats.arena_bytes = s->arena.size();
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return cudaSuccess;
}

extern "C" long long zkp_serve_submit(ZkpServer *s, const ZkpProverRequest *req) {
    if (!s || !req) return -1;
    auto *r = new Request();
    r->req = *req;
    memset(&r->res, 0, sizeof(r->res));
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) {
        delete r;
        return -1;
    }
    r->ticket = s->next_ticket++;
    r->res.submit_s = s->now();
    s->all[r->ticket] = r;
    Plan p;
    if (req->k < s->cfg.min_k || req->k > s->cfg.max_k || !plan_request(s, req->k, &p)) {
        finish(s, r, -1);
        s->cv_done.notify_all();
        return r->ticket;
    }
    r->bytes = p.total;
    r->res.footprint = p.total;
    if (al(p.total) > s->arena.size()) {
        finish(s, r, -2);
        s->cv_done.notify_all();
        return r->ticket;
    }
    s->pending.push_back(r);
    s->cv_work.notify_one();
    return r->ticket;
}

extern "C" int zkp_serve_wait(ZkpServer *s, long long ticket, ZkpProverResult *out, double timeout_s) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return -1;
    Request *r = it->second;
    auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (!r->done) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !r->done) return 1;
    }
    if (out) *out = r->res;
    return 0;
}

extern "C" void zkp_serve_stats(const ZkpServer *s, ZkpServeStats *out) {
    auto *m = const_cast<ZkpServer *>(s);
    std::lock_guard<std::mutex> g(m->mu);
    *out = s->stats;
    out->peak_bytes = s->arena.peak();
}

extern "C" double zkp_serve_now(const ZkpServer *s) { return s->now(); }

extern "C" void zkp_serve_set_policy(ZkpServer *s, const ZkpServePolicy *policy) {
    if (!s || !policy) return;
    std::lock_guard<std::mutex> g(s->mu);
    s->policy = *policy;
}

extern "C" void zkp_serve_destroy(ZkpServer *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto &slot : s->slots) {
        if (slot.stream) cudaStreamDestroy(slot.stream);
        if (slot.stream_hi) cudaStreamDestroy(slot.stream_hi);
        if (slot.done) cudaEventDestroy(slot.done);
        if (slot.host) cudaFreeHost(slot.host);
        if (slot.prog_host) cudaFreeHost(slot.prog_host);
    }
    for (auto &c : s->consts) {
        cudaFree(c.inv_tw);
        cudaFree(c.fwd_tw);
        cudaFree(c.inv_sh);
        cudaFree(c.fwd_sh);
        cudaFree(c.ninv);
        cudaFree(c.zh_inv);
    }
    if (s->shift) cudaFree(s->shift);
    for (auto &kv : s->all) delete kv.second;
    if (s->fused_lib) dlclose(s->fused_lib);
    delete s;
}

// ------------------------------------------------------------------ compiled programs
extern "C" cudaError_t zkp_serve_program_create(ZkpServer *s, const ZkpProgOp *ops, unsigned int n_ops,
                                                unsigned long long device_bytes, unsigned long long host_bytes,
                                                const ZkpProgOut *outs, unsigned int n_outs,
                                                const unsigned long long *input_bytes, unsigned int n_inputs,
                                                ZkpProgram **out) {
    if (!s || !out || (n_ops && !ops) || (n_outs && !outs) || (n_inputs && !input_bytes))
        return cudaErrorInvalidValue;
    for (unsigned i = 0; i < n_ops; i++) {
        const ZkpProgOp &op = ops[i];
        const u32 need = required_views(op);
        if (need == ~0u || op.n_views > ZKP_PROG_MAX_VIEWS || need > op.n_views) return cudaErrorInvalidValue;
        if (op.kind == ZKP_OP_FUSED && (op.imm[0] == 0 || op.imm[1] + op.imm[2] > 14 || op.imm[3] == 0))
            return cudaErrorInvalidValue;
        if (op.kind == ZKP_OP_MSM && (op.imm[0] == 0 || op.imm[3] == 0 || op.imm[3] > 7)) return cudaErrorInvalidValue;
        if ((op.kind == ZKP_OP_COPY || op.kind == ZKP_OP_ZERO) && op.imm[0] != 32 && op.imm[0] != 64)
            return cudaErrorInvalidValue;
        if (op.kind == ZKP_OP_COPY && op.v[0].len != op.v[1].len) return cudaErrorInvalidValue;
        for (u32 j = 0; j < ZKP_PROG_MAX_VIEWS; j++) {
            const ZkpProgView &v = op.v[j];
            if (v.space == ZKP_SPACE_NONE) continue;
            if (!view_well_formed(v)) return cudaErrorInvalidValue;
            const u64 end = v.addr + v.whole_len * view_elem_bytes(op, j);
            if (v.space == ZKP_SPACE_DEVICE && end > device_bytes) return cudaErrorInvalidValue;
            if (v.space == ZKP_SPACE_HOST && end > host_bytes) return cudaErrorInvalidValue;
            if (v.space == ZKP_SPACE_INPUT && (v.index >= n_inputs || end > input_bytes[v.index]))
                return cudaErrorInvalidValue;
            if (v.space > ZKP_SPACE_INPUT) return cudaErrorInvalidValue;
        }
        // the fused argument buffer and its staging, the MSM workspace: present and large enough
        if (op.kind == ZKP_OP_FUSED) {
            const u64 bytes = (op.imm[1] + op.imm[2]) * sizeof(PolyPtr);
            if (op.v[14].space != ZKP_SPACE_DEVICE || op.v[14].len < bytes || op.v[15].space != ZKP_SPACE_HOST ||
                op.v[15].len < bytes)
                return cudaErrorInvalidValue;
        }
        if (op.kind == ZKP_OP_MSM && op.v[15].space != ZKP_SPACE_DEVICE) return cudaErrorInvalidValue;
    }
    u64 extent = 0;
    for (unsigned i = 0; i < n_outs; i++) {
        if (outs[i].host_offset + outs[i].bytes > host_bytes) return cudaErrorInvalidValue;
        extent = std::max<u64>(extent, outs[i].result_offset + outs[i].bytes);
    }
    auto *p = new ZkpProgram();
    p->ops.assign(ops, ops + n_ops);
    p->device_bytes = std::max<u64>(device_bytes, 256);
    p->host_bytes = std::max<u64>(host_bytes, 256);
    p->outs.assign(outs, outs + n_outs);
    p->result_extent = extent;
    p->input_bytes.assign(input_bytes, input_bytes + n_inputs);
    *out = p;
    return cudaSuccess;
}

extern "C" long long zkp_serve_submit_program(ZkpServer *s, const ZkpProgram *prog, const void *const *inputs,
                                              unsigned int n_inputs, void *results,
                                              unsigned long long results_bytes) {
    if (!s || !prog) return -1;
    auto *r = new Request();
    memset(&r->req, 0, sizeof(r->req));
    memset(&r->res, 0, sizeof(r->res));
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop || prog->orphaned) {
        delete r;
        return -1;
    }
    r->prog = prog;
    const_cast<ZkpProgram *>(prog)->live++;
    r->ticket = s->next_ticket++;
    r->res.submit_s = s->now();
    s->all[r->ticket] = r;
    bool ok = n_inputs == prog->input_bytes.size() && (n_inputs == 0 || inputs != nullptr) &&
              results_bytes >= prog->result_extent && (prog->result_extent == 0 || results != nullptr);
    for (unsigned i = 0; ok && i < n_inputs; i++) ok = inputs[i] != nullptr || prog->input_bytes[i] == 0;
    if (!ok) {
        finish(s, r, -1);
        s->cv_done.notify_all();
        return r->ticket;
    }
    r->inputs.assign(inputs, inputs + n_inputs);
    r->results = results;
    r->bytes = prog->device_bytes;
    r->res.footprint = prog->device_bytes;
    if (al(prog->device_bytes) > s->arena.size()) {
        finish(s, r, -2);
        s->cv_done.notify_all();
        return r->ticket;
    }
    s->pending.push_back(r);
    s->cv_work.notify_one();
    return r->ticket;
}

extern "C" void zkp_serve_program_destroy(ZkpServer *s, ZkpProgram *prog) {
    if (!s || !prog) return;
    std::lock_guard<std::mutex> g(s->mu);
    if (prog->live > 0)
        prog->orphaned = true;  // the last of its requests to finish frees it
    else
        delete prog;
}
