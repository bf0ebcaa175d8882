"""The served form: a continuous-batching request loop (libzkp_runtime.so) and a Poisson
load generator that measures p50 / p99 latency and throughput against the plain path (the same
server with one request in flight at a time).  See include/zkp_runtime.h for the program a
request runs."""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from .native import (ZkpProverRequest, ZkpProverResult, ZkpServeConfig, ZkpServeStats, ZkpServeTableSet, check,
                     load)
from .scalar import require_cuda

LIB = "libzkp_runtime.so"


class Server:
    def __init__(self, bases, hbm_bytes: int, max_inflight: int = 8, ext_log: int = 2,
                 min_k: int = 14, max_k: int = 22, msm_window: int = 0):
        """bases: a (N, 16) int32 device tensor of affine points, a msm.ResidentBases (its
        precomputed tables and window are used for every size), or a list of
        (msm.ResidentBases, max_k) by ascending max_k (per-size table sets, see resident_sets)."""
        require_cuda()
        self.lib = load(LIB)
        self.bases = bases
        n_sets, sets = 0, []
        if isinstance(bases, (list, tuple)):
            ptr, n_bases, tables = None, 0, 1
            for rb, mk in bases:
                sets.append(ZkpServeTableSet(rb.tables.data_ptr(), rb.n, rb.window, rb.n_tables, mk))
            n_sets = len(sets)
        elif hasattr(bases, "tables"):
            ptr, n_bases, tables, msm_window = bases.tables.data_ptr(), bases.n, bases.n_tables, bases.window
        else:
            ptr, n_bases, tables = bases.data_ptr(), bases.shape[0], 1
        cfg = ZkpServeConfig(hbm_bytes, max_inflight, ext_log, min_k, max_k, msm_window, tables, n_sets)
        for i, t in enumerate(sets):
            cfg.sets[i] = t
        self.h = ctypes.c_void_p()
        check(self.lib.zkp_serve_create(ctypes.byref(cfg), ptr, n_bases, ctypes.byref(self.h)), "zkp_serve_create")

    def set_policy(self, priority_k: int = 0, large_k: int = 0, max_large_inflight: int = 0) -> None:
        """zkp_serve_set_policy with its thresholds given as sizes: requests at least as large
        (by planned footprint) as a built-in request of size priority_k run on high-priority
        streams; at most max_large_inflight requests at least as large as one of size large_k
        run at once.  Zeros turn each off."""
        from .native import ZkpServePolicy
        fp = lambda k: int(self.lib.zkp_serve_footprint(self.h, k)) if k else 0  # noqa: E731
        pol = ZkpServePolicy(fp(priority_k), fp(large_k), max_large_inflight)
        self.lib.zkp_serve_set_policy(self.h, ctypes.byref(pol))

    def footprint(self, k: int) -> int:
        return int(self.lib.zkp_serve_footprint(self.h, k))

    def submit(self, k: int, seed: int, inject_fault: int = 0) -> int:
        req = ZkpProverRequest(k, seed, inject_fault)
        t = self.lib.zkp_serve_submit(self.h, ctypes.byref(req))
        if t < 0:
            raise RuntimeError("server is shutting down")
        return t

    def wait(self, ticket: int, timeout_s: float = 600.0) -> ZkpProverResult:
        res = ZkpProverResult()
        rc = self.lib.zkp_serve_wait(self.h, ticket, ctypes.byref(res), timeout_s)
        if rc != 0:
            raise TimeoutError(f"ticket {ticket} not done after {timeout_s} s")
        return res

    def now(self) -> float:
        return float(self.lib.zkp_serve_now(self.h))

    def stats(self) -> dict:
        st = ZkpServeStats()
        self.lib.zkp_serve_stats(self.h, ctypes.byref(st))
        return {f: getattr(st, f) for f, _ in ZkpServeStats._fields_}

    def close(self):
        if self.h:
            self.lib.zkp_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def resident_sets(points: torch.Tensor, k_lo: int, k_hi: int):
    """Per-size resident table sets for a server: sizes 2^k_lo .. 2^k_hi grouped by the tuned
    (window, tables) of each size, one msm.ResidentBases per group over the first 2^(largest k)
    points.  Returns [(ResidentBases, max_k)] by ascending max_k."""
    from . import msm, tuner
    groups = []
    for k in range(k_lo, k_hi + 1):
        cfg = tuner.msm_resident_config(1 << k)
        if groups and groups[-1][0] == cfg:
            groups[-1][1] = k
        else:
            groups.append([cfg, k])
    assert len(groups) <= 8, "too many table sets"
    return [(msm.ResidentBases(points[: 1 << mk], window=c, n_tables=nt), mk) for (c, nt), mk in groups]


class PerCallProver:
    """The plain per-call path: the served program (include/zkp_runtime.h), one request at a
    time, every operator called through its own per-call entry point on one stream.  The four
    MSMs go through the reference ABI `msm` (core/src/msm.rs:302-369): the runtime hands that
    call host scalar arrays and host point tables and gets host affine results back, so each
    request moves its MSM inputs device -> host -> device, as the reference's runtime does.
    Results are bit-identical to the served form's (the test suite checks it)."""

    def __init__(self, bases, ext_log: int = 2, device="cuda", max_k: int | None = None):
        from . import msm
        require_cuda()
        if isinstance(bases, (list, tuple)):
            bases = bases[-1][0]  # the set that covers the largest size holds every base
        pts = bases.tables[: bases.n] if hasattr(bases, "tables") else bases
        # host point table (pinned, as a runtime's host pool would hand it out)
        self.h_bases = pts.cpu().pin_memory()
        self.h_bases_np = self.h_bases.numpy().view(np.uint32)
        self.ext = ext_log
        self.device = device
        self.cfg = msm.MsmConfig()
        self._ws = None
        self._stage = None
        if max_k is not None:  # the pinned staging area up front, outside any timed loop
            self._stage = torch.empty((4, 1 << max_k, 8), dtype=torch.int32).pin_memory()
        self._consts = {}

    def _const(self, k: int):
        from . import fused, ntt, pipeline
        if k not in self._consts:
            self._consts[k] = {
                "inv_tw": ntt.twiddle_table(k, True, self.device),
                "fwd_tw": ntt.twiddle_table(k + self.ext, False, self.device),
                "ninv": ntt.n_inv(k, self.device),
                "shift": ntt.scalar_const(pipeline.SHIFT, self.device),
                "zh": pipeline.zh_inv_device(k, self.ext, self.device),
            }
            if not hasattr(self, "quotient"):
                self.quotient = fused.quotient_kernel()
        return self._consts[k]

    def warm(self, ks) -> None:
        """Builds the per-size constants (root tables, n^-1, 1/Z_H) ahead of time, as the
        served form does when it is created."""
        for k in ks:
            self._const(k)
        torch.cuda.synchronize()

    def run(self, k: int, seed: int) -> np.ndarray:
        """Result words (4 MSM points, 2 evaluations) of request (k, seed), as result_words."""
        from . import gen, msm, ntt, pipeline, poly
        from .scalar import ScalarArray
        c = self._const(k)
        n, N = 1 << k, 1 << (k + self.ext)
        s = seed * 8
        a, b, cc = (ScalarArray(gen.fr(s + i, n, self.device)) for i in range(3))
        z = ScalarArray(gen.fr(s + 3, N, self.device))
        x = gen.fr(s + 4, 1, self.device)
        for v in (a, b, cc):
            ntt.ntt_ex(v, c["inv_tw"], None, c["ninv"])
        e = ScalarArray.alloc(N, self.device)
        ntt.coset_lde(e, cc, c["fwd_tw"], c["shift"])
        q = ScalarArray.alloc(N, self.device)
        self.quotient([q], [e, e, e, z, pipeline.rotated(z, self.ext), c["zh"]])
        # reference-ABI MSM: host scalars in (staged in pinned memory, as a runtime's host pool
        # would hold them), host affine points out
        if self._stage is None or self._stage.shape[1] < n:
            self._stage = torch.empty((4, n, 8), dtype=torch.int32).pin_memory()
        for i, t in enumerate((a, b, cc, q)):
            self._stage[i, :n].copy_(t.values[:n])
        stage = self._stage.numpy().view(np.uint32)
        host_scalars = [stage[i, :n] for i in range(4)]
        sizes = msm.MSM(self.cfg).get_buffer_size(n)
        if self._ws is None or self._ws.numel() < sizes[0]:
            self._ws = torch.empty(sizes[0], dtype=torch.uint8, device=self.device)
        points = msm.msm_host_batches(host_scalars, [self.h_bases_np[:n]], buffers=[self._ws], cfg=self.cfg)
        ev = torch.zeros((2, 8), dtype=torch.int32, device=self.device)
        poly.poly_eval(a, x, ev[0])
        poly.poly_eval(b, x, ev[1])
        return np.concatenate([p.view(np.uint32) for p in points] + [ev.cpu().numpy().view(np.uint32).ravel()])


def run_schedule_per_call(prover: PerCallProver, schedule):
    """The plain path under the same arrivals: requests run one after another in arrival
    order; latency = completion - arrival (host clock)."""
    start = time.perf_counter()
    lat, words = [], []
    first = last = None
    for t_arr, k, seed in schedule:
        delay = t_arr - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        t0 = time.perf_counter()
        words.append(prover.run(k, seed))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        first = t0 if first is None else first
        last = t1
        lat.append((t1 - start - t_arr) * 1e3)
    lat = np.array(lat)
    summary = {"requests": len(schedule), "ok": len(schedule), "p50_ms": float(np.percentile(lat, 50)),
               "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
               "req_per_s": len(schedule) / (last - start - schedule[0][0])}
    return words, summary


def result_words(res: ZkpProverResult) -> np.ndarray:
    """msm points and evals of a result as one uint32 vector (for bit-exact comparisons)."""
    return np.concatenate([np.frombuffer(bytes(res.msm), dtype=np.uint32),
                           np.frombuffer(bytes(res.evals), dtype=np.uint32)])


def poisson_schedule(n_req: int, rate: float, k_lo: int, k_hi: int, seed: int):
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n_req)
    arrivals = np.cumsum(gaps) - gaps[0]
    ks = rng.integers(k_lo, k_hi + 1, n_req)
    return [(float(t), int(k), 10_000 + i) for i, (t, k) in enumerate(zip(arrivals, ks))]


def run_schedule(server: Server, schedule, timeout_s: float = 900.0, submit=None, wait=None):
    """Submits each (arrival_s, k, seed) at its arrival time, waits for all; returns results
    and summary statistics (latency = completion - submission, server clock).  ``submit(k,
    seed)`` / ``wait(handle)`` replace the built-in program's submission (compiled programs:
    program.CompiledProgram)."""
    submit = submit or server.submit
    wait = wait or (lambda t: server.wait(t, timeout_s))
    start = time.perf_counter()
    tickets = []
    for t_arr, k, seed in schedule:
        delay = t_arr - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        tickets.append(submit(k, seed))
    results = [wait(t) for t in tickets]
    ok = [r for r in results if r.status == 0]
    lat = np.array([r.done_s - r.submit_s for r in ok]) * 1e3
    span = max(r.done_s for r in ok) - min(r.submit_s for r in ok) if ok else float("nan")
    summary = {
        "requests": len(results), "ok": len(ok),
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_ms": float(lat.mean()) if len(lat) else None,
        "req_per_s": len(ok) / span if ok else None,
        "stats": server.stats(),
    }
    return results, summary
