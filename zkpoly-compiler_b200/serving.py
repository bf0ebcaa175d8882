"""The served form: a continuous-batching request loop (libzkp_runtime.so) and a Poisson
load generator that measures p50 / p99 latency and throughput against the plain path (the same
server with one request in flight at a time).  See include/zkp_runtime.h for the program a
request runs."""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from .native import (ZkpProverRequest, ZkpProverResult, ZkpServeConfig, ZkpServeStats, check, load)
from .scalar import require_cuda

LIB = "libzkp_runtime.so"


class Server:
    def __init__(self, bases, hbm_bytes: int, max_inflight: int = 8, ext_log: int = 2,
                 min_k: int = 14, max_k: int = 22, msm_window: int = 0):
        """bases: a (N, 16) int32 device tensor of affine points, or a msm.ResidentBases
        (its precomputed tables and window are used)."""
        require_cuda()
        self.lib = load(LIB)
        self.bases = bases
        if hasattr(bases, "tables"):
            ptr, n_bases, tables, msm_window = bases.tables.data_ptr(), bases.n, bases.n_tables, bases.window
        else:
            ptr, n_bases, tables = bases.data_ptr(), bases.shape[0], 1
        cfg = ZkpServeConfig(hbm_bytes, max_inflight, ext_log, min_k, max_k, msm_window, tables)
        self.h = ctypes.c_void_p()
        check(self.lib.zkp_serve_create(ctypes.byref(cfg), ptr, n_bases, ctypes.byref(self.h)), "zkp_serve_create")

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


def run_schedule(server: Server, schedule, timeout_s: float = 900.0):
    """Submits each (arrival_s, k, seed) at its arrival time, waits for all; returns results
    and summary statistics (latency = completion - submission, server clock)."""
    start = time.perf_counter()
    tickets = []
    for t_arr, k, seed in schedule:
        delay = t_arr - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        tickets.append(server.submit(k, seed))
    results = [server.wait(t, timeout_s) for t in tickets]
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
