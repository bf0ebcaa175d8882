"""Benchmark: MSM points/s at n = 2^22 and NTT elems/s at n = 2^24 over BN254 on B200.

One step = one forward NTT of 2^24 Fr elements followed by one MSM of 2^22 G1 points, inputs
resident in HBM (both larger than L2, so nothing is served from cache between steps).  The
JSON line's `value` is the MSM throughput (points/s); the NTT throughput is under "ntt".
`e2e` repeats both through the reference-facing C ABI (msm() with host tables; ssip_ntt with a
host->device copy in and a device->host copy out) from pinned host memory.

`--impl reference` times the reference's CPU path instead: halo2 best_multiexp / best_fft as
restated by the oracle, on all host cores, on a bounded sample of the same workload.

Multi-GPU: one process per GPU (torchrun); every rank runs its own replica of the step
("replicas only": the path has no exchange step), timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MSM points/s (2^22) & NTT elems/s (2^24); served p50/p99 vs plain per-call"
MSM_LOG, NTT_LOG = 22, 24
# ncu DRAM bytes (read + write) of one whole 2^24 transform (all five passes) per element, from the
# capture summarised in profiles/ntt_passes_ntt2p24.md
NTT_TRAFFIC_PER_ELEM = 398.0


def workload_config(world: int) -> dict:
    """The workload both arms report (the GPU arm's resident-table choice is under "msm")."""
    return {"workload": f"MSM n=2^{MSM_LOG} (BN254 G1, seeded scalars, points k_i*G) + NTT n=2^{NTT_LOG} "
                        f"(BN254 Fr, natural order, seeded)",
            "msm_n": 1 << MSM_LOG, "ntt_n": 1 << NTT_LOG, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (NTT 512 MiB vector; MSM bases, sorted digits and pairing lists "
                  "of hundreds of MB to GBs)"}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(values, device=None):
    """Element-wise maximum of per-rank timings over all ranks (the job's time is its slowest
    rank's); the identity on one process.  Works on any initialised backend (nccl, gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ------------------------------------------------------------------ CPU (reference path)
_CPU_INPUTS = {}


def cpu_reference(sample_msm_log=22, sample_ntt_log=24, reps=1):
    """halo2 best_multiexp / best_fft restated (oracle), all host threads, bounded samples."""
    from oracle import oracle as orc
    orc.build()
    th = orc.threads()
    key = (sample_msm_log, sample_ntt_log)
    if key not in _CPU_INPUTS:
        _CPU_INPUTS[key] = (orc.gen_fr(1, 1 << sample_msm_log), orc.gen_points(2, 1 << sample_msm_log),
                            orc.gen_fr(0, 1 << sample_ntt_log))
    s, p, a = _CPU_INPUTS[key]
    t0 = time.perf_counter()
    for _ in range(reps):
        msm_out = orc.best_multiexp(s, p)
    msm_t = (time.perf_counter() - t0) / reps
    w = orc.root_of_unity(sample_ntt_log)
    t0 = time.perf_counter()
    for _ in range(reps):
        ntt_out = orc.best_fft(a, w, sample_ntt_log)
    ntt_t = (time.perf_counter() - t0) / reps
    return {
        "msm_points_per_s": (1 << sample_msm_log) / msm_t,
        "ntt_elems_per_s": (1 << sample_ntt_log) / ntt_t,
        "cores": th,
        "msm_s": msm_t, "ntt_s": ntt_t,
        "msm_sample": f"best_multiexp n=2^{sample_msm_log} (seeds 1/2), {msm_t:.2f} s",
        "ntt_sample": f"best_fft n=2^{sample_ntt_log} (seed 0), {ntt_t:.2f} s",
        # the outputs themselves: the GPU arm checks its timed results against them
        "logs": (sample_msm_log, sample_ntt_log), "msm_out": msm_out, "ntt_out": ntt_out, "ntt_in": a,
    }


def ntt_chain_expected(a, fft_a, t: int, log_n: int):
    """State of a vector after t in-place forward transforms, from one transform of it.

    Applying the size-n DFT twice gives F(F(a))[j] = n * a[-j mod n], so after t transforms
    the vector is n^m * b[(-1)^m j mod n] with m = t // 2 and b = a (t even) or F(a) (t odd).
    This lets the benchmark check the exact bytes its timed in-place transforms left behind
    against one best_fft of the input."""
    import numpy as np
    from oracle import oracle as orc
    n = 1 << log_n
    m = t // 2
    b = fft_a if t % 2 else a
    if m % 2:
        idx = (-np.arange(n, dtype=np.int64)) % n
        b = b[idx]
    if m:
        nm = orc.pow_(orc.to_mont(orc.int_to_limbs(n)), m)
        b = orc.vec_mul(np.ascontiguousarray(b), np.ascontiguousarray(np.broadcast_to(nm, b.shape)))
    return np.ascontiguousarray(b)


def verify_outputs(cpu, timed, e2e):
    """Bit-exact comparison of the timed results (and of the C-ABI e2e results) with the CPU
    port's best_multiexp / best_fft on the same seeded inputs."""
    import numpy as np
    from oracle import oracle as orc
    if cpu is None or cpu["logs"] != (MSM_LOG, NTT_LOG):
        orc.build()
        s, p = orc.gen_fr(1, 1 << MSM_LOG), orc.gen_points(2, 1 << MSM_LOG)
        a = orc.gen_fr(0, 1 << NTT_LOG)
        cpu = {"msm_out": orc.best_multiexp(s, p), "ntt_in": a,
               "ntt_out": orc.best_fft(a, orc.root_of_unity(NTT_LOG), NTT_LOG)}
    out = {}
    out["msm_timed"] = bool(np.array_equal(timed["msm"], cpu["msm_out"]))
    expect = ntt_chain_expected(cpu["ntt_in"], cpu["ntt_out"], timed["ntt_transforms"], NTT_LOG)
    out["ntt_timed"] = bool(np.array_equal(timed["ntt"], expect))
    if e2e is not None:
        out["msm_e2e"] = bool(np.array_equal(e2e["msm"], cpu["msm_out"]))
        out["ntt_e2e"] = bool(np.array_equal(e2e["ntt"], cpu["ntt_out"]))
    out["how"] = (f"MSM result of the last timed step and of the e2e msm() call == best_multiexp (seeds 1/2, "
                  f"n=2^{MSM_LOG}); NTT vector after the {timed['ntt_transforms']} in-place transforms of "
                  f"warm-up + timed region == n^m * best_fft(a)[(-1)^m j] (m = t // 2; F(F(a))[j] = n a[-j]); "
                  f"e2e ssip_ntt output == best_fft(a) (seed 0, n=2^{NTT_LOG})")
    return all(v for k, v in out.items() if k != "how"), out


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    steps = []
    for _ in range(args.warmup):
        cpu_reference(args.ref_msm_log, args.ref_ntt_log)
    for _ in range(args.steps):
        steps.append(cpu_reference(args.ref_msm_log, args.ref_ntt_log))
    v = statistics.median([s["msm_points_per_s"] for s in steps])
    ntt_v = statistics.median([s["ntt_elems_per_s"] for s in steps])
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (BN254 Montgomery limbs)", "data": "synthetic (seeded)",
        "config": workload_config(world),
        "ms_per_step": statistics.median([s["msm_s"] + s["ntt_s"] for s in steps]) * 1e3,
        "ntt": {"metric": f"NTT elems/s (2^{NTT_LOG})", "value": ntt_v, "unit": "elems/s"},
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": steps[-1]["cores"], "kind": "port",
                         "sample": steps[-1]["msm_sample"] + "; " + steps[-1]["ntt_sample"], "cpu": cpu_model()},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        line["ref_gpu"] = measure_reference_gpu(steps[-1])
    print(json.dumps(line), flush=True)


def measure_reference_gpu(cpu):
    """The reference's own CUDA kernels for the path, built from its sources for sm_100a
    (oracle/build_ref.py), timed on this box on the CPU arm's inputs and checked bit for bit
    against the CPU arm's outputs: ssip_ntt at 2^24 (root table from its ssip_precompute), msm
    at 2^22 through its host-buffer ABI in the configuration its cost model picks for that size
    (window 17, 8 target windows: two point tables from its msm_precompute, 16 parts, two
    stages; host clock, the call is synchronous), and poly_eval / batched_invert / kate_division
    / scan_mul at 2^22 (CUDA events).  Outside the timed CPU steps; none of this repository's
    kernels run here."""
    import ctypes
    import numpy as np
    here = os.path.join(ROOT, "oracle", "_ref")
    names = ("libref_ntt.so", "libref_msm_17_8.so", "libref_poly.so")
    if not all(os.path.exists(os.path.join(here, n)) for n in names):
        return {"unavailable": "the reference's kernels were not built (oracle/_ref absent)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
    except ImportError:
        return {"unavailable": "torch missing"}
    from oracle import oracle as orc

    class PolyPtr(ctypes.Structure):
        _fields_ = [("ptr", ctypes.c_void_p), ("len", ctypes.c_size_t), ("rotate", ctypes.c_size_t),
                    ("offset", ctypes.c_size_t), ("whole_len", ctypes.c_size_t)]

    V, U, UL = ctypes.c_void_p, ctypes.c_uint, ctypes.POINTER(ctypes.c_ulong)
    ntt = ctypes.CDLL(os.path.join(here, names[0]))
    ntt.ssip_ntt.argtypes = [PolyPtr, V, U, V, U, U]
    ntt.ssip_precompute.argtypes = [V, U, V]
    msm = ctypes.CDLL(os.path.join(here, names[1]))
    msm.msm.argtypes = [V, V, ctypes.c_ulonglong, U, U, U, U, U, V, V, U, V, V]
    msm.msm_precompute.argtypes = [ctypes.c_ulonglong, V, U]
    poly = ctypes.CDLL(os.path.join(here, names[2]))
    for name, a in (("poly_eval", [V, UL, PolyPtr, V, V, V]), ("batched_invert", [V, UL, PolyPtr, V]),
                    ("kate_division", [V, UL, U, PolyPtr, V, PolyPtr, V]), ("scan_mul", [V, UL, PolyPtr, V])):
        getattr(poly, name).argtypes = a
    for lib in (ntt, msm, poly):
        for f in ("ssip_ntt", "ssip_precompute", "msm", "msm_precompute", "poly_eval", "batched_invert",
                  "kate_division", "scan_mul"):
            if hasattr(lib, f):
                getattr(lib, f).restype = ctypes.c_int
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    out = {"built_from": "the reference's core/src/{ntt,msm,poly}/src sources, nvcc sm_100a (oracle/build_ref.py)"}

    def dev_words(a, words):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32).reshape(-1, words).copy()).to(dev)

    def pp(t, n):
        return PolyPtr(t.data_ptr(), n, 0, 0, n)

    def events(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # ---- ssip_ntt at the CPU arm's NTT size, on its input
    L = cpu["logs"][1]
    n = 1 << L
    w = np.ascontiguousarray(orc.root_of_unity(L)).view(np.uint32).copy()
    tw_h = np.zeros((n // 2, 8), dtype=np.uint32)
    assert ntt.ssip_precompute(tw_h.ctypes.data, n // 2, w.ctypes.data) == 0
    tw = dev_words(tw_h, 8)
    x0 = dev_words(cpu["ntt_in"], 8)
    x = x0.clone()
    assert ntt.ssip_ntt(pp(x, n), tw.data_ptr(), L, st, 8, 8) == 0
    torch.cuda.synchronize()
    got = x.cpu().numpy().view(np.uint64).reshape(-1, 4)
    ms = events(lambda: ntt.ssip_ntt(pp(x, n), tw.data_ptr(), L, st, 8, 8))
    out["ssip_ntt"] = {"log_n": L, "ms": ms, "elems_per_s": n / (ms / 1e3),
                       "matches_cpu_best_fft": bool(np.array_equal(got, cpu["ntt_out"]))}
    del x, x0, tw
    # ---- msm at the CPU arm's MSM size, its inputs, through the host-buffer ABI
    M = cpu["logs"][0]
    m = 1 << M
    s_h = np.ascontiguousarray(_CPU_INPUTS[cpu["logs"]][0]).view(np.uint32).reshape(m, 8)
    p_h = np.ascontiguousarray(_CPU_INPUTS[cpu["logs"]][1]).view(np.uint32).reshape(m, 16)
    pin = lambda a: torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32)  # noqa: E731
    s_h, tables = pin(s_h), [pin(p_h), pin(np.zeros_like(p_h))]
    h_tab = (ctypes.c_void_p * 2)(*[t.ctypes.data for t in tables])
    assert msm.msm_precompute(m, h_tab, 1) == 0
    parts = 16 if m >= (1 << 16) else 1
    cards = (ctypes.c_uint * 1)(0)
    sizes = (ctypes.c_ulong * 1)()
    assert msm.msm(None, sizes, m, 1, parts, 2, 2, 1, cards, None, 0, None, None) == 0
    buf = torch.empty(int(sizes[0]), dtype=torch.uint8, device=dev)
    bufs = (ctypes.c_void_p * 1)(buf.data_ptr())
    h_s = (ctypes.c_void_p * 1)(s_h.ctypes.data)
    res = np.zeros(16, dtype=np.uint32)
    h_r = (ctypes.c_void_p * 1)(res.ctypes.data)
    times = []
    for _ in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        assert msm.msm(bufs, None, m, 1, parts, 2, 2, 1, cards, h_tab, 1, h_s, h_r) == 0
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    best = min(times[1:])
    out["msm"] = {"log_n": M, "ms": best * 1e3, "points_per_s": m / best, "config": "window 17, 2 tables, 16 parts",
                  "timing": "host clock, best of 3 after one warm-up (synchronous host-buffer call)",
                  "matches_cpu_best_multiexp": bool(np.array_equal(res.view(np.uint64), cpu["msm_out"]))}
    del buf, tables
    # ---- poly library at 2^22 on seeded inputs (poly_eval checked against Horner)
    P = 22
    k = 1 << P
    p0 = orc.gen_fr(900, k)
    xh = orc.gen_fr(901, 1)
    pd, xd = dev_words(p0, 8), dev_words(xh, 8)
    r = torch.zeros(8, dtype=torch.int32, device=dev)
    q = torch.zeros((k, 8), dtype=torch.int32, device=dev)
    inv = pd.clone()
    scan = pd.clone()

    def temp(fn, *a):
        size = ctypes.c_ulong(0)
        assert fn(None, ctypes.byref(size), *a) == 0
        return torch.empty(max(size.value, 1), dtype=torch.uint8, device=dev), size
    te, ze = temp(poly.poly_eval, pp(pd, k), None, None, None)
    ti, zi = temp(poly.batched_invert, pp(inv, k), None)
    tk, zk_ = temp(poly.kate_division, P, pp(pd, k), None, pp(q, k), None)
    ts, zs = temp(poly.scan_mul, pp(scan, k), None)
    assert poly.poly_eval(te.data_ptr(), ctypes.byref(ze), pp(pd, k), r.data_ptr(), xd.data_ptr(), st) == 0
    torch.cuda.synchronize()
    eval_ok = bool(np.array_equal(r.cpu().numpy().view(np.uint64), orc.eval_poly(p0, xh[0])))
    out["poly"] = {"log_n": P, "poly_eval_matches_cpu_horner": eval_ok}
    for name, fn in (
            ("poly_eval", lambda: poly.poly_eval(te.data_ptr(), ctypes.byref(ze), pp(pd, k), r.data_ptr(),
                                                 xd.data_ptr(), st)),
            ("batched_invert", lambda: poly.batched_invert(ti.data_ptr(), ctypes.byref(zi), pp(inv, k), st)),
            ("kate_division", lambda: poly.kate_division(tk.data_ptr(), ctypes.byref(zk_), P, pp(pd, k),
                                                         xd.data_ptr(), pp(q, k), st)),
            ("scan_mul", lambda: poly.scan_mul(ts.data_ptr(), ctypes.byref(zs), pp(scan, k), st))):
        out["poly"][name + "_ms"] = events(fn)
    torch.cuda.synchronize()
    return out


# ------------------------------------------------------------------ GPU arm
def run_gpu(args):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    zk = importlib.import_module("zkpoly-compiler_b200")
    native, gen = zk.native, importlib.import_module("zkpoly-compiler_b200.gen")
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    n_msm, n_ntt = 1 << MSM_LOG, 1 << NTT_LOG

    with torch.cuda.stream(stream):
        # inputs generated on the device by the same counter-based generator as the oracle
        scalars = gen.fr(1, n_msm, dev)
        points = gen.points(2, n_msm, dev)
        ntt_in = gen.fr(0, n_ntt, dev)
        x = zk.ScalarArray(ntt_in.clone())
        tw = zk.ntt.twiddle_table(NTT_LOG)
        tw_shoup = zk.ntt.shoup_table(NTT_LOG)  # built once, like the root table
        if args.window:
            win, nt = args.window, args.tables or 1
        else:
            win, nt = zk.tuner.msm_resident_config(n_msm)
            if args.tables:
                nt = args.tables
        if args.msm_rounds >= 0:
            zk.msm.set_affine_rounds(args.msm_rounds)
        bases = zk.msm.ResidentBases(points, window=win, n_tables=nt)
        ws = bases.workspace()
        res = torch.zeros(16, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    def ntt_step():
        # the library's forward transform: register passes with the Shoup twiddle table
        zk.ntt.ntt_ex(x, tw, stream=stream, shoup=tw_shoup)

    def ssip_step():
        # the reference-ABI entry (Montgomery root table only), timed separately below
        zk.ntt.ssip_ntt(x, tw, stream)

    def msm_step():
        bases.msm(scalars, res, ws, stream)

    # ---- warm-up, then the timed region: K steps between barriers + syncs
    for _ in range(args.warmup):
        ntt_step()
        msm_step()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ntt_ms, msm_ms = 0.0, 0.0
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(args.steps):
            ntt_step()
        ev[1].record(stream)
        for _ in range(args.steps):
            msm_step()
        ev[2].record(stream)
        torch.cuda.synchronize()
    ntt_ms = ev[0].elapsed_time(ev[1]) / args.steps
    msm_ms = ev[1].elapsed_time(ev[2]) / args.steps
    step_ms = ntt_ms + msm_ms
    # the timed region's own results, kept for the bit-exact check against the CPU port: the
    # MSM result of the last timed step, and the vector the warm-up + timed in-place
    # transforms left behind
    timed_out = None
    if rank == 0 and not args.no_verify:
        timed_out = {"msm": res.cpu().numpy().view(np.uint64).copy(),
                     "ntt": x.values.cpu().numpy().view(np.uint64).reshape(n_ntt, 4).copy(),
                     "ntt_transforms": args.warmup + args.steps}
    # the same transform through ssip_ntt (every rank runs it, outside the timed region)
    for _ in range(2):
        ssip_step()
    ev[0].record(stream)
    for _ in range(args.steps):
        ssip_step()
    ev[1].record(stream)
    torch.cuda.synchronize()
    ssip_ms = ev[0].elapsed_time(ev[1]) / args.steps
    if world > 1:
        ntt_ms, msm_ms, ssip_ms = max_over_ranks([ntt_ms, msm_ms, ssip_ms], dev)
        step_ms = ntt_ms + msm_ms

    # ---- per-kernel timing from the libraries' own stream events (separate, untimed runs)
    native.profile_enable("libntt.so", True)
    pass_ms = []
    for _ in range(3):
        ntt_step()
        prof = native.profile_read("libntt.so")
        pass_ms += [ms for name, ms in prof if name == "ntt_pass"]
        bitrev_ms = [ms for name, ms in prof if name == "bitrev"]
    native.profile_enable("libntt.so", False)
    native.profile_enable("libmsm.so", True)
    stages = {}
    for _ in range(3):
        msm_step()
        for name, ms in native.profile_read("libmsm.so"):
            stages.setdefault(name, []).append(ms)
    native.profile_enable("libmsm.so", False)
    stage_ms = {k: statistics.median(v) for k, v in stages.items()}

    # ---- plain Pippenger over one table (no precomputation): the 2^22 bench size and the 2^20
    # size of the plain-MSM configuration, device-resident inputs, CUDA events
    one_table = measure_one_table_msm(zk, scalars, points, stream) if rank == 0 else None

    # ---- IMAD peak probe (measured on this GPU)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    probe_out = torch.empty(sms * 8 * 256, dtype=torch.int32, device=dev)
    lib_msm = native.load("libmsm.so")
    iters = 4096
    lib_msm.zkp_imad_probe(sms * 8, iters, probe_out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(5):
        lib_msm.zkp_imad_probe(sms * 8, iters, probe_out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    imad_per_s = 5 * sms * 8 * 256 * iters * 16 / (e0.elapsed_time(e1) / 1e3)

    # ---- Montgomery-product peak (the library's own product routine, measured on this GPU)
    mont_out = torch.empty(sms * 8 * 256 * 8, dtype=torch.int32, device=dev)
    mont_iters = 1024
    lib_msm.zkp_mont_probe(sms * 8, mont_iters, mont_out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(5):
        lib_msm.zkp_mont_probe(sms * 8, mont_iters, mont_out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    mont_per_s = 5 * sms * 8 * 256 * mont_iters * 2 / (e0.elapsed_time(e1) / 1e3)
    # ---- Shoup twiddle-product peak (the product of the NTT register passes)
    lib_ntt = native.load("libntt.so")
    lib_ntt.zkp_ntt_shoup_probe(sms * 8, mont_iters, mont_out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(5):
        lib_ntt.zkp_ntt_shoup_probe(sms * 8, mont_iters, mont_out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    shoup_per_s = 5 * sms * 8 * 256 * mont_iters * 2 / (e0.elapsed_time(e1) / 1e3)

    # ---- fused quotient kernel on the 2^24 extended coset (its HBM and product rooflines)
    fused = measure_fused(zk, gen, dev, stream, hbm_peak=peaks()[0],
                          mont_peak=mont_per_s, shoup_peak=shoup_per_s) if not args.no_fused else None

    # ---- poly library rows (evaluation, batched inversion, division by X - b)
    poly = measure_poly(zk, gen, dev, stream, hbm_peak=peaks()[0], mont_peak=mont_per_s) \
        if not args.no_fused else None
    # ---- the pipelined fused kernel over host-resident polynomials
    pipelined = measure_pipelined(zk, gen) if (not args.no_fused and rank == 0) else None

    # ---- batched form (mixed NTT/MSM workload) and served form (Poisson arrivals)
    batched = measure_batched(zk, args) if (not args.no_batched and rank == 0) else None
    served = measure_served(zk, bases, args) if (not args.no_served and rank == 0) else None

    # ---- e2e through the reference C ABI from pinned host memory
    e2e_msm_s = e2e_ntt_s = float("nan")
    e2e_out = None
    if not args.no_e2e:
        e2e_msm_s, e2e_ntt_s, e2e_out = run_e2e(zk, native, lib_msm, scalars, points, ntt_in, tw, stream, dev,
                                                local, args, n_msm, n_ntt)

    # ---- CPU baseline (rank 0 at N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference(args.ref_msm_log, args.ref_ntt_log)
    # ---- the timed and e2e results against the CPU port, bit for bit (rank 0)
    verified = None
    if timed_out is not None:
        verified = verify_outputs(cpu, timed_out, e2e_out if rank == 0 else None)
    emit(args, zk, rank, world, n_msm, n_ntt, ntt_ms, msm_ms, step_ms, pass_ms, bitrev_ms, stage_ms, imad_per_s,
         e2e_msm_s, e2e_ntt_s, cpu, clocks, bases, batched, served, fused, mont_per_s, poly, pipelined,
         ssip_ms, shoup_per_s, verified, one_table)


def measure_one_table_msm(zk, scalars, points, stream, reps=3):
    """zkp_msm_device over the plain bases (one table, the tuned one-table window, the library's
    pairing rounds) at the bench's MSM size and at 2^20, on prefixes of the same inputs."""
    import torch
    lib = zk.native.load("libmsm.so")
    out = {}
    for log_n in sorted({MSM_LOG, 20}):
        n = 1 << log_n
        if n > points.shape[0]:
            continue
        w = zk.tuner.msm_window(n)
        ws = torch.empty(zk.msm.workspace_size(n, w), dtype=torch.uint8, device=points.device)
        res = torch.zeros(16, dtype=torch.int32, device=points.device)

        def run():
            zk.native.check(lib.zkp_msm_device(ws.data_ptr(), ws.numel(), points.data_ptr(), 1, scalars.data_ptr(),
                                               n, w, res.data_ptr(), stream.cuda_stream), "zkp_msm_device")
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[f"2^{log_n}"] = {"ms": ms, "points_per_s": n / (ms / 1e3), "window": w or zk.msm.default_window(n),
                             "pairing_rounds": zk.msm.rounds_for(n, w, 1)}
        del ws
    torch.cuda.empty_cache()
    return out


def measure_fused(zk, gen, dev, stream, hbm_peak, mont_peak, shoup_peak, log_n=NTT_LOG, ext=3, reps=10):
    """q = (a*b - c - z*z(wX)) * Z_H^-1 over 2^log_n coset points (distinct a, b, c, z): 4 reads +
    1 write of 32 B per element (z(wX) is the same z one row on, served from cache) and 3 products
    (a*b, z*z(wX): Montgomery; the product with the periodic 1/Z_H: Shoup's, a fixed factor)."""
    import torch
    n = 1 << log_n
    with torch.cuda.stream(stream):
        a, b, c, z = (zk.ScalarArray(gen.fr(600 + i, n, dev)) for i in range(4))
        q = zk.ScalarArray.alloc(n, dev)
    zh = zk.pipeline.zh_inv_device(log_n - ext, ext, dev)
    kern = zk.fused.quotient_kernel()
    args_ = ([q], [a, b, c, z, zk.pipeline.rotated(z, ext), zh])
    torch.cuda.synchronize()
    for _ in range(3):
        kern(*args_, stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        kern(*args_, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    gbs = 160 * n / (ms / 1e3) / 1e9
    mults = 3 * n
    # time at the measured product peaks: two Montgomery products and one Shoup product per element
    floor_s = 2 * n / mont_peak + n / shoup_peak
    out = {"kernel": "zkp_quotient_z8_kernel (generated fused kernel)", "n": n, "ms": ms,
           "achieved_gbs": gbs, "hbm_peak_gbs": hbm_peak, "hbm_frac": gbs / hbm_peak,
           "fr_mults_per_s": mults / (ms / 1e3), "product_frac": floor_s / (ms / 1e3),
           "product_frac_note": "time of 2 Montgomery + 1 Shoup products per element at their measured peaks "
                                "/ kernel time",
           "bytes_per_elem": 160, "fr_mults_per_elem": 3}
    del a, b, c, z, q
    torch.cuda.empty_cache()
    return out


def measure_pipelined(zk, gen, log_n=22, parts=8, reps=5):
    """The pipelined fused kernel (host polynomials streamed through the device in chunks,
    libzkp_pipeline.so) on the quotient-shaped graph over 2^log_n host-resident points: five
    input polynomials and a periodic 1/Z_H in, one polynomial out, against the one-shot path
    (copy everything in, one kernel, copy the result out).  Host clock (the call blocks)."""
    import time
    import torch
    n = 1 << log_n
    g = zk.fused.FusedGraph([
        ("input", "a", "poly", "var", 0), ("input", "b", "poly", "var", 1), ("input", "c", "poly", "var", 2),
        ("input", "z", "poly", "var", 3), ("input", "zw", "poly", "var", 4), ("input", "zh", "periodic", "var", 5),
        ("mul", "ab", "a", "b"), ("sub", "t0", "ab", "c"), ("mul", "zz", "z", "zw"), ("sub", "t1", "t0", "zz"),
        ("mul", "q", "t1", "zh"), ("output", 0, "q")])
    op = zk.fused.FusedOp(g, "zkp_quotient_plain_inputs")
    ins = [gen.fr(800 + i, n).cpu().pin_memory() for i in range(5)] + [gen.fr(805, 8).cpu().pin_memory()]
    out = torch.empty((n, 8), dtype=torch.int32).pin_memory()
    pk = zk.fused.PipelinedFusedKernel(op, parts)
    kern = zk.fused.FusedKernel(op)
    dev_in = [zk.ScalarArray(t.cuda()) for t in ins]
    dev_out = zk.ScalarArray.zeros(n)

    def one_shot():
        for d, h in zip(dev_in, ins):
            d.values.copy_(h, non_blocking=True)
        kern([dev_out], dev_in)
        out.copy_(dev_out.values, non_blocking=True)
        torch.cuda.synchronize()

    def timed(fn):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t0) / reps

    t_pipe = timed(lambda: pk([out], ins, n))
    t_one = timed(one_shot)
    host_bytes = 5 * n * 32 + n * 32
    return {"n": n, "parts": parts, "ms": t_pipe * 1e3, "elems_per_s": n / t_pipe,
            "host_link_gbs": host_bytes / t_pipe / 1e9, "one_shot_ms": t_one * 1e3,
            "speedup_vs_one_shot": t_one / t_pipe,
            "device_bytes": pk.workspace.numel(), "one_shot_device_bytes": 6 * n * 32,
            "note": "host-resident operands over PCIe; the chunked form needs 5 parts' worth of device "
                    "buffers per operand set instead of the whole polynomials"}


def measure_poly(zk, gen, dev, stream, hbm_peak, mont_peak, log_n=22, reps=10):
    """poly_eval, batched_invert and kate_division over 2^log_n elements (inputs larger than L2):
    CUDA-event time per call, algorithmic bytes and Montgomery products per element as each
    kernel's cost model below states."""
    import torch
    n = 1 << log_n
    with torch.cuda.stream(stream):
        p = zk.ScalarArray(gen.fr(900, n, dev))
        x = gen.fr(901, 1, dev)
        res = torch.zeros(8, dtype=torch.int32, device=dev)
        inv = zk.ScalarArray(gen.fr(902, n, dev))
        q = zk.ScalarArray.zeros(n, dev)
    torch.cuda.synchronize()
    # (name, call, algorithmic bytes per element, algorithmic products per element): Horner
    # evaluation reads each coefficient once with one product; Montgomery's batched inversion
    # reads and writes each element with three products; division by X - b reads p, writes q,
    # one product per coefficient
    cases = [
        ("poly_eval", lambda: zk.poly.poly_eval(p, x, res, stream=stream), 32, 1),
        ("batched_invert", lambda: zk.poly.batched_invert(inv, stream=stream), 64, 3),
        ("kate_division", lambda: zk.poly.kate_division(p, x, q, stream=stream), 64, 1),
    ]
    # permute (lookup-argument permutation) over 2^20 rows, shaped like the reference's test
    # (core/tests/poly.rs:569-625): table values uniform below 2n, inputs drawn from the table's
    # distinct usable values, 25 unusable rows; small integers converted to Montgomery form
    import numpy as np
    m = 1 << 20
    usable = m - 25
    rng = np.random.default_rng(7)
    tab = rng.integers(0, 2 * m, m, dtype=np.uint64)
    distinct = np.unique(tab[:usable])
    inp = distinct[rng.integers(0, len(distinct), m)]
    r2 = zk.ScalarArray.from_numpy(np.array(zk.field.mont_words((1 << 256) % zk.field.FR_MODULUS),
                                            dtype=np.uint32).reshape(1, 8))
    lookup = []
    for vals in (inp, tab):
        limbs = np.zeros((m, 8), dtype=np.uint32)
        limbs[:, 0] = vals.astype(np.uint32)
        arr = zk.ScalarArray.from_numpy(limbs)
        zk.ntt.distribute_powers(arr, r2)
        lookup.append(arr)
    ri, rt = zk.ScalarArray.alloc(usable), zk.ScalarArray.alloc(usable)
    torch.cuda.synchronize()
    out = {"n": n}
    # permute: reads input and table (64 B a row), writes both outputs (64 B); no field products
    # beyond the conversions in and out of Montgomery form
    perm = ("permute", lambda: zk.poly.permute(lookup[0], lookup[1], usable, ri, rt, stream=stream), 128, 0)
    for name, call, bpe, mpe in cases + [perm]:
        rows = usable if name == "permute" else n
        for _ in range(2):
            call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": ms, "elems_per_s": rows / (ms / 1e3), "bytes_per_elem": bpe,
                     "hbm_frac": bpe * rows / (ms / 1e3) / 1e9 / hbm_peak, "fr_mults_per_elem": mpe,
                     "mont_frac": mpe * rows / (ms / 1e3) / mont_peak}
    out["permute"]["rows"] = usable
    del p, inv, q, lookup, ri, rt
    torch.cuda.empty_cache()
    return out


def measure_batched(zk, args, reps=3):
    """64 NTTs (log2 n uniform on 10..20, forward / inverse / coset) + 16 MSMs (log2 n uniform
    on 12..22), seed 3: per-call path vs one captured graph of the batched launches."""
    import torch
    import time
    w = zk.batched.MixedWorkload(seed=3)
    w.build_batched()
    # per-call path through the reference ABI (host arrays for the MSMs), host-clock timed:
    # each msm call returns its result to the host
    w.run_plain_ref_abi()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        w.run_plain_ref_abi()
    torch.cuda.synchronize()
    ref_ms = (time.perf_counter() - t0) * 1e3 / reps
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    w.run_plain()
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(reps):
        w.run_plain()
    ev[1].record()
    torch.cuda.synchronize()
    w.run_batched()
    torch.cuda.synchronize()
    ev[2].record()
    for _ in range(reps):
        w.run_batched()
    ev[3].record()
    torch.cuda.synchronize()
    plain_ms = ev[0].elapsed_time(ev[1]) / reps
    bat_ms = ev[2].elapsed_time(ev[3]) / reps
    # the per-call path over the batch's own tables (Shoup twiddles, resident table sets)
    w.run_plain_same_tables()
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(reps):
        w.run_plain_same_tables()
    ev[1].record()
    torch.cuda.synchronize()
    same_ms = ev[0].elapsed_time(ev[1]) / reps
    work = w.work()
    out = {"workload": "64 NTTs 2^10..2^20 (fwd/inv/coset) + 16 MSMs 2^12..2^22, seed 3",
           "ntt_logs": w.ntt_logs, "msm_logs": w.msm_logs, "msm_windows_plain": w.windows,
           "msm_resident_configs": [list(zk.tuner.msm_resident_config(1 << L)) for L in w.msm_logs],
           "plain_ref_abi_ms": ref_ms, "plain_device_ms": plain_ms, "batched_ms": bat_ms,
           "plain_same_tables_ms": same_ms,
           "speedup": ref_ms / bat_ms, "speedup_vs_plain_device": plain_ms / bat_ms,
           "speedup_vs_plain_same_tables": same_ms / bat_ms,
           "tasks_per_s_plain_ref_abi": work["tasks"] / (ref_ms / 1e3),
           "tasks_per_s_plain_device": work["tasks"] / (plain_ms / 1e3),
           "tasks_per_s_batched": work["tasks"] / (bat_ms / 1e3),
           "plain_ref_abi": "ssip_ntt / zkp_ntt_ex per transform on device buffers; one reference-ABI msm call per "
                            "MSM with pinned host scalars and host bases (one table), host result",
           "plain_device": "same order, zkp_msm_device per MSM over device-resident bases (one table)",
           "plain_same_tables": "same order, zkp_ntt_ex_shoup per transform and a one-task MSM batch per MSM over "
                                "the batch's own resident table sets (everything but the batching)",
           "work": work}
    del w
    torch.cuda.empty_cache()
    return out


def measure_served(zk, bases, args):
    """Poisson arrivals (50 req/s, k uniform on 14..22) of the prover-shaped program; the served
    form (continuous batching, 8 slots, HBM admission) vs the plain path (one request at a time)."""
    import torch
    sched = zk.serving.poisson_schedule(args.served_requests, rate=50.0, k_lo=14, k_hi=22, seed=5)
    out = {"workload": f"{args.served_requests} requests, Poisson 50 req/s, k uniform 14..22, program = "
                       "3 INTT + coset NTT 4x + fused quotient + 4 MSM (one batch) + 2 evals",
           "hbm_arena_gb": 48}
    burst = [(0.0, k, seed) for _, k, seed in sched[:120]]  # 120 requests at once: capacity
    # resident bases with the tuned (window, tables) per size range
    sets = zk.serving.resident_sets(bases.tables[: bases.n], 14, 22)
    out["table_sets"] = [{"max_k": mk, "window": rb.window, "tables": rb.n_tables} for rb, mk in sets]
    # the served form's admission policy: at most one request of size >= 2^21 in flight (the
    # latency tail is made of the largest requests; smaller ones are admitted past a waiting one)
    policy = {"priority_k": 0, "large_k": 21, "max_large_inflight": 1}
    out["policy"] = policy
    for name, inflight, pol in (("served", 8, policy), ("served_no_policy", 8, {}), ("served_1_slot", 1, {})):
        srv = zk.serving.Server(sets, hbm_bytes=48 << 30, max_inflight=inflight, ext_log=2, min_k=14, max_k=22)
        srv.set_policy(**pol)
        # warm the constants / kernels once
        srv.wait(srv.submit(14, 1))
        _, summary = zk.serving.run_schedule(srv, sched)
        out[name] = summary
        _, out[name.replace("served", "served_capacity", 1)] = zk.serving.run_schedule(srv, burst)
        srv.close()
    out["served_compiled"] = measure_served_compiled(zk, sets, sched, burst, policy)
    prover = zk.serving.PerCallProver(bases, ext_log=2, max_k=22)
    del sets
    prover.warm(range(14, 23))
    prover.run(14, 1)
    torch.cuda.synchronize()
    _, out["plain"] = zk.serving.run_schedule_per_call(prover, sched)
    _, out["plain_capacity"] = zk.serving.run_schedule_per_call(prover, burst)
    out["plain_path"] = ("one request at a time; INTT/coset/fused/eval through their per-call entry points, the "
                         "4 MSMs through the reference-ABI msm call with host scalars and host bases")
    out["capacity_speedup"] = out["served_capacity"]["req_per_s"] / out["plain_capacity"]["req_per_s"]
    del prover
    torch.cuda.empty_cache()
    return out


def measure_served_compiled(zk, sets, sched, burst, policy, k_lo=14, k_hi=22, ext=2):
    """The served workload with every request a compiled program: the prover program of each
    size written in the reference's artifact forms (program.prover_artifact), lowered once and
    registered with an 8-slot server; its MSMs use the same resident table sets.  Unlike the
    built-in program, which draws its inputs on the device, a compiled request reads its inputs
    from pinned host buffers (LoadInput + Transfer), one input set per size.  One request per
    size is checked against the built-in program on the same inputs."""
    import numpy as np
    import torch
    import time
    P = zk.program
    srv = zk.serving.Server(sets, hbm_bytes=48 << 30, max_inflight=8, ext_log=ext, min_k=k_lo, max_k=k_hi)
    srv.set_policy(**policy)
    progs, inputs = {}, {}
    t0 = time.perf_counter()
    for k in range(k_lo, k_hi + 1):
        rb = next(rb for rb, mk in sets if k <= mk)
        parts = P.prover_artifact(k, P.prover_constants(k, ext, rb.tables[: rb.n]), ext=ext)
        progs[k] = P.CompiledProgram.from_parts(srv, parts[1], parts[3], P.prover_input_types(k, ext),
                                                fused=P.prover_fused_graphs(), bases={"bases": rb})
        n, N = 1 << k, 1 << (k + ext)
        # the inputs of the built-in request (k, seed = k): a, b, c, z, x from seed*8 + i
        inputs[k] = [zk.gen.fr(k * 8 + i, m).cpu().pin_memory() for i, m in enumerate((n, n, n, N, 1))]
    load_s = time.perf_counter() - t0
    same = True
    for k in range(k_lo, k_hi + 1):
        r, leaves = progs[k].wait(progs[k].submit(inputs[k]))
        ref = srv.wait(srv.submit(k, k))
        got = np.concatenate([np.asarray(x, dtype=np.uint32).reshape(-1) for x in leaves])
        same = same and r.status == 0 and ref.status == 0 and np.array_equal(got, zk.serving.result_words(ref))

    def submit(k, seed):
        return progs[k], progs[k].submit(inputs[k])

    def wait(h):
        return h[0].wait(h[1])[0]

    _, summary = zk.serving.run_schedule(srv, sched, submit=submit, wait=wait)
    _, cap = zk.serving.run_schedule(srv, burst, submit=submit, wait=wait)
    out = {"served": summary, "served_capacity": cap, "matches_builtin": same,
           "programs": {k: {"ops": p.n_ops, "device_bytes": p.device_bytes, "host_bytes": p.host_bytes}
                        for k, p in progs.items()},
           "load_s": load_s,
           "path": "reference-form prover artifacts (instruction chunk + constant table) lowered by program.py to "
                   "zkp_serve_program ops; inputs copied from pinned host memory inside each request"}
    for p in progs.values():
        p.close()
    srv.close()
    del progs, inputs
    torch.cuda.empty_cache()
    return out


def run_e2e(zk, native, lib_msm, scalars, points, ntt_in, tw, stream, dev, local, args, n_msm, n_ntt):
    import ctypes
    import numpy as np
    import torch
    h_scal = scalars.cpu().pin_memory()
    h_pts = points.cpu().pin_memory()
    h_ntt = ntt_in.cpu().pin_memory()
    h_out = torch.empty_like(h_ntt).pin_memory()
    cfg = zk.msm.MsmConfig(cards=[local])
    sizes = zk.msm.MSM(cfg).get_buffer_size(n_msm)
    buf = torch.empty(sizes[0], dtype=torch.uint8, device=dev)
    ptrs = (ctypes.c_void_p * 1)(buf.data_ptr())
    cards = (ctypes.c_uint * 1)(local)
    hp = (ctypes.c_void_p * 1)(h_pts.data_ptr())
    hs = (ctypes.c_void_p * 1)(h_scal.data_ptr())
    result = np.zeros(16, dtype=np.uint32)
    hr = (ctypes.c_void_p * 1)(result.ctypes.data)
    x_e2e = zk.ScalarArray.alloc(n_ntt, dev)

    def e2e_msm():
        native.check(lib_msm.msm(ptrs, None, n_msm, 1, 1, 1, 1, 1, cards, hp, 1, hs, hr), "msm")

    def e2e_ntt():
        x_e2e.values.copy_(h_ntt, non_blocking=True)
        zk.ntt.ssip_ntt(x_e2e, tw, stream)
        h_out.copy_(x_e2e.values, non_blocking=True)

    with torch.cuda.stream(stream):
        for _ in range(max(1, args.warmup // 2)):
            e2e_msm()
            e2e_ntt()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_msm()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(args.steps):
            e2e_ntt()
        stream.synchronize()
        t2 = time.perf_counter()
    # the last e2e call's results, as the caller received them in host memory
    outs = {"msm": result.view(np.uint64).copy(), "ntt": h_out.numpy().view(np.uint64).reshape(n_ntt, 4).copy()}
    return (t1 - t0) / args.steps, (t2 - t1) / args.steps, outs


def emit(args, zk, rank, world, n_msm, n_ntt, ntt_ms, msm_ms, step_ms, pass_ms, bitrev_ms, stage_ms, imad_per_s,
         e2e_msm_s, e2e_ntt_s, cpu, clocks, bases, batched=None, served=None, fused=None, mont_per_s=None,
         poly=None, pipelined=None, ssip_ms=None, shoup_per_s=None, verified=None, one_table=None):
    import torch
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    hbm_peak, peak_kind = peaks()
    pass_avg = statistics.median(pass_ms)
    # one transform's passes (the last one fused with the bit reversal where the plan allows):
    # the profiling runs record every pass of each transform
    pass_total = sum(pass_ms) / max(1, len(pass_ms) // max(1, len(zk.ntt.plan_digits(NTT_LOG))))
    ntt_bytes_per_pass = 64 * n_ntt  # one read + one write of every element per pass
    ntt_alg_bytes = 64 * n_ntt       # algorithmic bytes of the whole transform
    ntt_alg_gbs = ntt_alg_bytes / (ntt_ms / 1e3) / 1e9
    # bucket accumulation = the affine pairing rounds (pair_*) + the XYZZ walk (accumulate)
    acc_ms = sum(v for k, v in stage_ms.items() if k.startswith("pair_") or k == "accumulate")
    c_msm = bases.window
    w_msm = (254 + c_msm - 1) // c_msm
    rounds = zk.msm.rounds_for(n_msm, bases.window, bases.n_tables)
    # executed Fq products of the accumulation: a pairing round adds about half of its list's
    # points pairwise at 6 products a pair (3 for the shared inversion, slope, square, new y);
    # the walk adds the rest at 10 (mixed XYZZ addition: 8 products + 2 squarings)
    entries = n_msm * w_msm
    acc_mults = 0
    for _ in range(rounds):
        acc_mults += 6 * (entries // 2)
        entries -= entries // 2
    acc_mults += 10 * entries
    # the algorithm-independent accounting of the MSM's work (fixed c = 16: 16 windows x 10
    # products per point, plus 2 full additions of 14 products per bucket of 16 windows)
    msm_mults = 160 * n_msm + 2 * (1 << 15) * 16 * 14
    imad_per_mult = 264
    msm_total_ms = sum(stage_ms.values())
    digits = zk.ntt.plan_digits(NTT_LOG)
    # algorithmic Fr products of a radix-2 transform: n/2 twiddle products in each of the
    # log2(n) - 1 stages that have non-trivial twiddles (independent of the pass split)
    ntt_mults = (n_ntt // 2) * (NTT_LOG - 1)
    launches_per_ntt = zk.ntt.num_passes(NTT_LOG)
    # sort (count, 3 scan, scatter), walk (accumulate, fixup, long chains), reduction (segment,
    # classes, window), combine, zero results = 13; a pairing round: halve, 3 scan, up, tree
    # (one level + top + one level at these sizes), down = 9
    launches_per_msm = 13 + 9 * rounds
    line = {
        "metric": METRIC, "value": world * n_msm / (msm_ms / 1e3), "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (BN254 Montgomery limbs, exact)",
        "data": "synthetic (seeded counter-based generator; points k_i*G)",
        "config": workload_config(world),
        "msm": {"metric": f"MSM points/s (2^{MSM_LOG})", "value": world * n_msm / (msm_ms / 1e3),
                "ms": msm_ms, "stages_ms": stage_ms, "window": bases.window, "tables": bases.n_tables,
                "pairing_rounds": rounds,
                "path": f"resident bases with {bases.n_tables} precomputed tables of 2^{MSM_LOG} points, window "
                        f"{bases.window}, {rounds} affine pairing rounds; tables built once outside the timed "
                        f"region"},
        "ntt": {"metric": f"NTT elems/s (2^{NTT_LOG})", "value": world * n_ntt / (ntt_ms / 1e3), "unit": "elems/s",
                "ms": ntt_ms, "pass_ms": pass_avg, "bitrev_ms": statistics.median(bitrev_ms) if bitrev_ms else None,
                "hbm_frac_whole_ntt": (64 * n_ntt / (ntt_ms / 1e3) / 1e9) / hbm_peak,
                "path": "zkp_ntt_ex_shoup: register passes with Shoup twiddle products (root table + Shoup "
                        "table of 64 B per root, both built once outside the timed region)",
                "ssip_ms": ssip_ms, "ssip_value": world * n_ntt / (ssip_ms / 1e3) if ssip_ms else None,
                "ssip_path": "ssip_ntt (reference ABI): the same passes with Montgomery twiddle products"},
        # the NTT's HBM roofline: 64 B per element (one read + one write
        # of the vector) for the whole transform, over the transform's CUDA-event time
        "roofline": {"kernel": f"NTT 2^{NTT_LOG} forward transform: {len(digits)} register passes "
                               f"(ntt_warp_pass_kernel, the last fused with the bit reversal in "
                               f"ntt_last_bitrev_kernel), digits {digits}, Shoup twiddle products",
                     "bound": "imad", "achieved": ntt_alg_gbs, "peak": hbm_peak, "unit": "GB/s",
                     "frac": ntt_alg_gbs / hbm_peak, "peak_source": peak_kind,
                     "bytes_per_launch": ntt_alg_bytes, "launch": "one whole transform (all passes)",
                     # ncu DRAM bytes of all passes of one transform, per element, scaled to 2^24
                     "traffic": NTT_TRAFFIC_PER_ELEM * n_ntt,
                     "frac_per_pass": ntt_bytes_per_pass / (pass_avg / 1e3) / 1e9 / hbm_peak,
                     "frac_per_pass_note": "64 B per element for ONE pass over the median pass time: every pass "
                                           "reads and writes the vector, so this credits each pass with the "
                                           "transform's algorithmic bytes",
                     "note": "bound by the integer multiply pipe, not HBM: the twiddle products at the measured "
                             "Shoup-product peak take longer than the vector's HBM traffic; the binding fraction "
                             "is int_roofline.ntt_passes.frac"},
        "int_roofline": {
            # denominator: Montgomery products per second of the library's own product routine
            # (zkp_mont_probe, measured in this run); the raw IMAD rate is listed beside it
            "mont_mul_peak_per_s": mont_per_s, "peak_source": "measured (zkp_mont_probe)",
            "imad_peak_per_s": imad_per_s, "imad_per_mont_mul": imad_per_mult,
            "msm_accumulate": {"kernels": f"{rounds} affine pairing rounds (pair_up / tree / pair_down) + "
                                          "accumulate_kernel walk",
                               "ms": acc_ms, "fq_mults_executed": acc_mults,
                               "fq_mults_per_s": acc_mults / (acc_ms / 1e3),
                               "frac": (acc_mults / (acc_ms / 1e3)) / mont_per_s},
            "msm_whole": {"fq_mults_accounted": msm_mults, "ms": msm_total_ms,
                          "accounting": "160 n + 2 * 2^15 * 16 * 14 (c = 16 mixed-addition count), "
                                        "independent of the window and of the pairing rounds",
                          "frac": (msm_mults / (msm_total_ms / 1e3)) / mont_per_s},
            # the register passes multiply by fixed twiddles with Shoup's product; their
            # denominator is that product's own peak (zkp_ntt_shoup_probe, measured in this run)
            "shoup_mul_peak_per_s": shoup_per_s,
            "ntt_passes": {"digits": digits, "fr_mults": ntt_mults, "ms": pass_total,
                           "fr_mults_per_s": ntt_mults / (pass_total / 1e3),
                           "frac": (ntt_mults / (pass_total / 1e3)) / shoup_per_s,
                           "peak": "shoup_mul_peak_per_s"},
        },
        "e2e": {"value": world * n_msm / e2e_msm_s if e2e_msm_s == e2e_msm_s else None, "unit": "points/s",
                "h2d_bytes_per_step": n_msm * (64 + 32) + n_ntt * 32, "d2h_bytes_per_step": 64 + n_ntt * 32,
                "ntt_elems_per_s": world * n_ntt / e2e_ntt_s if e2e_ntt_s == e2e_ntt_s else None,
                "path": "msm(): reference C ABI, host tables in, host result out; ssip_ntt with H2D/D2H"},
        "gpu_launches": args.steps * (launches_per_ntt + launches_per_msm),
        "clocks": clocks.summary(),
    }
    if fused:
        line["fused"] = fused
    if poly:
        line["poly"] = poly
    if pipelined:
        line["fused_pipelined"] = pipelined
    if batched:
        line["batched"] = batched
    if served:
        line["served"] = served
    if one_table:
        line["msm"]["one_table"] = one_table
        line["msm"]["one_table_note"] = ("plain Pippenger without precomputed tables (zkp_msm_device, device-resident "
                                         "inputs), outside the timed region")
    if verified is not None:
        line["verified"], line["verification"] = verified
    if cpu:
        line["cpu_baseline"] = {"value": cpu["msm_points_per_s"], "unit": "points/s", "cores": cpu["cores"],
                                "kind": "port", "sample": cpu["msm_sample"] + "; " + cpu["ntt_sample"],
                                "ntt_elems_per_s": cpu["ntt_elems_per_s"], "cpu": cpu_model()}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--window", type=int, default=0)
    ap.add_argument("--tables", type=int, default=0, help="precomputed point tables (0 = tuned / full)")
    ap.add_argument("--msm-rounds", type=int, default=-1,
                    help="affine pairing rounds of the MSM (-1 = the library's choice by size)")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-fused", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-requests", type=int, default=400)
    ap.add_argument("--ref-msm-log", type=int, default=22)
    ap.add_argument("--ref-ntt-log", type=int, default=24)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer C-ABI leg (profiling runs)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own CUDA kernels (oracle/_ref)")
    ap.add_argument("--no-verify", action="store_true",
                    help="skip the bit-exact check of the timed results against the CPU port (profiling runs)")
    ap.add_argument("--ntt-log", type=int, default=24)
    ap.add_argument("--msm-log", type=int, default=22)
    args = ap.parse_args()
    global MSM_LOG, NTT_LOG
    MSM_LOG, NTT_LOG = args.msm_log, args.ntt_log
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
