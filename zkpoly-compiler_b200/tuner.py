"""Project-written autotuner: measures candidate kernel parameters on the device and caches the
winners per GPU model (in the role of the reference's core/src/msm/tuning/cost_model.py, which
predicts a window from relative cost coefficients instead of measuring).

Tuned parameters:
  - MSM window width c in [8, 20] per log2 n (zkp_msm_device timed on seeded inputs);
  - MSM (window, precomputed tables) for resident bases per log2 n;
  - MSM block shapes: the CTA size of the pairing rounds' up and down passes and of the XYZZ
    walk (zkp_msm_set_block), by coordinate descent at the resident 2^22 configuration;
  - NTT largest digit (sub-transform size 2^D, which sets the pass split and the CTA shape)
    per log2 n (zkp_ntt_set_max_digit, timed on seeded inputs);
  - NTT block shape: the CTA size of the register passes per log2 n (zkp_ntt_set_block).
The cache is a JSON file next to the libraries.  Below it sit the shipped defaults
(tuning_defaults.json, winners this tuner measured on B200); without an entry in either the
libraries' own cost model / default plan is used.
"""
from __future__ import annotations

import json
import os
import threading

import torch

from .native import check, load

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "lib", "tuning.json")
DEFAULTS = os.path.join(HERE, "tuning_defaults.json")
_lock = threading.Lock()
_cache: dict | None = None


def _device_key() -> str:
    return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"


def _load() -> dict:
    global _cache
    if _cache is None:
        _cache = {}
        for path in (DEFAULTS, CACHE):  # measured entries override the shipped ones
            try:
                with open(path) as f:
                    data = json.load(f)
            except (OSError, ValueError):
                continue
            for dev, kinds in data.items():
                for kind, table in kinds.items():
                    _cache.setdefault(dev, {}).setdefault(kind, {}).update(table)
    return _cache


def _save():
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    tmp = CACHE + ".tmp"
    with open(tmp, "w") as f:
        json.dump(_cache, f, indent=1, sort_keys=True)
    os.replace(tmp, CACHE)


def msm_window(n: int) -> int:
    """Tuned window for n points (one table) if known, else 0 (the library's cost model)."""
    log_n = max(1, (n - 1).bit_length())
    entry = _load().get(_device_key(), {}).get("msm_window", {}).get(str(log_n))
    return int(entry) if entry else 0


def msm_resident_config(n: int):
    """(window, n_tables) for resident bases of n points: the tuned pair if known, else full
    precomputation (one table per window, so no doubling chain between windows) at c = 16."""
    log_n = max(1, (n - 1).bit_length())
    entry = _load().get(_device_key(), {}).get("msm_resident", {}).get(str(log_n))
    if entry:
        return int(entry[0]), int(entry[1])
    c = resident_window_model(1 << log_n)
    return c, (254 + c - 1) // c


def resident_window_model(n: int) -> int:
    """Untuned window for full precomputation: minimises n * ceil(254 / c) bucket additions
    plus a bucket-reduction cost of 40 * 2^c (in the same unit, fitted to B200 timings at
    n = 2^22 where it picks c = 17)."""
    return min(range(8, 21), key=lambda c: n * ((254 + c - 1) // c) + 40 * (1 << c))


def _time(fn, reps=3) -> float:
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_msm(log_ns=range(12, 23), candidates=range(8, 21), bases=None) -> dict:
    from . import gen, msm
    lib = load(msm.LIB)
    nmax = 1 << max(log_ns)
    bases = bases if bases is not None else gen.points(2, nmax)
    out = {}
    for L in log_ns:
        n = 1 << L
        s = gen.fr(77, n)
        res = torch.zeros(16, dtype=torch.int32, device="cuda")
        best = None
        for c in candidates:
            ws = torch.empty(msm.workspace_size(n, c), dtype=torch.uint8, device="cuda")

            def run():
                check(lib.zkp_msm_device(ws.data_ptr(), ws.numel(), bases.data_ptr(), 1, s.data_ptr(), n, c,
                                         res.data_ptr(), torch.cuda.current_stream().cuda_stream), "zkp_msm_device")
            t = _time(run, reps=2 if L >= 20 else 3)
            del ws
            if best is None or t < best[1]:
                best = (c, t)
        out[str(L)] = best[0]
    with _lock:
        _load().setdefault(_device_key(), {})["msm_window"] = out
        _save()
    return out


def tune_ntt(log_ns=range(14, 25), candidates=(8, 9, 10, 11, 12), apply: bool = True, path: str = "shoup") -> dict:
    """Times a forward NTT of 2^L seeded elements for each digit cap (zkp_ntt_set_max_digit)
    and caches the fastest per size; with apply the winners are set in the library.  path
    "shoup" times the library's own transform (ntt.ntt: register passes with the Shoup twiddle
    table), "ssip" the reference-ABI ssip_ntt (Montgomery twiddle products); the caps are shared
    by both."""
    from . import gen, ntt
    from .scalar import ScalarArray
    assert path in ("shoup", "ssip")
    lib = load(ntt.LIB)
    out, times = {}, {}
    for L in log_ns:
        x = ScalarArray(gen.fr(79, 1 << L))
        tw = ntt.twiddle_table(L)
        run = (lambda: ntt.ntt(x)) if path == "shoup" else (lambda: ntt.ssip_ntt(x, tw))
        best = None
        for d in candidates:
            check(lib.zkp_ntt_set_max_digit(L, d), "zkp_ntt_set_max_digit")
            t = _time(run, reps=10 if L < 20 else 3)
            times[f"{L}:{d}"] = t
            if best is None or t < best[1]:
                best = (d, t)
        check(lib.zkp_ntt_set_max_digit(L, 0), "zkp_ntt_set_max_digit")
        out[str(L)] = best[0]
        del x
    with _lock:
        _load().setdefault(_device_key(), {})["ntt_max_digit"] = out
        _save()
    if apply:
        apply_ntt_plans()
    return {"best": out, "ms": times}


def apply_ntt_plans() -> None:
    """Sets the cached digit caps and register-pass CTA sizes (if any) for this GPU model in
    libntt.so."""
    from . import ntt
    dev = _load().get(_device_key(), {})
    lib = load(ntt.LIB)
    for L, d in dev.get("ntt_max_digit", {}).items():
        check(lib.zkp_ntt_set_max_digit(int(L), int(d)), "zkp_ntt_set_max_digit")
    for L, t in dev.get("ntt_block", {}).items():
        check(lib.zkp_ntt_set_block(int(L), int(t)), "zkp_ntt_set_block")


MSM_BLOCK_STAGES = ("pair_up", "pair_down", "accumulate")  # zkp_msm_set_block stage ids 0, 1, 2


def apply_msm_blocks() -> None:
    """Sets the cached MSM stage CTA sizes (if any) for this GPU model in libmsm.so."""
    from . import msm
    table = _load().get(_device_key(), {}).get("msm_block", {})
    lib = load(msm.LIB)
    for i, name in enumerate(MSM_BLOCK_STAGES):
        if name in table:
            check(lib.zkp_msm_set_block(i, int(table[name])), "zkp_msm_set_block")


def tune_ntt_blocks(log_ns=range(18, 25), candidates=(64, 128, 256)) -> dict:
    """Times the library's forward NTT of 2^L seeded elements (its tuned digit plan) for each
    register-pass CTA size and caches the fastest per size."""
    from . import gen, ntt
    from .scalar import ScalarArray
    lib = load(ntt.LIB)
    apply_ntt_plans()
    out, times = {}, {}
    for L in log_ns:
        x = ScalarArray(gen.fr(81, 1 << L))
        best = None
        for t in candidates:
            check(lib.zkp_ntt_set_block(L, t), "zkp_ntt_set_block")
            ms = _time(lambda: ntt.ntt(x), reps=10 if L < 22 else 4)
            times[f"{L}:{t}"] = ms
            if best is None or ms < best[1]:
                best = (t, ms)
        out[str(L)] = best[0]
        check(lib.zkp_ntt_set_block(L, best[0]), "zkp_ntt_set_block")
        del x
    with _lock:
        _load().setdefault(_device_key(), {})["ntt_block"] = out
        _save()
    return {"best": out, "ms": times}


def tune_msm_blocks(log_n: int = 22, candidates=(64, 128, 256), bases=None, sweeps: int = 1) -> dict:
    """Coordinate descent over the CTA sizes of the pairing rounds' up pass, down pass and the
    XYZZ walk, timing an MSM over resident bases in the tuned (window, tables) configuration
    of 2^log_n points; caches the winners."""
    from . import gen, msm
    n = 1 << log_n
    lib = load(msm.LIB)
    pts = bases if bases is not None else gen.points(2, n)
    c, nt = msm_resident_config(n)
    rb = msm.ResidentBases(pts, window=c, n_tables=nt)
    ws = rb.workspace()
    s = gen.fr(82, n)
    res = torch.zeros(16, dtype=torch.int32, device="cuda")
    cur = {name: 256 for name in MSM_BLOCK_STAGES}
    cur.update(_load().get(_device_key(), {}).get("msm_block", {}))
    times = {}
    for _ in range(sweeps):
        for i, name in enumerate(MSM_BLOCK_STAGES):
            best = None
            for t in candidates:
                check(lib.zkp_msm_set_block(i, t), "zkp_msm_set_block")
                ms = _time(lambda: rb.msm(s, res, ws), reps=3)
                times[f"{name}:{t}"] = ms
                if best is None or ms < best[1]:
                    best = (t, ms)
            cur[name] = best[0]
            check(lib.zkp_msm_set_block(i, best[0]), "zkp_msm_set_block")
    with _lock:
        _load().setdefault(_device_key(), {})["msm_block"] = dict(cur)
        _save()
    del rb, ws
    torch.cuda.empty_cache()
    return {"best": cur, "ms": times}


def tune_msm_resident(log_n: int = 22, windows=range(8, 21), full_only: bool = True, bases=None,
                      batch: int = 4) -> tuple:
    """Times `batch` MSMs of 2^log_n points in one zkp_msm_batch launch sequence over
    precomputed tables (one per window when full_only) for each window width and caches the
    fastest (window, n_tables) for resident bases of 2^log_n.  The default batch of 4 is the
    served program's shape (its four MSMs run as one batch); batch=1 tunes for single calls."""
    from . import gen, msm
    n = 1 << log_n
    pts = bases if bases is not None else gen.points(2, n)
    scalars = [gen.fr(78 + i, n) for i in range(batch)]
    res = [torch.zeros(16, dtype=torch.int32, device="cuda") for _ in range(batch)]
    results = {}
    for c in windows:
        nt = (254 + c - 1) // c if full_only else 1
        rb = msm.ResidentBases(pts[:n], window=c, n_tables=nt)
        b = msm.MsmBatch([{"points": rb.tables, "n_tables": rb.n_tables, "table_stride": rb.n, "scalars": s,
                           "n": n, "window": c, "result": r} for s, r in zip(scalars, res)])
        results[(c, nt)] = _time(lambda: b.run(), reps=3)
        del rb, b
        torch.cuda.empty_cache()
    best = min(results, key=results.get)
    with _lock:
        _load().setdefault(_device_key(), {}).setdefault("msm_resident", {})[str(log_n)] = list(best)
        _save()
    return best, {f"{c}x{nt}": t for (c, nt), t in results.items()}
