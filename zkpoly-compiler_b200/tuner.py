"""Project-written autotuner: measures candidate kernel parameters on the device and caches the
winners per GPU model (in the role of the reference's core/src/msm/tuning/cost_model.py, which
predicts a window from relative cost coefficients instead of measuring).

Tuned parameters:
  - MSM window width c in [8, 20] per log2 n (zkp_msm_device timed on seeded inputs);
  - NTT largest digit (sub-transform size 2^D, which sets the pass split and the CTA shape)
    per log2 n (zkp_ntt_set_max_digit, timed on seeded inputs).
The cache is a JSON file next to the libraries; without an entry the libraries' own cost
model / default plan is used.
"""
from __future__ import annotations

import json
import os
import threading

import torch

from .native import check, load

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "lib", "tuning.json")
_lock = threading.Lock()
_cache: dict | None = None


def _device_key() -> str:
    return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"


def _load() -> dict:
    global _cache
    if _cache is None:
        try:
            with open(CACHE) as f:
                _cache = json.load(f)
        except (OSError, ValueError):
            _cache = {}
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
    c = 16
    return c, (254 + c - 1) // c


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


def tune_msm_resident(log_n: int = 22, windows=(13, 14, 15, 16, 17, 18, 19, 20), full_only: bool = True,
                      bases=None) -> tuple:
    """Times zkp_msm_device over precomputed tables (one per window when full_only) for each
    window width and caches the fastest (window, n_tables) for resident bases of 2^log_n."""
    from . import gen, msm
    n = 1 << log_n
    pts = bases if bases is not None else gen.points(2, n)
    s = gen.fr(78, n)
    res = torch.zeros(16, dtype=torch.int32, device="cuda")
    results = {}
    for c in windows:
        nt = (254 + c - 1) // c if full_only else 1
        rb = msm.ResidentBases(pts, window=c, n_tables=nt)
        ws = rb.workspace()
        results[(c, nt)] = _time(lambda: rb.msm(s, res, ws), reps=2)
        del rb, ws
        torch.cuda.empty_cache()
    best = min(results, key=results.get)
    with _lock:
        _load().setdefault(_device_key(), {}).setdefault("msm_resident", {})[str(log_n)] = list(best)
        _save()
    return best, {f"{c}x{nt}": t for (c, nt), t in results.items()}
