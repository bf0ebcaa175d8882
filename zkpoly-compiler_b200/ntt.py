"""NTT operators: host-side mirror of the reference's Rust wrappers (core/src/ntt.rs:97-378).

Each class has the reference's name and `get_fn()` returns a function with the runtime's
FuncCall convention `f(mut_vars, vars)` (runtime/src/functions.rs:19-35): SsipNtt takes
mut=[x], vars=[twiddle, stream]; RecomputeNtt mut=[x], vars=[pq, omegas, stream];
DistributePowers mut=[poly], vars=[powers, stream].  The same argument checks as the Rust
code are made (power-of-two length, twiddle.len * 2 == x.len, omegas.len == 32) and a non-zero
cudaError_t raises, as `cuda_check!` panics in the reference.
"""
from __future__ import annotations

import ctypes
import functools

import numpy as np
import torch

from . import field
from .native import check, load
from .scalar import ScalarArray, device_words, require_cuda, stream_handle

LIB = "libntt.so"


_plans_applied = False


def _lib():
    global _plans_applied
    require_cuda()
    lib = load(LIB)
    if not _plans_applied:
        _plans_applied = True
        from . import tuner
        tuner.apply_ntt_plans()  # tuned digit caps for this GPU model, if cached
    return lib


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _log2_exact(n: int) -> int:
    assert n > 0 and n & (n - 1) == 0, f"length {n} is not a power of two"
    return n.bit_length() - 1


# ------------------------------------------------------------------ raw C-ABI calls
def ssip_ntt(x: ScalarArray, twiddle: ScalarArray, stream=None) -> None:
    log_len = _log2_exact(x.len)
    assert twiddle.len * 2 == x.len or x.len == 1
    check(_lib().ssip_ntt(x.poly_ptr(), twiddle.values.data_ptr(), log_len, stream_handle(stream), 8, 8),
          "ssip_ntt")


def recompute_ntt(x: ScalarArray, pq: ScalarArray, omegas: ScalarArray, stream=None) -> None:
    log_len = _log2_exact(x.len)
    assert omegas.len == 32
    pq_deg = _log2_exact(pq.len) + 1
    check(_lib().recompute_ntt(x.poly_ptr(), pq.values.data_ptr(), pq_deg, omegas.values.data_ptr(), log_len,
                               stream_handle(stream), 8, 8), "recompute_ntt")


def distribute_powers(poly: ScalarArray, powers: ScalarArray, stream=None) -> None:
    check(_lib().distribute_powers(poly.poly_ptr(), powers.values.data_ptr(), powers.len, stream_handle(stream)),
          "distribute_powers")


def ssip_precompute(length: int, unit_mont: np.ndarray) -> np.ndarray:
    """Host table [unit^0 .. unit^(length-1)] (Montgomery limbs), like SsipPrecompute::get_fn."""
    out = np.zeros((length, 8), dtype=np.uint32)
    unit = np.ascontiguousarray(unit_mont, dtype=np.uint32)
    check(_lib().ssip_precompute(out.ctypes.data, length, unit.ctypes.data), "ssip_precompute")
    return out


def gen_pq_omegas(pq_len: int, length: int, unit_mont: np.ndarray):
    pq = np.zeros((pq_len, 8), dtype=np.uint32)
    omegas = np.zeros((32, 8), dtype=np.uint32)
    unit = np.ascontiguousarray(unit_mont, dtype=np.uint32).copy()
    pq_deg = _log2_exact(pq_len) + 1
    load(LIB).gen_pq_omegas(pq.ctypes.data, omegas.ctypes.data, pq_deg, length, unit.ctypes.data)
    return pq, omegas


def get_pq_len(log_len: int, stage_threads=(8, 8)) -> int:
    """GenPqOmegas::get_pq_len (core/src/ntt.rs:322-335)."""
    def get_deg(deg_stage, max_deg_stage):
        rounds = 1
        while True:
            d = deg_stage if rounds == 1 else (deg_stage - 1) // rounds + 1
            if d <= max_deg_stage:
                return d
            rounds += 1
    s1, s2 = stage_threads
    d1 = get_deg((log_len + 1) // 2, s1 + 1)
    d2 = get_deg(log_len // 2, (s2 + 2) // 2)
    return 1 << (max(d1, d2) - 1)


def ntt_ex(x: ScalarArray, twiddle: ScalarArray, shift: torch.Tensor | None = None,
           scale: torch.Tensor | None = None, stream=None, shoup: torch.Tensor | None = None) -> None:
    """zkp_ntt_ex; with `shoup` (shoup_table_of(twiddle)) the register passes use Shoup's product."""
    log_len = _log2_exact(x.len)
    if shoup is None:
        check(_lib().zkp_ntt_ex(x.poly_ptr(), twiddle.values.data_ptr(), log_len, _ptr(shift), _ptr(scale),
                                stream_handle(stream)), "zkp_ntt_ex")
    else:
        check(_lib().zkp_ntt_ex_shoup(x.poly_ptr(), twiddle.values.data_ptr(), shoup.data_ptr(), log_len,
                                      _ptr(shift), _ptr(scale), stream_handle(stream)), "zkp_ntt_ex_shoup")


def coset_lde(out: ScalarArray, inp: ScalarArray, twiddle: ScalarArray, shift: torch.Tensor,
              stream=None, shoup: torch.Tensor | None = None) -> None:
    if shoup is None:
        check(_lib().zkp_coset_lde(out.poly_ptr(), inp.poly_ptr(), twiddle.values.data_ptr(),
                                   _log2_exact(inp.len), _log2_exact(out.len), _ptr(shift), stream_handle(stream)),
              "zkp_coset_lde")
    else:
        check(_lib().zkp_coset_lde_shoup(out.poly_ptr(), inp.poly_ptr(), twiddle.values.data_ptr(),
                                         shoup.data_ptr(), _log2_exact(inp.len), _log2_exact(out.len), _ptr(shift),
                                         stream_handle(stream)), "zkp_coset_lde_shoup")


def shoup_table_of(twiddle: ScalarArray, stream=None) -> torch.Tensor:
    """Shoup twiddle table (16 words per root: the plain root and floor(root * 2^256 / r)) built on
    the device from the Montgomery table `twiddle` of a size-2 * twiddle.len transform."""
    out = torch.empty((twiddle.len, 16), dtype=torch.int32, device=twiddle.values.device)
    check(_lib().zkp_ntt_shoup_table(twiddle.values.data_ptr(), _log2_exact(twiddle.len) + 1, out.data_ptr(),
                                     stream_handle(stream)), "zkp_ntt_shoup_table")
    return out


def plan_digits(log_len: int) -> list[int]:
    """Digit widths (top first) of the passes the current plan for 2^log_len uses."""
    buf = (ctypes.c_uint * 8)()
    k = _lib().zkp_ntt_plan_digits(log_len, buf, 8)
    return [int(buf[i]) for i in range(k)]


def num_passes(log_len: int) -> int:
    return int(_lib().zkp_ntt_num_passes(log_len))


# ------------------------------------------------------------------ cached constants
@functools.lru_cache(maxsize=64)
def twiddle_table(log_n: int, inverse: bool = False, device: str = "cuda") -> ScalarArray:
    """Device table [w^0 .. w^(n/2-1)] for the size-2^log_n (inverse) root, built by
    ssip_precompute exactly as the compiler's precompute pass does
    (compiler/src/transit/type2/precompute.rs:30-249)."""
    w = field.mont_words(field.root_of_unity(log_n, inverse))
    tab = ssip_precompute(max(1, (1 << log_n) // 2), w)
    return ScalarArray(device_words(tab, device))


@functools.lru_cache(maxsize=64)
def scalar_const(value: int, device: str = "cuda") -> torch.Tensor:
    """One Montgomery-form Fr constant on the device."""
    return device_words(field.mont_words(value)[None, :], device)


@functools.lru_cache(maxsize=64)
def shoup_table(log_n: int, inverse: bool = False, device: str = "cuda") -> torch.Tensor:
    """Shoup table of twiddle_table(log_n, inverse), for the library's own transforms."""
    tab = shoup_table_of(twiddle_table(log_n, inverse, device))
    torch.cuda.current_stream().synchronize()
    return tab


def n_inv(log_n: int, device: str = "cuda") -> torch.Tensor:
    return scalar_const(pow(1 << log_n, -1, field.FR_MODULUS), device)


# ------------------------------------------------------------------ compiler-level compositions
def ntt(x: ScalarArray, stream=None) -> None:
    """Forward NTT at the natural root of the size (NTT(w)); the register passes multiply by the
    Shoup table of the root table (same values as ssip_ntt with the root table alone)."""
    log_n = _log2_exact(x.len)
    if log_n == 0:
        return
    ntt_ex(x, twiddle_table(log_n, False), stream=stream, shoup=shoup_table(log_n, False))


def intt(x: ScalarArray, stream=None) -> None:
    """INTT = NTT(w^-1) then * n^-1 (intt_mending.rs:11-70), the scale fused into the last pass."""
    log_n = _log2_exact(x.len)
    ntt_ex(x, twiddle_table(log_n, True), None, n_inv(log_n), stream,
           shoup=shoup_table(log_n, True) if log_n >= 1 else None)


def coset_ntt(out: ScalarArray, coef: ScalarArray, shift: int = field.GENERATOR, stream=None) -> None:
    """Evaluations of the coefficient vector `coef` on shift * <w_out>: zero-extend,
    multiply by shift^i, NTT at the extended size, all fused (poly_coef.rs:252-255 Extend +
    distribute_powers.cuh:5-21 + NTT)."""
    log_n = _log2_exact(out.len)
    coset_lde(out, coef, twiddle_table(log_n, False), scalar_const(shift), stream, shoup=shoup_table(log_n, False))


# ------------------------------------------------------------------ batched form
class NttBatch:
    """Many in-place transforms of uneven sizes as one graph-capturable launch sequence.

    tasks: list of (ScalarArray, kind) with kind in {"ntt", "intt", "coset"}; a coset task
    multiplies x[i] by GENERATOR^i before the forward transform (the input must already be
    the zero-extended coefficient vector)."""

    def __init__(self, tasks, shift: int = field.GENERATOR):
        from .native import ZkpNttTask
        lib = _lib()
        arr = (ZkpNttTask * len(tasks))()
        self._keep = []
        for i, (x, kind) in enumerate(tasks):
            log_n = _log2_exact(x.len)
            inverse = kind == "intt"
            tw = twiddle_table(log_n, inverse)
            sh = scalar_const(shift) if kind == "coset" else None
            sc = n_inv(log_n) if inverse else None
            st = shoup_table(log_n, inverse)
            self._keep += [x, tw, sh, sc, st]
            arr[i] = ZkpNttTask(x.poly_ptr(), tw.values.data_ptr(), log_n, _ptr(sh), _ptr(sc), st.data_ptr())
        self._plan = ctypes.c_void_p()
        self._destroy = lib.zkp_ntt_batch_plan_destroy  # kept: module globals may be gone at exit
        check(lib.zkp_ntt_batch_plan_create(ctypes.cast(arr, ctypes.c_void_p), len(tasks),
                                            ctypes.byref(self._plan)), "zkp_ntt_batch_plan_create")

    def run(self, stream=None):
        check(_lib().zkp_ntt_batch_run(self._plan, stream_handle(stream)), "zkp_ntt_batch_run")

    def __del__(self):
        if getattr(self, "_plan", None):
            self._destroy(self._plan)
            self._plan = None


# ------------------------------------------------------------------ RegisteredFunction mirrors
class SsipNtt:
    """core/src/ntt.rs:152-200"""
    name = "ssip_ntt"

    def get_fn(self):
        def f(mut_var, var):
            assert len(mut_var) == 1 and len(var) == 2
            ssip_ntt(mut_var[0], var[0], var[1])
        return f


class RecomputeNtt:
    """core/src/ntt.rs:237-290"""
    name = "recompute_ntt"

    def get_fn(self):
        def f(mut_var, var):
            assert len(mut_var) == 1 and len(var) == 3
            recompute_ntt(mut_var[0], var[0], var[1], var[2])
        return f


class DistributePowers:
    """core/src/ntt.rs:106-150"""
    name = "distribute_powers"

    def get_fn(self):
        def f(mut_var, var):
            assert len(mut_var) == 1 and len(var) == 2
            distribute_powers(mut_var[0], var[0], var[1])
        return f


class SsipPrecompute:
    """core/src/ntt.rs:202-235: fills a host twiddle array of `len` roots."""

    def get_fn(self):
        def f(twiddle_len: int, unit_mont: np.ndarray) -> np.ndarray:
            assert twiddle_len & (twiddle_len - 1) == 0
            return ssip_precompute(twiddle_len, unit_mont)
        return f


class GenPqOmegas:
    """core/src/ntt.rs:292-371"""

    def get_pq_len(self, log_len: int) -> int:
        return get_pq_len(log_len)

    def get_fn(self):
        return gen_pq_omegas
