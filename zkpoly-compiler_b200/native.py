"""Loads the in-tree CUDA libraries (lib/*.so) through ctypes and declares their C ABI.

There is no CPU fallback: every entry point of this package calls into these libraries, and
loading fails loudly when a library is missing or no CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")

c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_void_p = ctypes.c_void_p
cudaError_t = ctypes.c_int


class PolyPtr(ctypes.Structure):
    """core/src/common/iter/src/iter.cuh:12-18 / core/src/poly_ptr.rs:4-11"""
    _fields_ = [("ptr", ctypes.c_void_p), ("len", ctypes.c_size_t), ("rotate", ctypes.c_size_t),
                ("offset", ctypes.c_size_t), ("whole_len", ctypes.c_size_t)]


ConstPolyPtr = PolyPtr  # identical layout (iter.cuh:20-26)


class ZkpPipelineArg(ctypes.Structure):
    """include/zkp_pipeline.h: a host polynomial streamed in chunks (whole = 0) or a host array
    of `whole` elements copied once (scalars, periodic inputs)."""
    _fields_ = [("host", ctypes.c_void_p), ("whole", ctypes.c_ulonglong), ("write_only", ctypes.c_uint)]

_libs: dict[str, ctypes.CDLL] = {}

# symbol -> (restype, argtypes)
SIGNATURES = {
    "libntt.so": {
        "ssip_ntt": (cudaError_t, [PolyPtr, c_void_p, ctypes.c_uint, c_void_p, ctypes.c_uint, ctypes.c_uint]),
        "ssip_precompute": (cudaError_t, [c_void_p, ctypes.c_uint, c_void_p]),
        "recompute_ntt": (cudaError_t, [PolyPtr, c_void_p, ctypes.c_uint, c_void_p, ctypes.c_uint, c_void_p,
                                        ctypes.c_uint, ctypes.c_uint]),
        "gen_pq_omegas": (None, [c_void_p, c_void_p, ctypes.c_uint, ctypes.c_uint, c_void_p]),
        "distribute_powers": (cudaError_t, [PolyPtr, c_void_p, ctypes.c_ulonglong, c_void_p]),
        "zkp_ntt_ex": (cudaError_t, [PolyPtr, c_void_p, ctypes.c_uint, c_void_p, c_void_p, c_void_p]),
        "zkp_coset_lde": (cudaError_t, [PolyPtr, PolyPtr, c_void_p, ctypes.c_uint, ctypes.c_uint, c_void_p,
                                        c_void_p]),
        "zkp_ntt_shoup_table": (cudaError_t, [c_void_p, ctypes.c_uint, c_void_p, c_void_p]),
        "zkp_ntt_roots_device": (cudaError_t, [c_void_p, ctypes.c_ulonglong, c_void_p, c_void_p]),
        "zkp_ntt_shoup_probe": (cudaError_t, [ctypes.c_uint, ctypes.c_uint, c_void_p, c_void_p]),
        "zkp_ntt_ex_shoup": (cudaError_t, [PolyPtr, c_void_p, c_void_p, ctypes.c_uint, c_void_p, c_void_p, c_void_p]),
        "zkp_coset_lde_shoup": (cudaError_t, [PolyPtr, PolyPtr, c_void_p, c_void_p, ctypes.c_uint, ctypes.c_uint,
                                              c_void_p, c_void_p]),
        "zkp_ntt_num_passes": (ctypes.c_uint, [ctypes.c_uint]),
        "zkp_ntt_plan_digits": (ctypes.c_uint, [ctypes.c_uint, c_void_p, ctypes.c_uint]),
        "zkp_ntt_set_max_digit": (cudaError_t, [ctypes.c_uint, ctypes.c_uint]),
        "zkp_ntt_set_block": (cudaError_t, [ctypes.c_uint, ctypes.c_uint]),
        "zkp_ntt_batch_plan_create": (cudaError_t, [c_void_p, ctypes.c_uint, ctypes.POINTER(c_void_p)]),
        "zkp_ntt_batch_run": (cudaError_t, [c_void_p, c_void_p]),
        "zkp_ntt_batch_set_solo_log": (cudaError_t, [ctypes.c_uint]),
        "zkp_ntt_batch_plan_destroy": (None, [c_void_p]),
        "zkp_ntt_profile_enable": (None, [ctypes.c_int]),
        "zkp_ntt_profile_read": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_char_p),
                                                ctypes.c_int]),
    },
    "libmsm.so": {
        "msm": (cudaError_t, [ctypes.POINTER(c_void_p), ctypes.POINTER(ctypes.c_ulong), ctypes.c_ulonglong,
                              ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                              ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(c_void_p), ctypes.c_uint,
                              ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p)]),
        "msm_precompute": (cudaError_t, [ctypes.c_ulonglong, ctypes.POINTER(c_void_p), ctypes.c_uint]),
        "zkp_msm_workspace_size": (ctypes.c_ulonglong, [ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint]),
        "zkp_msm_default_window": (ctypes.c_uint, [ctypes.c_ulonglong]),
        "zkp_msm_set_affine_rounds": (cudaError_t, [ctypes.c_int]),
        "zkp_msm_set_block": (cudaError_t, [ctypes.c_uint, ctypes.c_uint]),
        "zkp_msm_rounds_for": (ctypes.c_uint, [ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint]),
        "zkp_msm_device": (cudaError_t, [c_void_p, ctypes.c_ulonglong, c_void_p, ctypes.c_uint, c_void_p,
                                         ctypes.c_ulonglong, ctypes.c_uint, c_void_p, c_void_p]),
        "zkp_msm_precompute_device": (cudaError_t, [c_void_p, ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_uint,
                                                    c_void_p]),
        "zkp_msm_batch_workspace_size": (ctypes.c_ulonglong, [c_void_p, ctypes.c_uint]),
        "zkp_msm_device_noalloc": (cudaError_t, [c_void_p, ctypes.c_uint, c_void_p, ctypes.c_ulonglong,
                                                 ctypes.c_uint, c_void_p, c_void_p]),
        "zkp_msm_noalloc_capacity": (ctypes.c_ulonglong, []),
        "zkp_msm_batch": (cudaError_t, [c_void_p, ctypes.c_uint, c_void_p, ctypes.c_ulonglong, c_void_p]),
        "zkp_msm_profile_enable": (None, [ctypes.c_int]),
        "zkp_msm_profile_read": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_char_p),
                                                ctypes.c_int]),
        "zkp_imad_probe": (cudaError_t, [ctypes.c_uint, ctypes.c_uint, c_void_p, c_void_p]),
        "zkp_mont_probe": (cudaError_t, [ctypes.c_uint, ctypes.c_uint, c_void_p, c_void_p]),
    },
    "libzkp_pipeline.so": {
        "zkp_fused_pipelined_workspace": (ctypes.c_ulonglong, [c_void_p, ctypes.c_uint, c_void_p, ctypes.c_uint,
                                                               ctypes.c_ulonglong, ctypes.c_ulonglong]),
        "zkp_fused_pipelined": (cudaError_t, [c_void_p, c_void_p, ctypes.c_uint, c_void_p, ctypes.c_uint,
                                              ctypes.c_ulonglong, ctypes.c_ulonglong, c_void_p, ctypes.c_ulonglong,
                                              c_void_p]),
    },
    "libzkp_gen.so": {
        "zkp_gen_fr": (cudaError_t, [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_ulonglong, c_void_p, c_void_p]),
        "zkp_gen_points": (cudaError_t, [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_ulonglong, c_void_p,
                                         c_void_p, c_void_p]),
    },
    "libzkp_runtime.so": {
        "zkp_serve_create": (cudaError_t, [c_void_p, c_void_p, ctypes.c_ulonglong, ctypes.POINTER(c_void_p)]),
        "zkp_serve_submit": (ctypes.c_longlong, [c_void_p, c_void_p]),
        "zkp_serve_footprint": (ctypes.c_ulonglong, [c_void_p, ctypes.c_uint]),
        "zkp_serve_wait": (ctypes.c_int, [c_void_p, ctypes.c_longlong, c_void_p, ctypes.c_double]),
        "zkp_serve_stats": (None, [c_void_p, c_void_p]),
        "zkp_serve_now": (ctypes.c_double, [c_void_p]),
        "zkp_serve_set_policy": (None, [c_void_p, c_void_p]),
        "zkp_serve_destroy": (None, [c_void_p]),
        "zkp_serve_program_create": (cudaError_t, [c_void_p, c_void_p, ctypes.c_uint, ctypes.c_ulonglong,
                                                   ctypes.c_ulonglong, c_void_p, ctypes.c_uint, c_void_p,
                                                   ctypes.c_uint, ctypes.POINTER(c_void_p)]),
        "zkp_serve_submit_program": (ctypes.c_longlong, [c_void_p, c_void_p, c_void_p, ctypes.c_uint, c_void_p,
                                                         ctypes.c_ulonglong]),
        "zkp_serve_program_destroy": (None, [c_void_p, c_void_p]),
    },
    "libpoly.so": {
        "poly_add": (cudaError_t, [PolyPtr, PolyPtr, PolyPtr, c_void_p]),
        "poly_sub": (cudaError_t, [PolyPtr, PolyPtr, PolyPtr, c_void_p]),
        "poly_mul": (cudaError_t, [PolyPtr, PolyPtr, PolyPtr, c_void_p]),
        "zkp_poly_square": (cudaError_t, [PolyPtr, PolyPtr, c_void_p]),
        "poly_one_lagrange": (cudaError_t, [PolyPtr, c_void_p]),
        "poly_one_coef": (cudaError_t, [PolyPtr, c_void_p]),
        "poly_zero": (cudaError_t, [PolyPtr, c_void_p]),
        "poly_eval": (cudaError_t, [c_void_p, ctypes.POINTER(ctypes.c_ulong), PolyPtr, c_void_p, c_void_p, c_void_p]),
        "kate_division": (cudaError_t, [c_void_p, ctypes.POINTER(ctypes.c_ulong), ctypes.c_uint, PolyPtr, c_void_p,
                                        PolyPtr, c_void_p]),
        "scan_mul": (cudaError_t, [c_void_p, ctypes.POINTER(ctypes.c_ulong), PolyPtr, c_void_p]),
        "batched_invert": (cudaError_t, [c_void_p, ctypes.POINTER(ctypes.c_ulong), PolyPtr, c_void_p]),
        "permute": (cudaError_t, [c_void_p, ctypes.POINTER(ctypes.c_ulong), ctypes.c_ulong, PolyPtr, PolyPtr, PolyPtr,
                                  PolyPtr, c_void_p]),
        "inv_scalar": (cudaError_t, [c_void_p, c_void_p]),
        "scalar_pow": (cudaError_t, [c_void_p, ctypes.c_ulonglong, c_void_p]),
    },
}


class ZkpNttTask(ctypes.Structure):
    """include/ntt.h ZkpNttTask"""
    _fields_ = [("x", PolyPtr), ("twiddle", ctypes.c_void_p), ("log_len", ctypes.c_uint),
                ("shift_d", ctypes.c_void_p), ("scale_d", ctypes.c_void_p), ("shoup_d", ctypes.c_void_p)]


class ZkpMsmTask(ctypes.Structure):
    """include/msm.h ZkpMsmTask"""
    _fields_ = [("points_d", ctypes.c_void_p), ("n_tables", ctypes.c_uint), ("scalars_d", ctypes.c_void_p),
                ("n", ctypes.c_ulonglong), ("window", ctypes.c_uint), ("result_d", ctypes.c_void_p),
                ("table_stride", ctypes.c_ulonglong)]


class ZkpServeTableSet(ctypes.Structure):
    _fields_ = [("tables_d", ctypes.c_void_p), ("rows", ctypes.c_ulonglong), ("window", ctypes.c_uint),
                ("n_tables", ctypes.c_uint), ("max_k", ctypes.c_uint)]


ZKP_SERVE_MAX_SETS = 8


class ZkpServeConfig(ctypes.Structure):
    _fields_ = [("hbm_bytes", ctypes.c_ulonglong), ("max_inflight", ctypes.c_uint), ("ext_log", ctypes.c_uint),
                ("min_k", ctypes.c_uint), ("max_k", ctypes.c_uint), ("msm_window", ctypes.c_uint),
                ("msm_tables", ctypes.c_uint), ("n_sets", ctypes.c_uint),
                ("sets", ZkpServeTableSet * ZKP_SERVE_MAX_SETS)]


class ZkpProverRequest(ctypes.Structure):
    _fields_ = [("k", ctypes.c_uint), ("seed", ctypes.c_ulonglong), ("inject_fault", ctypes.c_uint)]


class ZkpProverResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("msm", (ctypes.c_uint * 16) * 4), ("evals", (ctypes.c_uint * 8) * 2),
                ("submit_s", ctypes.c_double), ("start_s", ctypes.c_double), ("done_s", ctypes.c_double),
                ("footprint", ctypes.c_ulonglong)]


ZKP_PROG_MAX_VIEWS = 16


class ZkpProgView(ctypes.Structure):
    """include/zkp_runtime.h: one operand of a lowered program op."""
    _fields_ = [("space", ctypes.c_uint), ("index", ctypes.c_uint), ("addr", ctypes.c_ulonglong),
                ("len", ctypes.c_ulonglong), ("rotate", ctypes.c_ulonglong), ("offset", ctypes.c_ulonglong),
                ("whole_len", ctypes.c_ulonglong)]


class ZkpProgOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint), ("n_views", ctypes.c_uint), ("imm", ctypes.c_ulonglong * 4),
                ("v", ZkpProgView * ZKP_PROG_MAX_VIEWS)]


class ZkpProgOut(ctypes.Structure):
    _fields_ = [("host_offset", ctypes.c_ulonglong), ("bytes", ctypes.c_ulonglong),
                ("result_offset", ctypes.c_ulonglong)]


class ZkpServePolicy(ctypes.Structure):
    _fields_ = [("priority_bytes", ctypes.c_ulonglong), ("large_bytes", ctypes.c_ulonglong),
                ("max_large_inflight", ctypes.c_uint)]


class ZkpServeStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_ulonglong), ("failed", ctypes.c_ulonglong),
                ("peak_inflight", ctypes.c_ulonglong), ("peak_bytes", ctypes.c_ulonglong),
                ("arena_bytes", ctypes.c_ulonglong)]


class CudaError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where} returned cudaError_t {code}")
        self.code = code


def lib_path(name: str) -> str:
    return os.path.join(LIB_DIR, name)


def load(name: str) -> ctypes.CDLL:
    """dlopen lib/<name> and declare its symbols; raises if the library was not built."""
    if name in _libs:
        return _libs[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library {path} is missing: run __graft_entry__.build() first")
    lib = ctypes.CDLL(path)
    for sym, (res, args) in SIGNATURES.get(name, {}).items():
        fn = getattr(lib, sym)
        fn.restype = res
        fn.argtypes = args
    _libs[name] = lib
    return lib


def check(code: int, where: str) -> None:
    if code != 0:
        raise CudaError(code, where)


def profile_enable(name: str, on: bool) -> None:
    prefix = {"libntt.so": "zkp_ntt", "libmsm.so": "zkp_msm"}[name]
    getattr(load(name), prefix + "_profile_enable")(int(on))


def profile_read(name: str):
    """[(stage, ms)] of the last call of the library while profiling was on."""
    prefix = {"libntt.so": "zkp_ntt", "libmsm.so": "zkp_msm"}[name]
    ms = (ctypes.c_float * 32)()
    names = (ctypes.c_char_p * 32)()
    k = getattr(load(name), prefix + "_profile_read")(ms, names, 32)
    return [(names[i].decode(), ms[i]) for i in range(k)]


def loaded_paths():
    return {n: lib_path(n) for n in _libs}
