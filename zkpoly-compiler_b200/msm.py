"""MSM operators: host-side mirror of the reference's Rust wrapper (core/src/msm.rs:136-369)
plus the resident-bases device form used by the batched and served paths.

`MSM(config).get_buffer_size(len)` and `get_fn()` follow the reference: FuncCall vars are
[point tables..., scalar arrays...] (host), mut_vars [gpu buffer per card..., result points...]
(core/src/msm.rs:302-369).  Points are (n, 16) uint32 affine Montgomery (x limbs, y limbs);
scalars (n, 8) uint32 Montgomery Fr; results (16,) uint32 affine with (0, 0) the identity.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from .native import check, load
from .scalar import require_cuda, stream_handle

LIB = "libmsm.so"


_blocks_applied = False


def _lib():
    global _blocks_applied
    require_cuda()
    lib = load(LIB)
    if not _blocks_applied:
        _blocks_applied = True
        from . import tuner
        tuner.apply_msm_blocks()  # tuned stage CTA sizes for this GPU model, if cached
    return lib


def _u32(a: np.ndarray, words: int) -> np.ndarray:
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.uint32)
    return np.ascontiguousarray(a.reshape(-1, words), dtype=np.uint32)


@dataclass
class MsmConfig:
    """common/src/msm_config.rs:4-56 (window_size, target_window, cards, debug,
    batch_per_run, parts, stage_scalars, stage_points, bits)."""
    window_size: int = 0
    target_window: int = 1
    cards: list = field(default_factory=lambda: [0])
    debug: bool = False
    batch_per_run: int = 1
    parts: int = 1
    stage_scalars: int = 1
    stage_points: int = 1
    bits: int = 254

    def get_precompute(self) -> int:
        return 1


class MSM:
    """core/src/msm.rs:136-369"""

    def __init__(self, config: MsmConfig | None = None):
        self.config = config or MsmConfig()

    def get_buffer_size(self, length: int) -> list[int]:
        cfg = self.config
        sizes = (ctypes.c_ulong * len(cfg.cards))()
        cards = (ctypes.c_uint * len(cfg.cards))(*cfg.cards)
        check(_lib().msm(None, sizes, length, cfg.batch_per_run, cfg.parts, cfg.stage_scalars, cfg.stage_points,
                         len(cfg.cards), cards, None, 0, None, None), "msm(size query)")
        return list(sizes)

    def get_fn(self):
        cfg = self.config
        n_pre = cfg.get_precompute()

        def f(mut_var, var):
            batches = len(var) - n_pre
            assert len(mut_var) == batches + len(cfg.cards)
            buffers, answers = mut_var[:len(cfg.cards)], mut_var[len(cfg.cards):]
            results = msm_host_batches([_u32(s, 8) for s in var[n_pre:]], [_u32(p, 16) for p in var[:n_pre]],
                                       buffers=buffers, cfg=cfg)
            for ans, r in zip(answers, results):
                ans[:] = r
        return f


def msm_host_batches(scalar_batches, point_tables, buffers=None, cfg: MsmConfig | None = None):
    """Calls the reference-ABI `msm` with host arrays; allocates the device buffers when the
    caller does not supply them (the runtime normally hands in its own GpuBuffer)."""
    cfg = cfg or MsmConfig()
    lib = _lib()
    n = point_tables[0].shape[0]
    if buffers is None:
        sizes = MSM(cfg).get_buffer_size(n)
        buffers = []
        for card, sz in zip(cfg.cards, sizes):
            with torch.cuda.device(card):
                buffers.append(torch.empty(sz, dtype=torch.uint8, device=f"cuda:{card}"))
    ptrs = (ctypes.c_void_p * len(buffers))(*[b.data_ptr() for b in buffers])
    cards = (ctypes.c_uint * len(cfg.cards))(*cfg.cards)
    tables = [np.ascontiguousarray(t, dtype=np.uint32) for t in point_tables]
    h_points = (ctypes.c_void_p * len(tables))(*[t.ctypes.data for t in tables])
    scal = [np.ascontiguousarray(s, dtype=np.uint32) for s in scalar_batches]
    h_scal = (ctypes.c_void_p * len(scal))(*[s.ctypes.data for s in scal])
    results = [np.zeros(16, dtype=np.uint32) for _ in scal]
    h_res = (ctypes.c_void_p * len(results))(*[r.ctypes.data for r in results])
    torch.cuda.synchronize()
    check(lib.msm(ptrs, None, n, cfg.batch_per_run, cfg.parts, cfg.stage_scalars, cfg.stage_points,
                  len(cfg.cards), cards, h_points, len(scal), h_scal, h_res), "msm")
    return results


def msm_host(scalars: np.ndarray, points: np.ndarray) -> np.ndarray:
    """One MSM through the reference ABI; returns the affine result as (8,) uint64 limbs."""
    r = msm_host_batches([_u32(scalars, 8)], [_u32(points, 16)])[0]
    return r.view(np.uint64)


def workspace_size(n: int, window: int = 0, n_tables: int = 1) -> int:
    return int(_lib().zkp_msm_workspace_size(n, window, n_tables))


def default_window(n: int) -> int:
    return int(_lib().zkp_msm_default_window(n))


def rounds_for(n: int, window: int = 0, n_tables: int = 1) -> int:
    """Pairing rounds an MSM of n points runs under the current setting."""
    return int(_lib().zkp_msm_rounds_for(n, window, n_tables))


def set_affine_rounds(rounds: int = -1) -> None:
    """Affine pairing rounds for MSMs planned from now on (-1 = chosen by size).  Workspace
    sizes depend on it: size and run under the same setting."""
    check(_lib().zkp_msm_set_affine_rounds(int(rounds)), "zkp_msm_set_affine_rounds")


class ResidentBases:
    """Bases kept in HBM (optionally with precomputed tables) for repeated MSMs: the
    device-pointer form the served path uses."""

    def __init__(self, points: np.ndarray | torch.Tensor, window: int = 0, n_tables: int = 1, device="cuda"):
        require_cuda()
        if isinstance(points, np.ndarray):
            points = torch.from_numpy(_u32(points, 16).view(np.int32)).to(device)
        self.n = points.shape[0]
        self.window = window or default_window(self.n)
        self.n_tables = n_tables
        self.tables = torch.empty((n_tables * self.n, 16), dtype=torch.int32, device=points.device)
        self.tables[: self.n].copy_(points.reshape(self.n, 16))
        if n_tables > 1:
            check(_lib().zkp_msm_precompute_device(self.tables.data_ptr(), self.n, self.window, n_tables,
                                                   stream_handle()), "zkp_msm_precompute_device")
        self.ws_bytes = workspace_size(self.n, self.window, n_tables)

    def workspace(self) -> torch.Tensor:
        return torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.tables.device)

    def msm(self, scalars: torch.Tensor, result: torch.Tensor, workspace: torch.Tensor, stream=None) -> None:
        """result (16 int32) = MSM over device scalars (n, 8) int32; asynchronous on stream."""
        check(_lib().zkp_msm_device(workspace.data_ptr(), workspace.numel(), self.tables.data_ptr(), self.n_tables,
                                    scalars.data_ptr(), self.n, self.window, result.data_ptr(),
                                    stream_handle(stream)), "zkp_msm_device")


MAX_BATCH = 32


class MsmBatch:
    """Up to 32 MSMs of uneven sizes sharing every stage launch (zkp_msm_batch).

    tasks: list of dicts with keys points (device (N, 16) int32, first table), scalars (device
    (n, 8) int32), n, window (0 = auto), n_tables (default 1), result (device 16 int32).
    The call allocates nothing once the workspace exists, so it can be graph-captured."""

    def __init__(self, tasks):
        from .native import ZkpMsmTask
        assert 1 <= len(tasks) <= MAX_BATCH
        self.tasks = tasks
        self.arr = (ZkpMsmTask * len(tasks))()
        for i, t in enumerate(tasks):
            self.arr[i] = ZkpMsmTask(t["points"].data_ptr(), t.get("n_tables", 1), t["scalars"].data_ptr(), t["n"],
                                     t.get("window", 0), t["result"].data_ptr(), t.get("table_stride", 0))
        self.ws_bytes = int(_lib().zkp_msm_batch_workspace_size(ctypes.cast(self.arr, ctypes.c_void_p), len(tasks)))
        assert self.ws_bytes > 0, "invalid MSM batch"
        self.workspace = torch.empty(self.ws_bytes, dtype=torch.uint8, device=tasks[0]["scalars"].device)

    def run(self, stream=None):
        check(_lib().zkp_msm_batch(ctypes.cast(self.arr, ctypes.c_void_p), len(self.tasks), self.workspace.data_ptr(),
                                   self.ws_bytes, stream_handle(stream)), "zkp_msm_batch")
