"""Batched form: many NTTs and MSMs of uneven sizes as one captured CUDA graph.

The mixed workload (seeded): `n_ntt` transforms with log2 sizes uniform on [ntt_lo, ntt_hi],
kinds uniform over forward / inverse / coset, and `n_msm` MSMs with log2 sizes uniform on
[msm_lo, msm_hi] over prefixes of one resident base array.

plain (reference ABI): the per-call path as the reference's runtime drives it - one
         ssip_ntt / zkp_ntt_ex call per transform on the device buffer, and one `msm` call per
         MSM with host scalars and a host point table (core/src/msm.rs:302-369), in order.
plain (device): the same per-call order, but each MSM is zkp_msm_device over device-resident
         bases (one table) - the per-call path with the host copies taken out.
plain (same tables): the per-call order with everything the batch has except the batching:
         each transform through its own zkp_ntt_ex_shoup call (Shoup twiddle tables), each MSM
         a batch of one over the same resident precomputed table sets the batch reads.
batched: one NttBatch plan (a persistent launch per pass shared by every transform) on one
         stream and MsmBatch launches (every stage shared by up to 32 MSMs) over precomputed
         resident tables on a second stream, captured once into a CUDA graph and replayed.
"""
from __future__ import annotations

import numpy as np
import torch

from . import gen, msm, ntt, tuner
from .scalar import ScalarArray


class MixedWorkload:
    def __init__(self, seed: int = 3, n_ntt: int = 64, ntt_lo: int = 10, ntt_hi: int = 20, n_msm: int = 16,
                 msm_lo: int = 12, msm_hi: int = 22, device="cuda"):
        rng = np.random.default_rng(seed)
        self.ntt_logs = [int(x) for x in rng.integers(ntt_lo, ntt_hi + 1, n_ntt)]
        self.ntt_kinds = [["ntt", "intt", "coset"][int(k)] for k in rng.integers(0, 3, n_ntt)]
        self.msm_logs = [int(x) for x in rng.integers(msm_lo, msm_hi + 1, n_msm)]
        self.device = device
        nmax = 1 << max(self.msm_logs)
        self.bases = gen.points(2, nmax, device)
        self.ntt_init = [gen.fr(1000 + i, 1 << L, device) for i, L in enumerate(self.ntt_logs)]
        self.scalars = [gen.fr(2000 + i, 1 << L, device) for i, L in enumerate(self.msm_logs)]
        self.windows = [tuner.msm_window(1 << L) for L in self.msm_logs]
        self.ntt_bufs = [ScalarArray(t.clone()) for t in self.ntt_init]
        self.results = [torch.zeros(16, dtype=torch.int32, device=device) for _ in self.msm_logs]
        self.ws = torch.empty(max(msm.workspace_size(1 << L, w) for L, w in zip(self.msm_logs, self.windows)),
                              dtype=torch.uint8, device=device)
        self.graph = None
        self.tables = None
        self.h_bases = None

    # ---- useful work, for throughput
    def work(self):
        return {"ntt_elems": sum(1 << L for L in self.ntt_logs), "msm_points": sum(1 << L for L in self.msm_logs),
                "tasks": len(self.ntt_logs) + len(self.msm_logs)}

    def reset_inputs(self):
        for b, t in zip(self.ntt_bufs, self.ntt_init):
            b.values.copy_(t)

    # ---- per-call path
    def run_plain(self, stream=None):
        for x, L, kind in zip(self.ntt_bufs, self.ntt_logs, self.ntt_kinds):
            if kind == "ntt":
                ntt.ssip_ntt(x, ntt.twiddle_table(L), stream)
            elif kind == "intt":
                ntt.ntt_ex(x, ntt.twiddle_table(L, True), None, ntt.n_inv(L), stream)
            else:
                ntt.ntt_ex(x, ntt.twiddle_table(L), ntt.scalar_const(7), None, stream)
        from .native import check, load
        lib = load(msm.LIB)
        for s, L, w, r in zip(self.scalars, self.msm_logs, self.windows, self.results):
            check(lib.zkp_msm_device(self.ws.data_ptr(), self.ws.numel(), self.bases.data_ptr(), 1, s.data_ptr(),
                                     1 << L, w, r.data_ptr(), torch.cuda.current_stream().cuda_stream
                                     if stream is None else stream.cuda_stream), "zkp_msm_device")

    # ---- per-call path over the batch's own tables
    def build_plain_same_tables(self):
        if self.tables is None:
            self._resident_tables()
        self.single = []
        for s, L, r in zip(self.scalars, self.msm_logs, self.results):
            c, nt = tuner.msm_resident_config(1 << L)
            t, rows = self.tables[(c, nt)]
            self.single.append(msm.MsmBatch([{"points": t, "n_tables": nt, "table_stride": rows, "scalars": s,
                                               "n": 1 << L, "window": c, "result": r}]))

    def run_plain_same_tables(self, stream=None):
        if not hasattr(self, "single"):
            self.build_plain_same_tables()
        for x, L, kind in zip(self.ntt_bufs, self.ntt_logs, self.ntt_kinds):
            inv = kind == "intt"
            tw, sh = ntt.twiddle_table(L, inv), ntt.shoup_table(L, inv)
            if kind == "ntt":
                ntt.ntt_ex(x, tw, None, None, stream, shoup=sh)
            elif kind == "intt":
                ntt.ntt_ex(x, tw, None, ntt.n_inv(L), stream, shoup=sh)
            else:
                ntt.ntt_ex(x, tw, ntt.scalar_const(7), None, stream, shoup=sh)
        for b in self.single:
            b.run(stream)

    # ---- per-call path through the reference ABI (host arrays for the MSMs)
    def run_plain_ref_abi(self, stream=None):
        """Returns the MSM results (16 uint32 each, host); the NTTs transform ntt_bufs."""
        for x, L, kind in zip(self.ntt_bufs, self.ntt_logs, self.ntt_kinds):
            if kind == "ntt":
                ntt.ssip_ntt(x, ntt.twiddle_table(L), stream)
            elif kind == "intt":
                ntt.ntt_ex(x, ntt.twiddle_table(L, True), None, ntt.n_inv(L), stream)
            else:
                ntt.ntt_ex(x, ntt.twiddle_table(L), ntt.scalar_const(7), None, stream)
        if self.h_bases is None:
            # host copies a runtime's host pool would hold (pinned)
            self.h_bases = self.bases.cpu().pin_memory().numpy().view(np.uint32)
            self.h_scalars = [s.cpu().pin_memory().numpy().view(np.uint32) for s in self.scalars]
            n_max = 1 << max(self.msm_logs)
            self.ref_ws = torch.empty(msm.MSM().get_buffer_size(n_max)[0], dtype=torch.uint8, device=self.device)
        out = []
        for hs, L in zip(self.h_scalars, self.msm_logs):
            out.append(msm.msm_host_batches([hs], [self.h_bases[: 1 << L]], buffers=[self.ref_ws])[0])
        return out

    # ---- batched path
    def _resident_tables(self):
        """Precomputed tables over the shared bases: one set per (window, table count) that the
        resident configuration picks for the batch's sizes.  A task of n points reads the first
        n rows of each table of its set (table_stride = the set's row count)."""
        from .native import check, load
        sets = {}
        for L in self.msm_logs:
            cfg = tuner.msm_resident_config(1 << L)
            sets[cfg] = max(sets.get(cfg, 0), 1 << L)
        lib = load(msm.LIB)
        self.tables = {}
        for (c, nt), rows in sets.items():
            t = torch.empty((nt * rows, 16), dtype=torch.int32, device=self.device)
            t[:rows].copy_(self.bases[:rows])
            if nt > 1:
                check(lib.zkp_msm_precompute_device(t.data_ptr(), rows, c, nt,
                                                    torch.cuda.current_stream().cuda_stream),
                      "zkp_msm_precompute_device")
            self.tables[(c, nt)] = (t, rows)
        torch.cuda.synchronize()

    def build_batched(self):
        self.ntt_batch = ntt.NttBatch(list(zip(self.ntt_bufs, self.ntt_kinds)))
        if self.tables is None:
            self._resident_tables()
        tasks = []
        for s, L, r in zip(self.scalars, self.msm_logs, self.results):
            c, nt = tuner.msm_resident_config(1 << L)
            t, rows = self.tables[(c, nt)]
            tasks.append({"points": t, "n_tables": nt, "table_stride": rows, "scalars": s, "n": 1 << L,
                          "window": c, "result": r})
        self.msm_batches = [msm.MsmBatch(tasks[i:i + msm.MAX_BATCH]) for i in range(0, len(tasks), msm.MAX_BATCH)]
        self.s_main = torch.cuda.Stream()
        self.s_side = torch.cuda.Stream()
        # warm the plans once outside capture (loads every kernel), then restore the inputs the
        # warm-up transformed in place
        self._launch_batched()
        torch.cuda.synchronize()
        self.reset_inputs()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.s_main):
            self._launch_batched()

    def _launch_batched(self):
        cur = torch.cuda.current_stream()
        self.s_side.wait_stream(cur)
        self.ntt_batch.run(cur)
        with torch.cuda.stream(self.s_side):
            for b in self.msm_batches:
                b.run(self.s_side)
        cur.wait_stream(self.s_side)

    def run_batched(self):
        if self.graph is None:
            self.build_batched()
        self.graph.replay()

    def snapshot(self):
        return ([b.values.clone() for b in self.ntt_bufs], [r.clone() for r in self.results])
