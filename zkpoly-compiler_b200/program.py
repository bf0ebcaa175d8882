"""Compiled programs in the served loop: a reference artifact's instruction chunk, lowered once
to the native op list of libzkp_runtime.so and run per request like the built-in prover.

An artifact directory (compiler/src/driver/artifect.rs:65-86) holds, per memory version,
``version_<size>.json`` = serde_json of ``(MemoryInfo, Chunk, Statistics)``, where the chunk is
serialised through ``ChunkDeserializer`` (compiler/src/transit/type3/lowering/serialization.rs
:16-44): ``{"instructions", "f_table", "event_table", "n_variables", "n_threads", "lbss"}``.
``instructions`` are ``Instruction {node, track, stream}`` (runtime/src/instructions.rs:51-206)
with serde's default external tagging (``{"FuncCall": {"func_id": 3, "arg_mut": [...], "arg":
[...]}}``, ``{"Return": 12}``); ids (VariableId, FunctionId, EventId, EntryId, ConstantId) are
newtype structs and serialise as bare integers; ``f_table`` and ``event_table`` are
``Heap(Vec, PhantomData)`` pairs ``[[...], null]`` of ``KernelType`` (runtime/src/functions.rs
:52-80) and ``EventType`` (runtime/src/devices.rs:13-17).  The constants are the artifact's
constant table (artifact.py).

The reference's runtime interprets the chunk on CPU threads, calling one kernel wrapper per
FuncCall with the argument orders fixed by compiler/src/transit/type3/lowering/emit_func.rs
:25-46, :335-453.  This module resolves the chunk once instead:

* every variable becomes a view into a request's device block (GPU allocations: the
  compiler's ``Offset(offset, size)`` plan as is, ``Dynamic`` ones after it), its pinned host
  block (CPU allocations), an input buffer (``LoadInput``) or a resident constant
  (``LoadConstant``; GPU constants in HBM, CPU ones in pinned host memory);
* ``Rotation`` / ``Slice`` / ``SetSliceMeta`` / ``SliceBuffer`` / ``AssembleTuple`` /
  ``MoveRegister`` / ``CopyRegister`` are view arithmetic (runtime/src/scalar.rs:300-445);
* ``Transfer``, ``GetScalarFromArray`` and every supported ``FuncCall`` become ops;
* ``Record`` / ``Wait`` / ``Join`` / ``Deallocate`` / ``RemoveRegister`` need no op: a request
  runs all of its program's streams as the one stream of its slot, in program order, and its
  memory is one block released when it completes;
* ``Return`` names the results, copied to the caller when the request completes.

Supported kernels (the single-GPU data plane): NttPrcompute, NttRecompute, DistributePowers,
FusedArith (not pipelined; the kernel is this package's FusedOp registered under the artifact's
kernel name, since an artifact names its generated libraries but holds no graph), Msm (device
bases; a point-base constant registered with precomputed tables uses them), EvaluatePoly,
BatchedInvert, KateDivision, ScanMul, PolyAdd, PolySub, NewZero, NewOneLagrange, NewOneCoef,
ScalarInvert and ScalarPow on the GPU.  Anything else - CPU kernels, transcripts, user
functions, Fork, Blind, disk and paged allocations - raises ``ValueError`` naming the
instruction, where the reference would run it on the host.
"""
from __future__ import annotations

import ctypes
import glob
import json
import os
from dataclasses import dataclass, field, replace

import numpy as np
import torch

from . import artifact as art
from .native import ZKP_PROG_MAX_VIEWS, PolyPtr, ZkpMsmTask, ZkpProgOp, ZkpProgOut, ZkpProgView, check, load

SPACE_NONE, SPACE_DEVICE, SPACE_HOST, SPACE_ABS, SPACE_INPUT = range(5)
(OP_COPY, OP_ZERO, OP_NTT, OP_NTT_RECOMPUTE, OP_DISTRIBUTE, OP_FUSED, OP_MSM, OP_EVAL, OP_INVERT, OP_KATE,
 OP_SCAN, OP_ADD, OP_SUB, OP_ZERO_POLY, OP_ONE_LAGRANGE, OP_ONE_COEF, OP_SCALAR_INV, OP_SCALAR_POW) = range(1, 19)

ALIGN = 256
POLYPTR_BYTES = ctypes.sizeof(PolyPtr)


def _al(x: int) -> int:
    return (x + ALIGN - 1) // ALIGN * ALIGN


# ------------------------------------------------------------------ artifact files
def version_files(directory: str) -> list[str]:
    """The ``version_*.json`` chunks of an artifact (Versions::load, compiler/src/driver.rs:542-565)."""
    return sorted(p for p in glob.glob(os.path.join(directory, "version_*.json")) if os.path.isfile(p))


def read_chunk(directory: str, version: str | None = None) -> tuple[dict, dict, dict]:
    """(memory_info, chunk, statistics) of one version (the only one when ``version`` is None)."""
    files = version_files(directory)
    if version is not None:
        files = [f for f in files if os.path.basename(f) == version]
    if len(files) != 1:
        raise ValueError(f"{directory}: expected one version file, found {[os.path.basename(f) for f in files]}")
    with open(files[0]) as f:
        doc = json.load(f)
    if not (isinstance(doc, list) and len(doc) == 3 and isinstance(doc[1], dict)):
        raise ValueError(f"{files[0]}: not a (MemoryInfo, Chunk, Statistics) triple")
    chunk = doc[1]
    for key in ("instructions", "f_table", "event_table", "n_variables", "n_threads"):
        if key not in chunk:
            raise ValueError(f"{files[0]}: chunk has no {key!r}")
    return doc[0], chunk, doc[2]


def heap_items(h) -> list:
    """Items of a serialised ``Heap(Vec<T>, PhantomData)`` (common/src/heap.rs:74-75)."""
    if isinstance(h, list) and len(h) == 2 and isinstance(h[0], list) and h[1] is None:
        return h[0]
    raise ValueError(f"not a serialised Heap: {h!r:.80}")


def node_of(instr):
    """(kind, payload) of an Instruction's node (serde external tagging)."""
    node = instr["node"] if isinstance(instr, dict) and "node" in instr else instr
    if isinstance(node, str):
        return node, None
    if isinstance(node, dict) and len(node) == 1:
        return next(iter(node.items()))
    raise ValueError(f"malformed instruction {instr!r:.120}")


def kernel_kind(kt) -> tuple[str, object]:
    if isinstance(kt, str):
        return kt, None
    if isinstance(kt, dict) and len(kt) == 1:
        return next(iter(kt.items()))
    raise ValueError(f"malformed KernelType {kt!r:.80}")


def msm_precompute_tables(config: dict) -> int:
    """Point tables an Msm call takes (MsmConfig::get_precompute, common/src/msm_config.rs:17-25)."""
    bits, w, target = int(config["bits"]), int(config["window_size"]), int(config["target_window"])
    actual = -(-bits // w)
    n_windows = actual if actual < target else target
    return -(-actual // n_windows)


# ------------------------------------------------------------------ variables
@dataclass
class Var:
    """A resolved variable: elements of ``eb`` bytes, element i at
    base + ((i + offset + whole - rotate) mod whole) * eb in ``space``."""
    kind: str                    # poly, scalar, point, points, buffer, stream, tuple
    device: str                  # gpu or cpu
    space: int = SPACE_NONE
    addr: int = 0
    index: int = 0
    len: int = 0
    rotate: int = 0
    offset: int = 0
    whole: int = 0
    sliced: bool = False
    members: list = field(default_factory=list)

    @property
    def eb(self) -> int:
        return {"poly": 32, "scalar": 32, "point": 64, "points": 64, "buffer": 1}.get(self.kind, 0)

    def view(self) -> ZkpProgView:
        return ZkpProgView(self.space, self.index, self.addr, self.len, self.rotate % max(self.whole, 1),
                           self.offset, self.whole)

    def contiguous(self) -> bool:
        start = (self.offset - self.rotate) % max(self.whole, 1)
        return start + self.len <= self.whole

    def start(self) -> int:
        return (self.offset - self.rotate) % max(self.whole, 1)


def _typ_var(typ, device: str) -> Var:
    kind = art.typ_kind(typ)
    if kind == "ScalarArray":
        n = int(typ["ScalarArray"]["len"])
        return Var("poly", device, len=n, whole=n)
    if kind == "PointBase":
        n = int(typ["PointBase"]["len"])
        return Var("points", device, len=n, whole=n)
    if kind == "Scalar":
        return Var("scalar", device, len=1, whole=1)
    if kind == "Point":
        return Var("point", device, len=1, whole=1)
    if kind == "GpuBuffer":
        n = int(typ["GpuBuffer"][0])
        return Var("buffer", device, len=n, whole=n)
    if kind == "Stream":
        return Var("stream", device)
    raise ValueError(f"type {typ!r} is not part of the served data plane")


def _device_of(d) -> str:
    if d == "CPU":
        return "cpu"
    if isinstance(d, dict) and set(d) == {"GPU"}:
        return "gpu"
    raise ValueError(f"device {d!r} is not part of the served data plane (disk pools stay out)")


# ------------------------------------------------------------------ lowering
class Lowering:
    """Turns a chunk into the native op list (see the module docstring)."""

    def __init__(self, chunk: dict, constants: list, input_types: list, fused: dict, bases: dict | None = None):
        self.chunk = chunk
        self.constants = constants
        self.input_types = list(input_types)
        self.fused = fused
        self.bases = bases or {}
        self.f_table = heap_items(chunk["f_table"])
        self.vars: dict[int, Var] = {}
        self.ops: list[ZkpProgOp] = []
        self.keep: list = []            # tensors the ops address (device copies, Shoup tables)
        self.fns: dict[str, object] = {}
        self.dev_top = 0
        self.host_top = 0
        self.outputs: list[tuple[int, int, str]] = []  # (host offset, bytes, kind)
        self.returned = None
        self._shoup: dict[int, torch.Tensor] = {}
        self._dev_const: dict[int, torch.Tensor] = {}
        self._tensors: dict[int, torch.Tensor] = {}   # address -> constant tensor

    # ---- planning
    def dev_alloc(self, nbytes: int) -> int:
        off = self.dev_top
        self.dev_top += _al(max(nbytes, 1))
        return off

    def host_alloc(self, nbytes: int) -> int:
        off = self.host_top
        self.host_top += _al(max(nbytes, 1))
        return off

    def fresh(self, kind: str, device: str, n: int) -> Var:
        eb = {"poly": 32, "scalar": 32, "point": 64, "points": 64, "buffer": 1}[kind]
        if device == "gpu":
            return Var(kind, device, SPACE_DEVICE, self.dev_alloc(n * eb), len=n, whole=n)
        return Var(kind, device, SPACE_HOST, self.host_alloc(n * eb), len=n, whole=n)

    def get(self, vid: int, where: str) -> Var:
        if vid not in self.vars:
            raise ValueError(f"{where}: variable {vid} is undefined")
        return self.vars[vid]

    # ---- op emission
    def emit(self, kind: int, views: dict, imm=(0, 0, 0, 0)) -> None:
        op = ZkpProgOp()
        op.kind = kind
        op.n_views = ZKP_PROG_MAX_VIEWS
        for j, x in enumerate(imm):
            op.imm[j] = int(x)
        for j, v in views.items():
            op.v[j] = v if isinstance(v, ZkpProgView) else v.view()
        self.ops.append(op)

    def copy(self, dst: Var, src: Var, where: str) -> None:
        if dst.len != src.len or dst.eb != src.eb or dst.eb not in (32, 64):
            raise ValueError(f"{where}: cannot copy {src.kind}[{src.len}] into {dst.kind}[{dst.len}]")
        if dst.space == SPACE_INPUT or dst.space == SPACE_ABS:
            raise ValueError(f"{where}: the destination is read-only (an input or a constant)")
        if dst.len:
            self.emit(OP_COPY, {0: dst, 1: src}, (dst.eb, 0, 0, 0))

    @staticmethod
    def need(cond: bool, where: str, what: str) -> None:
        if not cond:
            raise ValueError(f"{where}: {what}")

    def gpu(self, v: Var, where: str, kinds=("poly",)) -> Var:
        self.need(v.kind in kinds, where, f"expected {'/'.join(kinds)}, got {v.kind}")
        self.need(v.device == "gpu" and v.space in (SPACE_DEVICE, SPACE_ABS), where,
                  f"{v.kind} operand must be in GPU memory")
        return v

    def temp(self, given: Var, nbytes: int) -> Var:
        """The FuncCall's temp buffer when it is a device buffer large enough for this
        package's kernel; otherwise a buffer of the right size in the request block (the
        reference sizes temps for its own kernels)."""
        if given is not None and given.kind == "buffer" and given.space == SPACE_DEVICE and given.len >= nbytes:
            return given
        return self.fresh("buffer", "gpu", max(nbytes, 1))

    # ---- constants
    def const_var(self, cid: int, where: str) -> Var:
        self.need(0 <= cid < len(self.constants), where, f"constant {cid} is not in the table")
        c = self.constants[cid]
        kind = art.typ_kind(c.typ)
        value = c.value
        if kind == "ScalarArray":
            t = value.values[: value.len] if hasattr(value, "values") else value
            v = Var("poly", "gpu" if t.is_cuda else "cpu", len=value.len if hasattr(value, "len") else t.shape[0])
        elif kind == "PointBase":
            t = value
            v = Var("points", "gpu" if t.is_cuda else "cpu", len=t.shape[0])
        elif kind == "Scalar":
            t = value
            v = Var("scalar", "gpu" if t.is_cuda else "cpu", len=1)
        elif kind == "Point":
            t = value
            v = Var("point", "gpu" if t.is_cuda else "cpu", len=1)
        else:
            raise ValueError(f"{where}: constant {cid} ({c.name!r}) of type {c.typ!r} is not part of the data plane")
        t = t.contiguous()
        self.keep.append(t)
        self._tensors[t.data_ptr()] = t
        v.space, v.addr, v.whole = SPACE_ABS, t.data_ptr(), v.len
        v.members = [cid]  # remembers the constant it came from
        return v

    def device_copy(self, v: Var) -> Var:
        """A host-resident constant made resident in HBM once, at program load."""
        if v.addr not in self._dev_const:
            t = self._tensors[v.addr].cuda()
            self._dev_const[v.addr] = t
            self._tensors[t.data_ptr()] = t
            self.keep.append(t)
        return replace(v, device="gpu", addr=self._dev_const[v.addr].data_ptr())

    def shoup_for(self, tw: Var, log_n: int) -> int:
        """Shoup table of a full root table constant (built once, like the root table itself)."""
        from . import ntt
        from .scalar import ScalarArray
        if tw.space != SPACE_ABS or tw.len != (1 << log_n) // 2 or tw.whole != tw.len or tw.rotate or tw.offset \
                or log_n < 1:
            return 0
        if tw.addr not in self._shoup:
            words = self._tensors.get(tw.addr)
            if words is None or not words.is_cuda:
                return 0
            self._shoup[tw.addr] = ntt.shoup_table_of(ScalarArray(words.view(torch.int32).reshape(-1, 8)))
            self.keep.append(self._shoup[tw.addr])
        return self._shoup[tw.addr].data_ptr()

    # ---- fused kernels
    def fused_fn(self, meta: dict, where: str):
        from .fused import FusedGraph, FusedKernel, FusedOp
        name = meta["name"]
        self.need(meta.get("pipelined_meta") is None, where, f"pipelined fused kernel {name!r} is not served")
        if name not in self.fns:
            self.need(name in self.fused, where, f"no fused kernel registered under {name!r}")
            k = self.fused[name]
            if isinstance(k, FusedGraph):
                k = FusedOp(k, name)
            if isinstance(k, FusedOp):
                k = FusedKernel(k)
            g = k.op.graph
            self.need(g.num_vars == meta["num_vars"] and g.num_mut_vars == meta["num_mut_vars"], where,
                      f"fused kernel {name!r}: graph has {g.num_vars}/{g.num_mut_vars} inputs/outputs, "
                      f"the artifact {meta['num_vars']}/{meta['num_mut_vars']}")
            self.fns[name] = k
        return self.fns[name]

    # ---- the walk
    def run(self) -> None:
        instrs = self.chunk["instructions"]
        # the compiler's device plan: offsets of Offset allocations; Dynamic ones go after it
        for i, ins in enumerate(instrs):
            kind, p = node_of(ins)
            if kind == "Allocate" and _device_of(p["device"]) == "gpu":
                am = p["alloc_method"]
                if isinstance(am, dict) and "Offset" in am:
                    off, size = am["Offset"]
                    self.dev_top = max(self.dev_top, _al(int(off) + int(size)))
        for i, ins in enumerate(instrs):
            self.step(i, *node_of(ins))

    def step(self, i: int, kind: str, p) -> None:
        where = f"instruction {i} ({kind})"
        V = self.vars
        if kind == "Allocate":
            dev = _device_of(p["device"])
            v = _typ_var(p["typ"], dev)
            am = p["alloc_method"]
            if v.kind == "stream":
                pass
            elif dev == "gpu":
                if isinstance(am, dict) and "Offset" in am:
                    off, size = (int(x) for x in am["Offset"])
                    self.need(size >= v.whole * v.eb, where, f"Offset size {size} < {v.whole * v.eb} bytes")
                    v.space, v.addr = SPACE_DEVICE, off
                elif isinstance(am, dict) and "Dynamic" in am:
                    v.space, v.addr = SPACE_DEVICE, self.dev_alloc(v.whole * v.eb)
                else:
                    raise ValueError(f"{where}: allocation {am!r:.60} is not served (paged memory stays out)")
            else:
                v.space, v.addr = SPACE_HOST, self.host_alloc(v.whole * v.eb)
            V[int(p["id"])] = v
        elif kind in ("Deallocate", "RemoveRegister"):
            self.get(int(p["id"]), where)
            V.pop(int(p["id"]))
        elif kind == "Transfer":
            src, dst = self.get(int(p["src_id"]), where), self.get(int(p["dst_id"]), where)
            self.need(src.kind == dst.kind or {src.kind, dst.kind} <= {"poly", "scalar"}, where,
                      f"transfer {src.kind} -> {dst.kind}")
            self.copy(dst, src, where)
        elif kind == "FuncCall":
            self.func_call(where, int(p["func_id"]), [int(x) for x in p["arg_mut"]], [int(x) for x in p["arg"]])
        elif kind in ("Record", "Wait", "Join"):
            pass  # one stream per request: program order is stream order
        elif kind == "Fork":
            raise ValueError(f"{where}: multi-threaded chunks are not served")
        elif kind == "Rotation":
            src = self.get(int(p["src"]), where)
            self.need(src.kind == "poly" and not src.sliced, where, "rotation of a sliced or non-poly variable")
            V[int(p["dst"])] = replace(src, rotate=(src.rotate + int(p["shift"])) % max(src.len, 1))
        elif kind == "Slice":
            src = self.get(int(p["src"]), where)
            start, end = int(p["start"]), int(p["end"])
            self.need(src.kind == "poly" and not src.sliced and 0 <= start <= end <= src.len, where,
                      f"slice [{start}, {end}) of {src.kind}[{src.len}]")
            actual = (src.len + start - src.rotate) % max(src.len, 1)
            V[int(p["dst"])] = replace(src, len=end - start, rotate=0, offset=actual, whole=src.len, sliced=True)
        elif kind == "SetSliceMeta":
            src = self.get(int(p["src"]), where)
            whole = src.whole
            off, n = int(p["offset"]) % max(whole, 1), int(p["len"])
            self.need(n <= whole, where, "slice longer than its array")
            V[int(p["dst"])] = replace(src, len=n, rotate=0, offset=off, whole=whole,
                                       sliced=not (n == whole and off == 0))
        elif kind == "SliceBuffer":
            src = self.get(int(p["src"]), where)
            off, n = int(p["offset"]), int(p["len"])
            self.need(src.kind == "buffer" and off + n <= src.len, where, "buffer slice out of range")
            V[int(p["dst"])] = replace(src, addr=src.addr + off, len=n, whole=n)
        elif kind == "LoadConstant":
            V[int(p["dst"])] = self.const_var(int(p["src"]), where)
        elif kind == "LoadInput":
            e = int(p["src"])
            self.need(0 <= e < len(self.input_types), where, f"input {e} has no declared type")
            v = _typ_var(self.input_types[e], "cpu")
            v.space, v.index, v.addr = SPACE_INPUT, e, 0
            V[int(p["dst"])] = v
        elif kind == "AssembleTuple":
            V[int(p["dst"])] = Var("tuple", "cpu", members=[self.get(int(x), where) for x in p["vars"]])
        elif kind in ("MoveRegister", "CopyRegister"):
            src = self.get(int(p["src"]), where)
            V[int(p["dst"])] = src
            if kind == "MoveRegister":
                V.pop(int(p["src"]))
        elif kind == "GetScalarFromArray":
            src, dst = self.get(int(p["src"]), where), self.get(int(p["dst"]), where)
            idx = int(p["idx"])
            self.need(src.kind == "poly" and dst.kind == "scalar" and idx < src.len, where, "bad scalar extraction")
            elem = replace(src, len=1, offset=(src.start() + idx) % src.whole, rotate=0, sliced=True)
            self.copy(dst, elem, where)
        elif kind == "Return":
            self.returned = self.get(int(p), where)
        else:
            raise ValueError(f"{where}: not part of the served data plane")

    def func_call(self, where: str, fid: int, arg_mut: list, arg: list) -> None:
        self.need(0 <= fid < len(self.f_table), where, f"function {fid} is not in the table")
        kt, meta = kernel_kind(self.f_table[fid])
        where = f"{where} {kt}"
        m = [self.get(x, where) for x in arg_mut]
        a = [self.get(x, where) for x in arg]

        def stream_last():
            self.need(a and a[-1].kind == "stream", where, "the last argument must be the stream")

        if kt == "NttPrcompute":
            self.need(len(m) == 1 and len(a) == 2, where, "arg_mut = [poly], arg = [twiddle, stream]")
            stream_last()
            x, tw = self.gpu(m[0], where), self.gpu(a[0], where)
            log_n = x.len.bit_length() - 1
            self.need(x.len == 1 << log_n and tw.len * 2 >= x.len, where, "size is not a power of two / short table")
            self.emit(OP_NTT, {0: x, 1: tw}, (self.shoup_for(tw, log_n), 0, 0, 0))
        elif kt == "NttRecompute":
            self.need(len(m) == 1 and len(a) == 3, where, "arg_mut = [poly], arg = [pq, omega, stream]")
            stream_last()
            x, pq, om = self.gpu(m[0], where), self.gpu(a[0], where), self.gpu(a[1], where)
            pq_deg = (pq.len & -pq.len).bit_length() - 1 + 1  # trailing zeros + 1 (core/src/ntt.rs:265)
            self.emit(OP_NTT_RECOMPUTE, {0: x, 1: pq, 2: om}, (pq_deg, 0, 0, 0))
        elif kt == "DistributePowers":
            self.need(len(m) == 1 and len(a) == 2, where, "arg_mut = [poly], arg = [powers, stream]")
            stream_last()
            self.emit(OP_DISTRIBUTE, {0: self.gpu(m[0], where), 1: self.gpu(a[0], where)})
        elif kt == "FusedArith":
            self.fused_call(where, meta, m, a)
        elif kt == "Msm":
            self.msm_call(where, meta, m, a)
        elif kt == "EvaluatePoly":
            self.need(len(m) == 2 and len(a) == 3, where, "arg_mut = [temp, res], arg = [poly, x, stream]")
            stream_last()
            poly = self.gpu(a[0], where)
            temp = self.temp(m[0], self.poly_temp("poly_eval", poly.len))
            self.emit(OP_EVAL, {0: temp, 1: self.gpu(m[1], where, ("scalar",)), 2: poly,
                                3: self.gpu(a[1], where, ("scalar",))})
        elif kt == "BatchedInvert":
            self.need(len(m) == 2 and len(a) == 1, where, "arg_mut = [temp, poly], arg = [stream]")
            stream_last()
            poly = self.gpu(m[1], where)
            self.emit(OP_INVERT, {0: self.temp(m[0], self.poly_temp("batched_invert", poly.len)), 1: poly})
        elif kt == "KateDivision":
            self.need(len(m) == 2 and len(a) == 3, where, "arg_mut = [temp, res], arg = [poly, b, stream]")
            stream_last()
            p = self.gpu(a[0], where)
            self.emit(OP_KATE, {0: self.temp(m[0], self.poly_temp("kate_division", p.len)),
                                1: self.gpu(m[1], where), 2: p, 3: self.gpu(a[1], where, ("scalar",))})
        elif kt == "ScanMul":
            # core/src/poly.rs:428-468: target[0] = x0, target[1..] = poly[..len-1], then the scan
            self.need(len(m) == 2 and len(a) == 3, where, "arg_mut = [temp, res], arg = [poly, x0, stream]")
            stream_last()
            t, p, x0 = self.gpu(m[1], where), self.gpu(a[0], where), self.gpu(a[1], where, ("scalar",))
            self.need(t.len == p.len and t.len >= 1, where, "target and poly differ in length")
            self.copy(replace(t, len=1, offset=t.start(), rotate=0, sliced=True), x0, where)
            if t.len > 1:
                self.copy(replace(t, len=t.len - 1, offset=(t.start() + 1) % t.whole, rotate=0, sliced=True),
                          replace(p, len=p.len - 1, offset=p.start(), rotate=0, sliced=True), where)
            self.emit(OP_SCAN, {0: self.temp(m[0], self.poly_temp("scan_mul", t.len)), 1: t})
        elif kt in ("PolyAdd", "PolySub"):
            self.need(len(m) == 1 and len(a) == 3, where, "arg_mut = [res], arg = [a, b, stream]")
            stream_last()
            self.emit(OP_ADD if kt == "PolyAdd" else OP_SUB,
                      {0: self.gpu(m[0], where), 1: self.gpu(a[0], where), 2: self.gpu(a[1], where)})
        elif kt in ("NewZero", "NewOneLagrange", "NewOneCoef"):
            self.need(len(m) == 1 and len(a) == 1, where, "arg_mut = [target], arg = [stream]")
            stream_last()
            op = {"NewZero": OP_ZERO_POLY, "NewOneLagrange": OP_ONE_LAGRANGE, "NewOneCoef": OP_ONE_COEF}[kt]
            self.emit(op, {0: self.gpu(m[0], where)})
        elif kt in ("ScalarInvert", "ScalarPow"):
            self.need(len(m) == 1 and len(a) == 1, where, "a GPU scalar and a stream (CPU scalar kernels are not "
                                                          "served)")
            stream_last()
            x = self.gpu(m[0], where, ("scalar",))
            if kt == "ScalarInvert":
                self.emit(OP_SCALAR_INV, {0: x})
            else:
                self.emit(OP_SCALAR_POW, {0: x}, (int(meta), 0, 0, 0))
        else:
            raise ValueError(f"{where}: kernel type {kt} is not part of the served data plane")

    def poly_temp(self, fn: str, n: int) -> int:
        from .poly import _lib, _null_ptr, _query
        lib = _lib()
        if fn == "poly_eval":
            return _query(lib.poly_eval, _null_ptr(n), None, None, None)
        if fn == "kate_division":
            log_p = max(n.bit_length() - 1, 0)
            return _query(lib.kate_division, log_p, _null_ptr(n), None, _null_ptr(n), None)
        return _query(getattr(lib, fn), _null_ptr(n), None)

    def fused_call(self, where: str, meta: dict, m: list, a: list) -> None:
        # emit_func.rs:25-46: arg_mut = [arg buffer, local buffer, outputs...], arg = [stream, inputs...]
        k = self.fused_fn(meta, where)
        nv, nm = int(meta["num_vars"]), int(meta["num_mut_vars"])
        self.need(len(a) == nv + 1 and len(m) == nm + 2, where, "argument count differs from the kernel's")
        self.need(a[0].kind == "stream", where, "the first argument must be the stream")
        self.need(nv + nm <= 14, where, "more than 14 fused operands")
        argbuf = m[0]
        self.need(argbuf.kind == "buffer" and argbuf.space == SPACE_DEVICE and
                  argbuf.len >= (nv + nm) * POLYPTR_BYTES, where, "the argument buffer is too small")
        g = k.op.graph
        periodic = {n[4] for n in g.nodes if n[0] == "input" and n[2] == "periodic" and n[3] == "var"}
        views, length = {}, 0
        for j, v in enumerate(a[1:] + m[2:]):
            self.gpu(v, where, ("poly", "scalar"))
            views[j] = v
            if v.kind == "poly" and not (j < nv and j in periodic):
                if length in (0, 1):
                    length = v.len
                else:
                    self.need(length == v.len, where, "fused operands differ in length")
            elif length == 0:
                length = 1
        self.need(length > 0, where, "fused kernel over nothing")
        views[14] = replace(argbuf, len=(nv + nm) * POLYPTR_BYTES, whole=(nv + nm) * POLYPTR_BYTES)
        views[15] = self.fresh("buffer", "cpu", (nv + nm) * POLYPTR_BYTES)
        fn = ctypes.cast(k.fn, ctypes.c_void_p).value
        self.emit(OP_FUSED, views, (fn, nv, nm, length))

    def msm_call(self, where: str, config: dict, m: list, a: list) -> None:
        # emit_func.rs:364-391: arg = [point tables..., scalars...], arg_mut = [buffers per card..., answers...]
        n_pre = msm_precompute_tables(config)
        cards = len(config["cards"])
        tables, scal = a[:n_pre], a[n_pre:]
        answers = m[cards:]
        self.need(len(tables) == n_pre and scal and len(answers) == len(scal), where,
                  f"expected {n_pre} tables, then one scalar array per answer")
        self.need(len(scal) <= 7, where, "more than 7 MSMs in one call")
        for t in tables:
            self.need(t.kind == "points", where, "point tables must be PointBase values")
        rows = tables[0].len
        registered = None
        if tables[0].members and tables[0].members[0] < len(self.constants):
            registered = self.bases.get(self.constants[tables[0].members[0]].name)
        if registered is not None:
            base_ptr, nt, window, rows = (registered.tables.data_ptr(), registered.n_tables, registered.window,
                                          registered.n)
        else:
            dev = [self.device_copy(t) if t.device == "cpu" else t for t in tables]
            if n_pre > 1:
                # the n tables of MSMPrecompute side by side, as zkp_msm_batch reads them
                stacked = torch.empty((n_pre * rows, 16), dtype=torch.int32, device="cuda")
                for j, t in enumerate(dev):
                    stacked[j * rows:(j + 1) * rows].copy_(self._tensors[t.addr].view(torch.int32).reshape(-1, 16))
                self.keep.append(stacked)
                base_ptr = stacked.data_ptr()
            else:
                base_ptr = dev[0].addr
            nt, window = n_pre, int(config["window_size"])
        tasks = (ZkpMsmTask * len(scal))()
        views, posts = {}, []
        for j, s in enumerate(scal):
            self.need(s.kind == "poly" and s.len <= rows and s.contiguous() and s.rotate % max(s.whole, 1) == 0,
                      where, "MSM scalars must be an unrotated contiguous array no longer than the bases")
            if s.device != "gpu":
                staged = self.fresh("poly", "gpu", s.len)
                self.copy(staged, s, where)
                s = staged
            views[j] = replace(s, addr=s.addr + s.start() * 32, offset=0, rotate=0, whole=s.len, sliced=False)
            ans = answers[j]
            self.need(ans.kind == "point", where, "MSM answers are Point variables")
            if ans.device == "gpu" and ans.space == SPACE_DEVICE:
                views[len(scal) + j] = ans
            else:
                slot = self.fresh("point", "gpu", 1)
                views[len(scal) + j] = slot
                posts.append((ans, slot))
            tasks[j] = ZkpMsmTask(base_ptr, nt, 16, s.len, window, 16, rows)
        ws_bytes = int(load("libmsm.so").zkp_msm_batch_workspace_size(tasks, len(scal)))
        self.need(ws_bytes > 0, where, "MSM configuration refused by the library")
        views[15] = self.fresh("buffer", "gpu", ws_bytes)
        self.emit(OP_MSM, views, (base_ptr, nt | (window << 16), rows, len(scal)))
        for ans, slot in posts:
            self.copy(ans, slot, where)

    # ---- results
    def results(self) -> list[tuple[int, int, str, int]]:
        """(host offset, bytes, kind, elements) per returned leaf, copied to host space first
        where a leaf lives elsewhere or is not contiguous."""
        if self.returned is None:
            return []
        leaves = []

        def walk(v):
            if v.kind == "tuple":
                for x in v.members:
                    walk(x)
            else:
                leaves.append(v)
        walk(self.returned)
        out = []
        for v in leaves:
            if v.kind not in ("poly", "scalar", "point", "points"):
                raise ValueError(f"Return: a {v.kind} value cannot be returned to the host")
            if not (v.space == SPACE_HOST and v.contiguous()):
                h = self.fresh(v.kind, "cpu", v.len)
                self.copy(h, v, "Return")
                v = h
            out.append((v.addr + v.start() * v.eb, v.len * v.eb, v.kind, v.len))
        return out


def resident_table(table: list, gpu_mapping=None) -> list:
    """A constant table with every binary value on its manifest device, in the forms
    artifact.load_constant_table returns (ScalarArray polynomials, int32 word tensors)."""
    out = []
    for c in table:
        if art.binary_size(c.typ) is None:
            out.append(c)
            continue
        words = art._value_tensor(c).to(art.torch_device(c.device, gpu_mapping), copy=True)
        out.append(art.Constant(c.name, c.typ, c.device, art._wrap(c.typ, words)))
    return out


# ------------------------------------------------------------------ the served program
class CompiledProgram:
    """A compiled artifact registered with a serving.Server.

    ``fused`` maps the artifact's fused kernel names to this package's graphs (FusedGraph /
    FusedOp / FusedKernel), ``bases`` point-base constant names to msm.ResidentBases whose
    precomputed tables the MSMs should use, ``input_types`` the serde Typ of each input entry
    (the runtime's input table, which the artifact does not record)."""

    def __init__(self, server, chunk: dict, constants: list, input_types: list, fused: dict | None = None,
                 bases: dict | None = None):
        self.server = server
        low = Lowering(chunk, constants, input_types, fused or {}, bases)
        low.run()
        self.lowering = low
        self.leaves = low.results()
        self.ops = (ZkpProgOp * max(len(low.ops), 1))(*low.ops)
        self.n_ops = len(low.ops)
        self.device_bytes, self.host_bytes = low.dev_top, low.host_top
        self.input_bytes = [_typ_var(t, "cpu").whole * _typ_var(t, "cpu").eb for t in input_types]
        outs, off = [], 0
        for host_off, nbytes, _, _ in self.leaves:
            outs.append(ZkpProgOut(host_off, nbytes, off))
            off += nbytes
        self.result_bytes = off
        self._outs = (ZkpProgOut * max(len(outs), 1))(*outs)
        ib = (ctypes.c_ulonglong * max(len(self.input_bytes), 1))(*self.input_bytes)
        self.h = ctypes.c_void_p()
        torch.cuda.synchronize()  # constants and derived tables resident before any request
        check(server.lib.zkp_serve_program_create(server.h, self.ops, self.n_ops, self.device_bytes, self.host_bytes,
                                                  self._outs, len(outs), ib, len(self.input_bytes),
                                                  ctypes.byref(self.h)), "zkp_serve_program_create")
        self._live = {}

    @staticmethod
    def from_parts(server, chunk: dict, table: list, input_types: list, fused: dict | None = None,
                   bases: dict | None = None, gpu_mapping=None) -> "CompiledProgram":
        """A program built in memory (prover_artifact) rather than read from files: the same
        lowering over the constant table placed as load_constant_table would place it."""
        return CompiledProgram(server, chunk, resident_table(table, gpu_mapping), input_types, fused, bases)

    @staticmethod
    def load(server, directory: str, input_types: list, fused: dict | None = None, bases: dict | None = None,
             version: str | None = None, table: list | None = None, gpu_mapping=None) -> "CompiledProgram":
        """Reads an artifact directory: its chunk and its constant table (loaded into memory)."""
        _, chunk, _ = read_chunk(directory, version)
        constants = art.load_constant_table(directory, table, gpu_mapping)
        return CompiledProgram(server, chunk, constants, input_types, fused, bases)

    def submit(self, inputs: list) -> int:
        """inputs: host arrays (numpy uint32/uint64 or CPU tensors) per input entry."""
        arrs = []
        for i, (x, need) in enumerate(zip(inputs, self.input_bytes)):
            if isinstance(x, torch.Tensor):
                x = x.numpy()
            x = np.ascontiguousarray(x)
            if x.nbytes != need:
                raise ValueError(f"input {i}: {x.nbytes} bytes, the program reads {need}")
            arrs.append(x)
        if len(arrs) != len(self.input_bytes):
            raise ValueError(f"{len(arrs)} inputs given, the program has {len(self.input_bytes)}")
        res = np.zeros(max(self.result_bytes, 1), dtype=np.uint8)
        ptrs = (ctypes.c_void_p * max(len(arrs), 1))(*[a.ctypes.data for a in arrs])
        t = self.server.lib.zkp_serve_submit_program(self.server.h, self.h, ptrs, len(arrs), res.ctypes.data,
                                                     res.nbytes)
        if t < 0:
            raise RuntimeError("server is shutting down")
        self._live[t] = (arrs, res, ptrs)  # kept alive until the request completes
        return t

    def wait(self, ticket: int, timeout_s: float = 600.0):
        """(ZkpProverResult, [leaf arrays]) - each returned value as uint32 words (points (16,),
        scalars (8,), polynomials (n, 8))."""
        r = self.server.wait(ticket, timeout_s)
        arrs, res, _ = self._live.pop(ticket)
        out = []
        off = 0
        for _, nbytes, kind, n in self.leaves:
            w = res[off:off + nbytes].view(np.uint32)
            out.append(w.reshape(n, -1) if kind in ("poly", "points") else w.copy())
            off += nbytes
        return r, out

    def close(self):
        """Waits for this program's outstanding requests (their input and result buffers live
        in this object), then destroys the native program."""
        if self.h:
            for t in list(self._live):
                self.wait(t)
            self.server.lib.zkp_serve_program_destroy(self.server.h, self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass



# ------------------------------------------------------------------ the prover program as an artifact
def _ins(node, track="MemoryManagement", stream=None) -> dict:
    return {"node": node, "track": track, "stream": stream}


def prover_fused_graphs() -> dict:
    """The two fused kernels of the prover program, by the names its artifact gives them:
    the INTT's scaling by n^-1 in place (intt_mending.rs:11-70, fused) and the quotient
    (e*e - e - z*z(wX)) / Z_H with 1/Z_H periodic."""
    from .fused import FusedGraph
    scale = FusedGraph([
        ("input", "p", "poly", "mut", 0),
        ("input", "s", "scalar", "var", 0),
        ("mul", "r", "p", "s"),
        ("output", 0, "r"),
    ])
    quotient = FusedGraph([
        ("input", "a", "poly", "var", 0), ("input", "b", "poly", "var", 1), ("input", "c", "poly", "var", 2),
        ("input", "z", "poly", "var", 3), ("input", "zw", "poly", "var", 4), ("input", "zh", "periodic", "var", 5),
        ("mul", "ab", "a", "b"), ("sub", "t0", "ab", "c"), ("mul", "zz", "z", "zw"), ("sub", "t1", "t0", "zz"),
        ("mul", "q", "t1", "zh"), ("output", 0, "q"),
    ])
    return {"prover_scale_ninv": scale, "prover_quotient": quotient}


def prover_input_types(k: int, ext: int = 2) -> list:
    n, N = 1 << k, 1 << (k + ext)
    return [art.scalar_array_typ(n)] * 3 + [art.scalar_array_typ(N), "Scalar"]


def prover_constants(k: int, ext: int = 2, points=None) -> dict:
    """The prover program's constants, computed by this package (device tensors, small host
    arrays): inverse roots of 2^k, forward roots of 2^(k+ext) (the ssip_precompute tables),
    n^-1, the coset powers 7^i (i < 2^k), 1/Z_H at the 2^ext coset classes, and the first 2^k
    rows of ``points`` ((rows, 16) int32 device tensor) as the bases."""
    from . import ntt, pipeline
    from .field import FR_MODULUS, GENERATOR, mont_words
    n = 1 << k
    out = {"inv_twiddle": ntt.twiddle_table(k, True).values,
           "fwd_twiddle": ntt.twiddle_table(k + ext, False).values,
           "n_inv": mont_words(pow(n, -1, FR_MODULUS)).reshape(1, 8),
           "zh_inv": np.stack([mont_words(v) for v in pipeline.zh_inv_values(k, ext)])}
    g = mont_words(GENERATOR)
    powers = torch.from_numpy(np.tile(g.view(np.int32)[None, :], (n, 1)).copy()).cuda()
    # [1, g, g^2, ...]: the roots routine over the generator instead of a root of unity
    unit = torch.from_numpy(g.view(np.int32).copy()).cuda()
    check(load("libntt.so").zkp_ntt_roots_device(powers.data_ptr(), n, unit.data_ptr(), None),
          "zkp_ntt_roots_device")
    out["coset_powers"] = powers
    if points is not None:
        out["bases"] = points[:n]
    torch.cuda.synchronize()
    return out


def prover_artifact(k: int, consts: dict, ext: int = 2, window: int = 16, device_id: int = 0):
    """The served prover program of size k (include/zkp_runtime.h) as the reference's compiler
    hands a program to its runtime: (memory_info, chunk, statistics, constant table).

    Inputs (entries 0-4): a, b, c (Lagrange, 2^k values), z (on the 2^ext-times coset), x.
    Program: three INTTs (NttPrcompute with the inverse roots, then the fused scaling by
    n^-1), the coset NTT of c (NewZero of the extended array, c copied into its first 2^k
    entries, DistributePowers by 7^i, NttPrcompute), the fused quotient over (e, e, e, z, z
    rotated by -2^ext, 1/Z_H), one Msm call of four scalar arrays (a, b, c and the first 2^k
    values of q), two EvaluatePoly at x, and the two values copied to the host; returns the
    tuple (P0, P1, P2, P3, a(x), b(x)).  ``consts``: host arrays by constant name
    (prover_constants); n^-1 is a CPU scalar (the reference dumps scalars only from the CPU)
    and the bases a CPU point base (the reference's MSM reads host point tables)."""
    n, N = 1 << k, 1 << (k + ext)
    gpu = art.gpu_device(device_id)
    track, st = {"Gpu": device_id}, "Gpu"
    table = [
        art.Constant("inv_twiddle", art.scalar_array_typ(n // 2), gpu, consts["inv_twiddle"]),
        art.Constant("fwd_twiddle", art.scalar_array_typ(N // 2), gpu, consts["fwd_twiddle"]),
        art.Constant("n_inv", "Scalar", "CPU", consts["n_inv"]),
        art.Constant("coset_powers", art.scalar_array_typ(n), gpu, consts["coset_powers"]),
        art.Constant("zh_inv", art.scalar_array_typ(1 << ext), gpu, consts["zh_inv"]),
        art.Constant("bases", art.point_base_typ(n), "CPU", consts["bases"]),
    ]
    fused = [{"name": "prover_scale_ninv", "num_vars": 1, "num_mut_vars": 1, "pipelined_meta": None,
              "lib_path": "lib/libprover_scale_ninv.so"},
             {"name": "prover_quotient", "num_vars": 6, "num_mut_vars": 1, "pipelined_meta": None,
              "lib_path": "lib/libprover_quotient.so"}]
    W = -(-254 // window)
    msm_cfg = {"window_size": window, "target_window": W, "cards": [device_id], "debug": False,
               "batch_per_run": 4, "parts": 1, "stage_scalars": 1, "stage_points": 1, "bits": 254}
    f_table = ["NttPrcompute", {"FusedArith": fused[0]}, "NewZero", "DistributePowers",
               {"FusedArith": fused[1]}, {"Msm": msm_cfg}, "EvaluatePoly"]
    F_NTT, F_SCALE, F_ZERO, F_DIST, F_QUOT, F_MSM, F_EVAL = range(7)
    ins, vid, dev_off = [], [0], [0]

    def new():
        vid[0] += 1
        return vid[0] - 1

    def alloc_gpu(typ, nbytes):
        v = new()
        ins.append(_ins({"Allocate": {"device": gpu, "typ": typ, "id": v,
                                      "alloc_method": {"Offset": [dev_off[0], nbytes]}}}))
        dev_off[0] += _al(nbytes)
        return v

    def alloc_cpu(typ):
        v = new()
        ins.append(_ins({"Allocate": {"device": "CPU", "typ": typ, "id": v, "alloc_method": {"Dynamic": 0}}}))
        return v

    def call(f, arg_mut, arg):
        ins.append(_ins({"FuncCall": {"func_id": f, "arg_mut": arg_mut, "arg": arg}}, track, st))

    def transfer(src_dev, dst_dev, s, d):
        ins.append(_ins({"Transfer": {"src_device": src_dev, "dst_device": dst_dev, "stream": stream,
                                      "src_id": s, "dst_id": d}}, "ToGpu" if dst_dev != "CPU" else "FromGpu", st))

    stream = new()
    ins.append(_ins({"Allocate": {"device": gpu, "typ": "Stream", "id": stream, "alloc_method": {"Dynamic": 0}}}))
    inputs = []
    for e in range(5):
        v = new()
        ins.append(_ins({"LoadInput": {"src": e, "dst": v}}))
        inputs.append(v)
    cs = []
    for c in range(len(table)):
        v = new()
        ins.append(_ins({"LoadConstant": {"src": c, "dst": v}}))
        cs.append(v)
    inv_tw, fwd_tw, ninv_c, powers, zh, bases = cs
    A, B, C = (alloc_gpu(art.scalar_array_typ(n), n * 32) for _ in range(3))
    Z, E, Q = (alloc_gpu(art.scalar_array_typ(N), N * 32) for _ in range(3))
    X, NINV, R0, R1 = (alloc_gpu("Scalar", 32) for _ in range(4))
    argbuf = alloc_gpu({"GpuBuffer": [7 * POLYPTR_BYTES, None]}, 7 * POLYPTR_BYTES)
    local = alloc_gpu({"GpuBuffer": [0, None]}, 0)
    msm_buf = alloc_gpu({"GpuBuffer": [0, None]}, 0)
    t0, t1 = (alloc_gpu({"GpuBuffer": [0, None]}, 0) for _ in range(2))
    P = [alloc_cpu("Point") for _ in range(4)]
    r0, r1 = alloc_cpu("Scalar"), alloc_cpu("Scalar")
    for src, dst in zip(inputs, (A, B, C, Z, X)):
        transfer("CPU", gpu, src, dst)
    transfer("CPU", gpu, ninv_c, NINV)
    for poly in (A, B, C):
        call(F_NTT, [poly], [inv_tw, stream])
        call(F_SCALE, [argbuf, local, poly], [stream, NINV])
    call(F_ZERO, [E], [stream])
    e_lo = new()
    ins.append(_ins({"Slice": {"src": E, "dst": e_lo, "start": 0, "end": n}}))
    transfer(gpu, gpu, C, e_lo)
    call(F_DIST, [e_lo], [powers, stream])
    ins.append(_ins({"RemoveRegister": {"id": e_lo}}))
    call(F_NTT, [E], [fwd_tw, stream])
    zw = new()
    ins.append(_ins({"Rotation": {"src": Z, "dst": zw, "shift": -(1 << ext)}}))
    call(F_QUOT, [argbuf, local, Q], [stream, E, E, E, Z, zw, zh])
    q_lo = new()
    ins.append(_ins({"Slice": {"src": Q, "dst": q_lo, "start": 0, "end": n}}))
    call(F_MSM, [msm_buf] + P, [bases, A, B, C, q_lo])
    call(F_EVAL, [t0, R0], [A, X, stream])
    call(F_EVAL, [t1, R1], [B, X, stream])
    transfer(gpu, "CPU", R0, r0)
    transfer(gpu, "CPU", R1, r1)
    ins.append(_ins({"Record": {"stream": stream, "event": 0}}, track, st))
    ins.append(_ins({"Wait": {"slave": "CPU", "stream": None, "event": 0}}, "Cpu"))
    for v in (zw, q_lo):
        ins.append(_ins({"RemoveRegister": {"id": v}}))
    for v in (A, B, C, Z, E, Q, X, NINV, R0, R1, argbuf, local, msm_buf, t0, t1):
        ins.append(_ins({"Deallocate": {"id": v, "alloc_method": "Offset"}}))
    out = new()
    ins.append(_ins({"AssembleTuple": {"vars": P + [r0, r1], "dst": out}}))
    ins.append(_ins({"Return": out}))
    chunk = {"instructions": ins, "f_table": [f_table, None], "event_table": [[{"GpuEvent": device_id}], None],
             "n_variables": vid[0], "n_threads": 1, "lbss": [k + ext + 5]}
    memory_info = {"memory_limit": dev_off[0], "smithereen_space": 0}
    zero = {"gpu": [0], "cpu": 0, "stack": 0, "disk": 0}
    statistics = {"transfer_sizes": {"gpu": [dict(zero)], "cpu": dict(zero), "stack": dict(zero),
                                     "disk": dict(zero)}}
    return memory_info, chunk, statistics, table


def dump_artifact(directory: str, memory_info: dict, chunk: dict, statistics: dict, table: list) -> str:
    """Writes version_<size>.json (artifect.rs:72-77) and the constant table; returns the chunk path."""
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, f"version_{memory_info['memory_limit']}B.json")
    with open(path, "w") as f:
        json.dump([memory_info, chunk, statistics], f, indent=1)
    art.dump_constant_table(directory, table)
    return path
