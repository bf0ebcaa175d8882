"""The constant table of a compiled program artifact, loaded into HBM.

A program compiled by the reference is dumped as a directory (compiler/src/driver/artifect.rs:65-86)
holding the instruction chunks of each memory version plus two files for its constants:

* ``constants-manifest.json`` - serde_json of ``Header {entries, data_size}``
  (runtime/src/args/serialization.rs:159-173), one ``Entry {position, name, typ, device}`` per
  constant-table slot in slot order.  ``position`` is ``[offset, size]`` into constants.bin, or
  ``null`` for a constant without a binary form (a transcript, a tuple, a stream, ...);
  offsets are the running sum of the sizes before it (:175-206).
* ``constants.bin`` - the raw bytes of every entry that has a position, back to back
  (:208-220; each value written by :17-91).  A polynomial is ``len`` Fr elements of 32 bytes,
  a scalar one element, a point 64 bytes (affine x || y, Fq), a point base ``len`` points.  Both
  fields are in Montgomery form with little-endian limbs, the layout every kernel of this
  package reads, so the bytes go to the device unchanged.

The JSON forms are serde's default external tagging of ``Typ<()>`` (common/src/typ.rs:120-130,
:204) and ``DeviceType`` (common/src/devices.rs:3-8)::

    {"ScalarArray": {"len": 1024, "meta": null}}   {"PointBase": {"len": 1024}}
    "Scalar"  "Point"  "Transcript"  "Tuple"  "Stream"
    {"Any": [[id0, id1], size]}  {"GpuBuffer": [size, null]}
    "CPU"  {"GPU": {"device_id": 0}}  "Disk"

Loading follows ``Header::load_constant_table`` (serialization.rs:222-271): each entry with a
position is read from its offset (the type fixes how many bytes; the recorded size is not
consulted) and placed on the entry's device; an entry without one must already be present in
the caller's table at the same slot, with the same name and type.  GPU device ids go through a
mapping, as the runtime's ``GpuMapping`` does (compiler/src/driver/artifect.rs:96).  Where the
reference panics (a missing or mismatched slot, a type without a binary form that has a
position) this module raises ``ValueError``; a short constants.bin raises ``EOFError`` (the reference's
``read_exact`` error).  ``Disk`` constants are loaded into host memory: this package keeps no
disk pool.

The instruction chunks of the artifact are the reference runtime's interpreter input and are
not read here; the loaded constants feed this package's kernels directly (``ScalarArray``
polynomials, ``msm.ResidentBases`` / ``serving.Server`` point bases).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass
from typing import Callable

import numpy as np
import torch

from .scalar import ScalarArray

MANIFEST = "constants-manifest.json"
DATA = "constants.bin"
FR_BYTES = 32      # halo2curves bn256::Fr, [u64; 4] Montgomery
POINT_BYTES = 64   # halo2curves bn256::G1Affine, x || y in Montgomery Fq; identity = (0, 0)

_UNIT_TYPS = ("Scalar", "Point", "Transcript", "Tuple", "Stream")


@dataclass
class Constant:
    """One slot of a program's constant table (runtime/src/args.rs:290).

    ``typ`` and ``device`` keep their manifest JSON forms.  ``value`` is a ``ScalarArray`` for a
    polynomial, an int32 tensor for the other binary types ((8,) scalar, (16,) point, (len, 16)
    point base), or whatever the caller put in its table for a type without a binary form."""
    name: str | None
    typ: object
    device: object
    value: object = None


# ---- type and device forms

def typ_kind(typ) -> str:
    if isinstance(typ, str):
        if typ not in _UNIT_TYPS:
            raise ValueError(f"unknown Typ {typ!r}")
        return typ
    if isinstance(typ, dict) and len(typ) == 1:
        kind = next(iter(typ))
        if kind in ("ScalarArray", "PointBase", "Any", "GpuBuffer"):
            return kind
    raise ValueError(f"unknown Typ {typ!r}")


def scalar_array_typ(length: int) -> dict:
    return {"ScalarArray": {"len": int(length), "meta": None}}


def point_base_typ(length: int) -> dict:
    return {"PointBase": {"len": int(length)}}


def gpu_device(device_id: int = 0) -> dict:
    return {"GPU": {"device_id": int(device_id)}}


def binary_size(typ) -> int | None:
    """Bytes a constant of this type occupies in constants.bin, or None when the type has no
    binary form (``Variable::dump_size``, serialization.rs:93-101)."""
    kind = typ_kind(typ)
    if kind == "ScalarArray":
        return int(typ["ScalarArray"]["len"]) * FR_BYTES
    if kind == "PointBase":
        return int(typ["PointBase"]["len"]) * POINT_BYTES
    if kind == "Scalar":
        return FR_BYTES
    if kind == "Point":
        return POINT_BYTES
    return None


def torch_device(device, gpu_mapping: Callable[[int], int] | None = None) -> torch.device:
    if device in ("CPU", "Disk"):
        return torch.device("cpu")
    if isinstance(device, dict) and set(device) == {"GPU"}:
        dev_id = int(device["GPU"]["device_id"])
        return torch.device("cuda", gpu_mapping(dev_id) if gpu_mapping else dev_id)
    raise ValueError(f"unknown DeviceType {device!r}")


# ---- values <-> bytes

def _shape_of(typ) -> tuple[int, ...]:
    kind = typ_kind(typ)
    if kind == "ScalarArray":
        return (int(typ["ScalarArray"]["len"]), 8)
    if kind == "PointBase":
        return (int(typ["PointBase"]["len"]), 16)
    return (8,) if kind == "Scalar" else (16,)


def _value_tensor(c: Constant) -> torch.Tensor:
    """The int32 words of a binary constant, checked against its type (``dump_binary``,
    serialization.rs:17-91: a polynomial must be unrotated and unsliced)."""
    v = c.value
    if isinstance(v, ScalarArray):
        if v.slice_info is not None or v.get_rotation() != 0:
            raise ValueError(f"constant {c.name!r}: polynomial must be unrotated and unsliced")
        v = v.values[: v.len]
    if isinstance(v, np.ndarray):
        v = torch.from_numpy(np.ascontiguousarray(v).view(np.int32))
    if not isinstance(v, torch.Tensor):
        raise ValueError(f"constant {c.name!r}: no value to write for {c.typ!r}")
    words = v.contiguous().view(torch.int32)
    shape = _shape_of(c.typ)
    if words.numel() != int(np.prod(shape)):
        raise ValueError(f"constant {c.name!r}: value has {words.numel() * 4} bytes, "
                         f"{c.typ!r} needs {binary_size(c.typ)}")
    return words.reshape(shape)


def _wrap(typ, words: torch.Tensor):
    return ScalarArray(words) if typ_kind(typ) == "ScalarArray" else words


# ---- load / dump

def read_manifest(directory: str) -> dict:
    with open(os.path.join(directory, MANIFEST)) as f:
        header = json.load(f)
    if not isinstance(header, dict) or "entries" not in header or "data_size" not in header:
        raise ValueError(f"{MANIFEST}: not a constant-table header")
    for e in header["entries"]:
        typ_kind(e["typ"])
        pos = e.get("position")
        if pos is not None and (len(pos) != 2 or pos[0] < 0 or pos[1] < 0):
            raise ValueError(f"{MANIFEST}: bad position {pos!r}")
    return header


def load_constant_table(directory: str, table: list[Constant] | None = None,
                        gpu_mapping: Callable[[int], int] | None = None) -> list[Constant]:
    """Read an artifact's constants into ``table`` (created when None) and return it.

    Binary constants land on their manifest device: GPU constants are read from the file into
    pinned host memory and copied to HBM, and the call returns once every copy has finished."""
    header = read_manifest(directory)
    table = [] if table is None else table
    touched: set[torch.device] = set()
    with open(os.path.join(directory, DATA), "rb") as f:
        for i, e in enumerate(header["entries"]):
            name, typ, device = e.get("name"), e["typ"], e["device"]
            if e.get("position") is None:
                if len(table) <= i:
                    raise ValueError(f"constant slot {i} ({name!r}) has no data and the table has no entry for it")
                have = table[i]
                if have.name != name:
                    raise ValueError(f"constant name mismatch at index {i}: expect {name!r}, got {have.name!r}")
                if have.typ != typ:
                    raise ValueError(f"constant type mismatch at index {i}: expect {typ!r}, got {have.typ!r}")
                continue
            size = binary_size(typ)
            if size is None:
                raise ValueError(f"constant slot {i} ({name!r}): type {typ!r} has no binary form")
            dev = torch_device(device, gpu_mapping)
            host = torch.empty(size, dtype=torch.uint8, pin_memory=dev.type == "cuda")
            f.seek(int(e["position"][0]))
            got = f.readinto(memoryview(host.numpy())) if size else 0
            if got != size:
                raise EOFError(f"{DATA}: slot {i} ({name!r}) needs {size} bytes at offset "
                               f"{e['position'][0]}, file has {got}")
            words = host.view(torch.int32).reshape(_shape_of(typ))
            if dev.type == "cuda":
                words = words.to(dev, non_blocking=True)
                touched.add(dev)
            while len(table) <= i:
                table.append(Constant(name, "Tuple", "CPU", None))  # placeholder, as the reference does
            table[i] = Constant(name, typ, device, _wrap(typ, words))
    for dev in touched:
        torch.cuda.synchronize(dev)
    return table


def dump_constant_table(directory: str, table: list[Constant]) -> dict:
    """Write ``table`` as constants-manifest.json + constants.bin (``Header::build`` and
    ``dump_entries_data``, serialization.rs:175-220) and return the header."""
    for c in table:
        # the reference writes a scalar only from host memory (dump_binary panics with "scalar
        # must be on CPU", serialization.rs:47-50), so no artifact it reads back holds another
        if typ_kind(c.typ) == "Scalar" and c.device != "CPU":
            raise ValueError(f"constant {c.name!r}: scalar must be on CPU, not {c.device!r}")
    os.makedirs(directory, exist_ok=True)
    entries, offset = [], 0
    for c in table:
        size = binary_size(c.typ)
        entries.append({"position": None if size is None else [offset, size], "name": c.name,
                        "typ": c.typ, "device": c.device})
        offset += size or 0
    header = {"entries": entries, "data_size": offset}
    with open(os.path.join(directory, DATA), "wb") as f:
        for c in table:
            if binary_size(c.typ) is not None:
                f.write(_value_tensor(c).cpu().numpy().tobytes())
    with open(os.path.join(directory, MANIFEST), "w") as f:
        json.dump(header, f, indent=2)
    return header


# ---- handing constants to the kernels

def by_name(table: list[Constant], name: str) -> Constant:
    for c in table:
        if c.name == name:
            return c
    raise KeyError(name)


def resident_bases(c: Constant, window: int = 0, n_tables: int = 1):
    """A loaded point-base constant as ``msm.ResidentBases`` (precomputed tables built in HBM
    when ``n_tables`` > 1), ready for device-pointer MSMs or ``serving.Server``."""
    from . import msm
    if typ_kind(c.typ) != "PointBase":
        raise ValueError(f"constant {c.name!r} is {c.typ!r}, not a PointBase")
    if not isinstance(c.value, torch.Tensor) or c.value.device.type != "cuda":
        raise ValueError(f"constant {c.name!r} is not resident on a GPU")
    return msm.ResidentBases(c.value, window=window, n_tables=n_tables, device=c.value.device)
