"""Compiled-program artifacts on the CPU: the reference's serde forms are read, and what the
served data plane does not cover is refused before any device work."""
import copy
import json
import os

import pytest

from conftest import GOLDEN

ART = os.path.join(GOLDEN, "prover_k10")


def test_golden_artifact_reads(zk):
    p = zk.program
    mem, chunk, stats = p.read_chunk(ART)
    assert mem["memory_limit"] > 0 and set(stats) == {"transfer_sizes"}
    f_table = p.heap_items(chunk["f_table"])
    kinds = [p.kernel_kind(kt)[0] for kt in f_table]
    assert kinds == ["NttPrcompute", "FusedArith", "NewZero", "DistributePowers", "FusedArith", "Msm",
                     "EvaluatePoly"]
    assert p.heap_items(chunk["event_table"]) == [{"GpuEvent": 0}]
    nodes = [p.node_of(i)[0] for i in chunk["instructions"]]
    for kind in ("Allocate", "LoadInput", "LoadConstant", "Transfer", "FuncCall", "Slice", "Rotation", "Record",
                 "Wait", "AssembleTuple", "Return", "Deallocate", "RemoveRegister"):
        assert kind in nodes, kind
    assert nodes[-1] == "Return"
    # every id is a bare integer (newtype structs), and every use follows a definition
    defined = set()
    for ins in chunk["instructions"]:
        kind, body = p.node_of(ins)
        if kind in ("Allocate",):
            defined.add(body["id"])
        elif kind in ("LoadInput", "LoadConstant", "Slice", "Rotation", "AssembleTuple"):
            defined.add(body["dst"])
        elif kind == "FuncCall":
            assert set(body["arg"]) | set(body["arg_mut"]) <= defined
    # the constant table reads back with the loader
    header = zk.artifact.read_manifest(ART)
    assert [e["name"] for e in header["entries"]] == ["inv_twiddle", "fwd_twiddle", "n_inv", "coset_powers",
                                                      "zh_inv", "bases"]


def test_msm_precompute_count(zk):
    """MsmConfig::get_precompute (common/src/msm_config.rs:17-25)."""
    f = zk.program.msm_precompute_tables
    assert f({"bits": 254, "window_size": 16, "target_window": 16}) == 1
    assert f({"bits": 254, "window_size": 17, "target_window": 8}) == 2
    assert f({"bits": 254, "window_size": 20, "target_window": 1}) == 13


def _lower(zk, chunk):
    p = zk.program
    low = p.Lowering(chunk, [], p.prover_input_types(10), {})
    low.run()
    return low


@pytest.mark.parametrize("bad,match", [
    ({"Fork": {"new_thread": 1, "instructions": []}}, "multi-threaded"),
    ({"Allocate": {"device": "Disk", "typ": "Scalar", "id": 99, "alloc_method": {"Dynamic": 0}}}, "disk"),
    ({"Allocate": {"device": {"GPU": {"device_id": 0}}, "typ": "Scalar", "id": 99,
                   "alloc_method": {"Paged": {"va_size": 64, "pa": [0]}}}}, "paged"),
    ({"Allocate": {"device": "CPU", "typ": "Transcript", "id": 99, "alloc_method": {"Dynamic": 0}}},
     "not part of the served"),
    ({"Blind": {"dst": 1, "start": 0, "end": 4}}, "not part of the served"),
    ({"Rotation": {"src": 12345, "dst": 99, "shift": 1}}, "undefined"),
])
def test_unsupported_instructions_refused(zk, bad, match):
    _, chunk, _ = zk.program.read_chunk(ART)
    chunk = copy.deepcopy(chunk)
    chunk["instructions"].insert(1, {"node": bad, "track": "MemoryManagement", "stream": None})
    with pytest.raises(ValueError, match=match):
        _lower(zk, chunk)


def test_unsupported_kernel_refused(zk):
    _, chunk, _ = zk.program.read_chunk(ART)
    chunk = copy.deepcopy(chunk)
    chunk["f_table"][0].append("HashTranscript")
    chunk["instructions"].insert(1, {"node": {"FuncCall": {"func_id": len(chunk["f_table"][0]) - 1,
                                                           "arg_mut": [], "arg": []}},
                                     "track": "Cpu", "stream": None})
    with pytest.raises(ValueError, match="HashTranscript"):
        _lower(zk, chunk)


def test_malformed_version_file(zk, tmp_path):
    (tmp_path / "version_1B.json").write_text(json.dumps({"not": "a triple"}))
    with pytest.raises(ValueError, match="triple"):
        zk.program.read_chunk(str(tmp_path))
    (tmp_path / "version_2B.json").write_text("[]")
    with pytest.raises(ValueError, match="one version"):
        zk.program.read_chunk(str(tmp_path))
