"""Constant table of a program artifact (constants-manifest.json + constants.bin): parsing of the
reference's serde forms, round trips, the reference loader's error cases, and (on a GPU) the
loaded constants driving the NTT and MSM kernels, bit-exact against the oracle.

No artifact written by the reference exists in its tree and its Rust toolchain is absent here,
so the manifest below is written out by hand from the serde derives it is serialised with
(runtime/src/args/serialization.rs:159-173, common/src/typ.rs:120-130, common/src/devices.rs:3-8;
serde_json::to_writer_pretty, compiler/src/driver/artifect.rs:80).
"""
import os

import numpy as np
import pytest
import torch

# Five slots as a compiled program dumps them: a transcript (no binary form), a polynomial of 4
# elements on GPU 0, a scalar on the CPU, a point and a base of 2 points on GPU 0.
MANIFEST = """{
  "entries": [
    {
      "position": null,
      "name": "transcript",
      "typ": "Transcript",
      "device": "CPU"
    },
    {
      "position": [
        0,
        128
      ],
      "name": "fixed_0",
      "typ": {
        "ScalarArray": {
          "len": 4,
          "meta": null
        }
      },
      "device": {
        "GPU": {
          "device_id": 0
        }
      }
    },
    {
      "position": [
        128,
        32
      ],
      "name": null,
      "typ": "Scalar",
      "device": "CPU"
    },
    {
      "position": [
        160,
        64
      ],
      "name": "g",
      "typ": "Point",
      "device": "Disk"
    },
    {
      "position": [
        224,
        128
      ],
      "name": "bases",
      "typ": {
        "PointBase": {
          "len": 2
        }
      },
      "device": {
        "GPU": {
          "device_id": 0
        }
      }
    }
  ],
  "data_size": 352
}"""


def _fixture_bytes(orc):
    poly = orc.gen_fr(11, 4)
    scalar = orc.gen_fr(12, 1)
    g = orc.g1_generator().reshape(1, 8)
    bases = orc.gen_points(13, 2)
    return poly, scalar, g, bases, b"".join(a.tobytes() for a in (poly, scalar, g, bases))


def _write(tmp_path, manifest, data):
    (tmp_path / "constants-manifest.json").write_text(manifest)
    (tmp_path / "constants.bin").write_bytes(data)
    return str(tmp_path)


def _words(t):
    return np.ascontiguousarray(t.cpu().numpy()).view(np.uint64)


_GPU0 = '{\n        "GPU": {\n          "device_id": 0\n        }\n      }'
HOST_MANIFEST = MANIFEST.replace(_GPU0, '"CPU"')  # the same slots, all in host memory


def test_reference_manifest_parses(zk, orc, tmp_path):
    a = zk.artifact
    poly, scalar, g, bases, data = _fixture_bytes(orc)
    d = _write(tmp_path, MANIFEST, data)
    header = a.read_manifest(d)
    assert header["data_size"] == len(data) == 352
    assert [a.binary_size(e["typ"]) for e in header["entries"]] == [None, 128, 32, 64, 128]
    assert [e["position"] for e in header["entries"]][1:] == [[0, 128], [128, 32], [160, 64], [224, 128]]
    assert a.torch_device(header["entries"][1]["device"]).type == "cuda"
    assert a.torch_device(header["entries"][1]["device"], lambda i: i + 3) == torch.device("cuda", 3)
    assert a.torch_device("Disk") == torch.device("cpu")
    # a serde form of every Typ variant is recognised
    for typ in ("Scalar", "Point", "Transcript", "Tuple", "Stream", {"Any": [[1, 2], 64]},
                {"GpuBuffer": [4096, None]}, a.scalar_array_typ(8), a.point_base_typ(8)):
        a.typ_kind(typ)
    with pytest.raises(ValueError):
        a.typ_kind({"Polynomial": {"len": 4}})


def test_host_constants_load(zk, orc, tmp_path):
    """CPU and Disk slots load to host memory with the bytes of constants.bin, unchanged."""
    a = zk.artifact
    poly, scalar, g, bases, data = _fixture_bytes(orc)
    d = _write(tmp_path, HOST_MANIFEST, data)
    table = [a.Constant("transcript", "Transcript", "CPU", object())]
    out = a.load_constant_table(d, table)
    assert out is table and len(out) == 5
    assert isinstance(out[1].value, zk.ScalarArray) and out[1].value.len == 4
    assert np.array_equal(_words(out[1].value.values).reshape(4, 4), poly)
    assert np.array_equal(_words(out[2].value), scalar[0])
    assert np.array_equal(_words(out[3].value), g[0])
    assert orc.g1_on_curve(_words(out[3].value))
    assert np.array_equal(_words(out[4].value).reshape(2, 8), bases)
    assert a.by_name(out, "bases") is out[4]
    assert out[2].name is None and out[3].device == "Disk"


def test_round_trip(zk, orc, tmp_path):
    a = zk.artifact
    poly = orc.gen_fr(21, 33)
    pts = orc.gen_points(22, 5)
    table = [
        a.Constant("p", a.scalar_array_typ(33), "CPU", zk.ScalarArray.from_numpy(poly, device="cpu")),
        a.Constant("stream", "Stream", "CPU", "opaque"),
        a.Constant(None, "Scalar", "CPU", orc.gen_fr(23, 1)[0]),
        a.Constant("pt", "Point", "Disk", pts[0]),
        a.Constant("bases", a.point_base_typ(5), "CPU", pts),
        a.Constant("empty", a.scalar_array_typ(0), "CPU", np.zeros((0, 4), dtype=np.uint64)),
    ]
    header = a.dump_constant_table(str(tmp_path), table)
    assert header["data_size"] == 33 * 32 + 32 + 64 + 5 * 64
    assert header["entries"][1]["position"] is None
    assert header["entries"][5]["position"] == [header["data_size"], 0]
    assert os.path.getsize(tmp_path / "constants.bin") == header["data_size"]
    back = a.load_constant_table(str(tmp_path), [a.Constant("p", "Tuple", "CPU"),
                                                 a.Constant("stream", "Stream", "CPU", "opaque")])
    assert np.array_equal(_words(back[0].value.values).reshape(33, 4), poly)
    assert back[1].value == "opaque"
    assert np.array_equal(_words(back[2].value), table[2].value)
    assert np.array_equal(_words(back[3].value), pts[0])
    assert np.array_equal(_words(back[4].value).reshape(5, 8), pts)
    assert back[5].value.len == 0
    # a second dump of what was loaded writes the same files
    a.dump_constant_table(str(tmp_path / "again"), back)
    assert (tmp_path / "again" / "constants.bin").read_bytes() == (tmp_path / "constants.bin").read_bytes()


def test_loader_errors(zk, orc, tmp_path):
    """The reference loader's panics (serialization.rs:154, :252-268) and read_exact error."""
    a = zk.artifact
    _, _, _, _, data = _fixture_bytes(orc)
    host = HOST_MANIFEST
    d = _write(tmp_path, host, data)
    with pytest.raises(ValueError, match="no data"):            # slot 0 has no data and no entry
        a.load_constant_table(d)
    with pytest.raises(ValueError, match="name mismatch"):
        a.load_constant_table(d, [a.Constant("other", "Transcript", "CPU")])
    with pytest.raises(ValueError, match="type mismatch"):
        a.load_constant_table(d, [a.Constant("transcript", "Tuple", "CPU")])
    (tmp_path / "short").mkdir()
    d2 = _write(tmp_path / "short", host, data[:-1])
    with pytest.raises(EOFError):
        a.load_constant_table(d2, [a.Constant("transcript", "Transcript", "CPU")])
    bad = host.replace('"position": null,\n      "name": "transcript"', '"position": [0, 0],\n      "name": "transcript"')
    (tmp_path / "bad").mkdir()
    d3 = _write(tmp_path / "bad", bad, data)
    with pytest.raises(ValueError, match="no binary form"):
        a.load_constant_table(d3)
    rotated = zk.ScalarArray.from_numpy(orc.gen_fr(1, 8), device="cpu")
    rotated.rotate(3)
    with pytest.raises(ValueError, match="unrotated"):
        a.dump_constant_table(str(tmp_path / "rot"), [a.Constant("r", a.scalar_array_typ(8), "CPU", rotated)])
    with pytest.raises(ValueError, match="needs"):
        a.dump_constant_table(str(tmp_path / "len"), [a.Constant("r", a.scalar_array_typ(9), "CPU",
                                                                 orc.gen_fr(1, 8))])
    # a scalar is written only from host memory (the reference panics "scalar must be on CPU"),
    # checked before any file is written
    for dev in (a.gpu_device(0), "Disk"):
        with pytest.raises(ValueError, match="scalar must be on CPU"):
            a.dump_constant_table(str(tmp_path / "sc"), [a.Constant("s", "Scalar", dev, orc.gen_fr(1, 1)[0])])
        assert not (tmp_path / "sc").exists()


@pytest.mark.gpu
def test_gpu_constants_drive_kernels(zk, orc, tmp_path):
    """Polynomial and point-base constants loaded straight into HBM: an NTT of the loaded
    polynomial and an MSM over the loaded bases (with precomputed tables) match the oracle."""
    a = zk.artifact
    log_n, n = 12, 1 << 12
    poly = orc.gen_fr(31, n)
    scalars = orc.gen_fr(32, n)
    pts = orc.gen_points(33, n)
    gpu = a.gpu_device(3)  # a device id of the machine that wrote the artifact, mapped to GPU 0 below
    a.dump_constant_table(str(tmp_path), [
        a.Constant("coeffs", a.scalar_array_typ(n), gpu, poly),
        a.Constant("scalars", a.scalar_array_typ(n), gpu, scalars),
        a.Constant("srs", a.point_base_typ(n), gpu, pts),
    ])
    table = a.load_constant_table(str(tmp_path), gpu_mapping=lambda i: i - 3)
    assert all((c.value.values if isinstance(c.value, zk.ScalarArray) else c.value).device == torch.device("cuda", 0)
               for c in table)
    x = table[0].value
    zk.ntt.ntt(x)
    assert np.array_equal(x.numpy_u64(), orc.ntt(poly, log_n))
    for n_tables in (1, 4):
        bases = a.resident_bases(a.by_name(table, "srs"), window=12, n_tables=n_tables)
        res = torch.zeros(16, dtype=torch.int32, device="cuda")
        bases.msm(a.by_name(table, "scalars").value.values, res, bases.workspace())
        assert np.array_equal(_words(res), orc.best_multiexp(scalars, pts)), n_tables
    with pytest.raises(ValueError):
        a.resident_bases(table[0])


@pytest.mark.gpu
def test_gpu_constants_feed_the_server(zk, tmp_path):
    """A served prover built on point bases loaded from an artifact gives the same results as one
    built on the same bases generated in HBM."""
    a = zk.artifact
    pts = zk.gen.points(2, 1 << 12)
    a.dump_constant_table(str(tmp_path), [a.Constant("srs", a.point_base_typ(1 << 12), a.gpu_device(0), pts)])
    loaded = a.by_name(a.load_constant_table(str(tmp_path)), "srs").value
    assert torch.equal(loaded, pts)
    results = []
    for bases in (pts, loaded):
        srv = zk.serving.Server(bases, hbm_bytes=2 << 30, max_inflight=2, ext_log=2, min_k=10, max_k=12)
        try:
            got = []
            for k, seed in ((10, 1), (12, 2)):
                r = srv.wait(srv.submit(k, seed))
                assert r.status == 0
                got.append(zk.serving.result_words(r))
            results.append(got)
        finally:
            srv.close()
    for x, y in zip(*results):
        assert np.array_equal(x, y)
