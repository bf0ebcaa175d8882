"""Build recipe for the CUDA libraries (sm_100a), compiled in-tree into lib/.

Each reference library name gets its own shared object so a maintainer can point the
reference's loader (common/src/load_dynamic.rs:44-64, $ZKPOLY_COMPILER_PROJECT_ROOT/lib/)
at this directory: libntt.so, libpoly.so, libmsm.so, plus libzkp_runtime.so for the batched
and served forms.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-shared", "--expt-relaxed-constexpr"]

# library -> (main source, extra link flags)
LIBS = {
    "libntt.so": ("ntt.cu", []),
    "libmsm.so": ("msm.cu", ["-ldl"]),
    "libpoly.so": ("poly.cu", []),
    "libzkp_gen.so": ("gen.cu", []),
    "libzkp_pipeline.so": ("pipeline.cu", []),
    # the served form links the kernel libraries above and finds them next to itself
    "libzkp_runtime.so": ("serve.cu", ["-L" + LIB, "-lntt", "-lmsm", "-lpoly", "-lzkp_gen", "-ldl", "-lpthread",
                                       "-Xlinker", "-rpath=$ORIGIN"]),
}


def _deps(src: str):
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".cu"))] + \
        [os.path.join(HERE, "..", "include", f) for f in os.listdir(os.path.join(HERE, "..", "include"))]


def _stale(target: str, src: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in _deps(src))


def build_one(name: str, force: bool = False, verbose: bool = False) -> str:
    src, extra = LIBS[name]
    target = os.path.join(LIB, name)
    if not force and not _stale(target, src):
        return target
    os.makedirs(LIB, exist_ok=True)
    cmd = [NVCC, *ARCH, *FLAGS, "-o", target + ".tmp", os.path.join(CSRC, src), *extra]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{res.stderr}")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(target + ".tmp", target)
    return target


def build_all(force: bool = False, verbose: bool = False):
    out = [build_one(n, force, verbose) for n in LIBS]
    # fused kernels the hot path uses, generated from their graphs (fused.py)
    sys.path.insert(0, os.path.dirname(HERE))
    import importlib
    fused = importlib.import_module(os.path.basename(HERE) + ".fused")
    out += fused.build_path_kernels()
    return out


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv, verbose="-v" in sys.argv):
        print(p)
