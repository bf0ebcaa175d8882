"""Builds oracle/_ref/libref.so (test infrastructure): oracle/ref_driver.cu compiled against the
reference's own headers where they lie under the reference checkout (host code only, nvcc as
the C++ compiler; the reference's build system is not used).  Skipped when the checkout is
absent; the built library travels with the repository snapshot.

Usage: python oracle/build_ref.py [reference_root]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
OUT = os.path.join(HERE, "_ref", "libref.so")


def main():
    if not os.path.isdir(REF):
        print("reference checkout absent; oracle/_ref not built")
        return
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    src = os.path.join(HERE, "ref_driver.cu")
    if os.path.exists(OUT) and os.path.getmtime(OUT) > os.path.getmtime(src):
        return
    cmd = ["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(REF, "core/src/common/curve/src"),
           "-I" + os.path.join(REF, "core/src/ntt/src"),
           "-DNTT_FIELD=bn254_fr::Element",
           "-o", OUT, src]
    subprocess.run(cmd, check=True)
    print(OUT)


if __name__ == "__main__":
    main()
