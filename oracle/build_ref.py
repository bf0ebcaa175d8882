"""Builds the reference's own code into oracle/_ref/ (test infrastructure only), from the sources
where they lie in the reference checkout, with nvcc for sm_100a (the reference's build system,
xmake / Makefile.msm, is not used):

  libref.so                oracle/ref_driver.cu against the reference's host arithmetic headers
  libref_ntt.so            core/src/ntt/src/ntt.cu (ssip_ntt, ssip_precompute, recompute_ntt,
                           gen_pq_omegas, distribute_powers) with NTT_FIELD = bn254_fr::Element,
                           the definition the reference's build uses for BN254
  libref_msm_<s>_<t>.so    core/src/msm/src/msm.cu with MSM_WINDOW_SIZE = s and
                           MSM_TARGET_WINDOWS = t (the per-configuration library the reference
                           builds, Makefile.msm), MSM_BITS 254, curve bn254, debug off
  libref_poly.so           core/src/poly/src/*.cu (poly_basic, poly_eval, kate_division,
                           scan_mul, batched_invert, permute) with POLY_FIELD = bn254_fr::Element;
                           each source compiled to an object in parallel, then linked

Skipped when the checkout is absent; the built libraries travel with the repository snapshot.
The GPU libraries serve the parity tests that run the reference's kernels next to this
repository's on the same inputs.

Usage: python oracle/build_ref.py [reference_root]
The checkout is the argument, else $ZKPOLY_REFERENCE_DIR, else a directory named `reference`
beside this repository's own directory; when none exists, nothing is built.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ZKPOLY_REFERENCE_DIR")
       or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
OUT_DIR = os.path.join(HERE, "_ref")
NVCC = "/usr/local/cuda/bin/nvcc"
BASE = [NVCC, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
        "-diag-suppress", "550,177"]
# (window, target windows): 16/16 is the default library name the reference's runtime loads
# (one point table); 17/8 is its cost model's choice for 2^22 points (two tables)
MSM_CONFIGS = [(16, 16), (17, 8)]


def jobs():
    out = []
    driver = os.path.join(HERE, "ref_driver.cu")
    out.append((os.path.join(OUT_DIR, "libref.so"), [driver],
                BASE[:1] + ["-O2"] + BASE[2:] + [
                    "-I" + os.path.join(REF, "core/src/common/curve/src"),
                    "-I" + os.path.join(REF, "core/src/ntt/src"),
                    "-DNTT_FIELD=bn254_fr::Element", driver]))
    ntt_src = os.path.join(REF, "core/src/ntt/src/ntt.cu")
    out.append((os.path.join(OUT_DIR, "libref_ntt.so"), [ntt_src],
                BASE + ["-DNTT_FIELD=bn254_fr::Element", ntt_src]))
    msm_src = os.path.join(REF, "core/src/msm/src/msm.cu")
    for s, t in MSM_CONFIGS:
        out.append((os.path.join(OUT_DIR, f"libref_msm_{s}_{t}.so"), [msm_src],
                    BASE + ["-I" + os.path.join(REF, "core/src/msm"), "-DMSM_BITS=254", "-DMSM_CURVE=bn254",
                            f"-DMSM_WINDOW_SIZE={s}", f"-DMSM_TARGET_WINDOWS={t}", "-DMSM_DEBUG=false",
                            msm_src]))
    return out


POLY_SOURCES = ["poly_basic", "poly_eval", "kate_division", "scan_mul", "batched_invert", "permute"]


def poly_objects():
    """(object, source, command) for each reference poly source."""
    src_dir = os.path.join(REF, "core/src/poly/src")
    obj_dir = os.path.join(OUT_DIR, "obj")
    out = []
    for name in POLY_SOURCES:
        src = os.path.join(src_dir, name + ".cu")
        obj = os.path.join(obj_dir, name + ".o")
        cmd = [NVCC, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-c", "-gencode", "arch=compute_100a,code=sm_100a",
               "--extended-lambda", "-diag-suppress", "550,177", "-DPOLY_FIELD=bn254_fr::Element", src]
        out.append((obj, src, cmd))
    return out


def build_poly(failed):
    target = os.path.join(OUT_DIR, "libref_poly.so")
    objs = poly_objects()
    srcs = [src for _, src, _ in objs]
    if os.path.exists(target) and all(os.path.getmtime(target) > os.path.getmtime(s) for s in srcs):
        return
    os.makedirs(os.path.join(OUT_DIR, "obj"), exist_ok=True)
    procs = [(obj, subprocess.Popen(cmd + ["-o", obj], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
             for obj, _, cmd in objs]
    ok = True
    for obj, proc in procs:
        log, _ = proc.communicate()
        if proc.returncode != 0:
            failed.append(f"{obj}:\n{log}")
            ok = False
    if not ok:
        return
    link = subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", target + ".tmp",
                           *[obj for obj, _, _ in objs]], capture_output=True, text=True)
    if link.returncode != 0:
        failed.append(f"{target}:\n{link.stderr}")
        return
    os.replace(target + ".tmp", target)
    print(target)


def main():
    if not os.path.isdir(REF):
        print("reference checkout absent; oracle/_ref not built")
        return
    os.makedirs(OUT_DIR, exist_ok=True)
    running = []
    for target, srcs, cmd in jobs():
        if os.path.exists(target) and all(os.path.getmtime(target) > os.path.getmtime(s) for s in srcs):
            continue
        running.append((target, subprocess.Popen(cmd + ["-o", target + ".tmp"], stdout=subprocess.PIPE,
                                                 stderr=subprocess.STDOUT, text=True)))
    failed = []
    build_poly(failed)
    for target, proc in running:
        log, _ = proc.communicate()
        if proc.returncode != 0:
            failed.append(f"{target}:\n{log}")
        else:
            os.replace(target + ".tmp", target)
            print(target)
    if failed:
        raise RuntimeError("reference build failed:\n" + "\n".join(failed))


if __name__ == "__main__":
    main()
