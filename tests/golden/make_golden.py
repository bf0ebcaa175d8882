"""Extract the reference's known-answer vectors for this path into reference_vectors.json.

Reads, as text, the BN254 test files of the reference:
  core/src/common/mont/tests/main.cu   (Fr: instance1 :238-253, instance2 :369-382,
                                        instance3 :527-535, to/from Montgomery :502-503)
  core/src/common/curve/tests/bn254.cu (G1: p1, p2, p1+p2, p1+100*p2, 128*p1 :174-203)
  core/src/common/mont/src/bn254_fr.cuh, bn254_fq.cuh (m, 2m, m-2, R mod m, R^2 mod m, m')
and writes each constant as a little-endian list of u32 limbs (BIG_INTEGER_CHUNKSk lists the
most significant chunk first; the reference macro reverses it, field.cuh:10-16).

Usage: python tests/golden/make_golden.py [reference_root]
"""
import json
import os
import re
import sys

ROOT = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")

DECL = re.compile(
    r"const\s+u32\s+(\w+)\s*\[[^\]]*\]\s*=\s*BIG_INTEGER_CHUNKS(\d+)\(([^)]*)\)", re.S)
NS = re.compile(r"namespace\s+(\w+)\s*\{")


def parse(path):
    text = open(path).read()
    # map each declaration to the innermost namespace that opens before it
    ns_starts = [(m.start(), m.group(1)) for m in NS.finditer(text)]
    out = {}
    for m in DECL.finditer(text):
        name, k, body = m.group(1), int(m.group(2)), m.group(3)
        chunks = [int(c.strip(), 0) for c in body.split(",") if c.strip()]
        assert len(chunks) == k, (name, len(chunks), k)
        ns = None
        for pos, nname in ns_starts:
            if pos < m.start():
                ns = nname
        # a namespace closes before top-level decls; decide by brace depth
        depth_ns = _namespace_at(text, m.start())
        key = f"{depth_ns}.{name}" if depth_ns else name
        out[key] = list(reversed(chunks))
    return out


def _namespace_at(text, pos):
    stack = []
    i = 0
    tok = re.compile(r"namespace\s+(\w+)\s*\{|\{|\}")
    for m in tok.finditer(text, 0, pos):
        if m.group(0).startswith("namespace"):
            stack.append(m.group(1))
        elif m.group(0) == "{":
            stack.append(None)
        else:
            if stack:
                stack.pop()
    names = [s for s in stack if s]
    return names[-1] if names else None


PARAM = re.compile(r"const\s+Number\s+(\w+)\s*=\s*BIG_INTEGER_CHUNKS8\(([^)]*)\)")
MPRIME = re.compile(r"m_prime\s*=\s*(\d+)")


def parse_params(path):
    """host_constants of a field header (bn254_fr.cuh:31-38, bn254_fq.cuh:21-28) + m_prime."""
    text = open(path).read()
    host = text[text.index("namespace host_constants"):]
    out = {}
    for m in PARAM.finditer(host):
        if m.group(1) in out:
            continue
        chunks = [int(c.strip(), 0) for c in m.group(2).split(",")]
        out[m.group(1)] = list(reversed(chunks))
    out["m_prime"] = int(MPRIME.search(text).group(1))
    return out


def main():
    params = {
        "fr": parse_params(os.path.join(ROOT, "core/src/common/mont/src/bn254_fr.cuh")),
        "fq": parse_params(os.path.join(ROOT, "core/src/common/mont/src/bn254_fq.cuh")),
    }
    mont = parse(os.path.join(ROOT, "core/src/common/mont/tests/main.cu"))
    curve = parse(os.path.join(ROOT, "core/src/common/curve/tests/bn254.cu"))
    # drop the commented-out lt_2m block constants (inside a // comment in the source)
    curve = {k: v for k, v in curve.items() if k in
             ("p1_x", "p1_y", "p2_x", "p2_y", "pr_x", "pr_y", "pr100_x", "pr100_y",
              "p1r128_x", "p1r128_y")}
    data = {
        "source": {
            "mont": "core/src/common/mont/tests/main.cu",
            "curve": "core/src/common/curve/tests/bn254.cu",
        },
        "limb_order": "little-endian u32 limbs",
        "params": params,
        "fr": mont,
        "g1": curve,
    }
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    print(f"wrote {OUT}: {len(mont)} Fr vectors, {len(curve)} G1 coordinates")


if __name__ == "__main__":
    main()
