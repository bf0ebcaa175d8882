"""Host-side check of the MSM pairing rounds' index arithmetic (csrc/msm.cu, stage 4a), restated
in Python: slot-major pair slots (thread t takes slots t, t + T, ...), list r + 1's bucket counts
o + ceil((m_b - o) / 2) with o = s_b mod 2, a point's destination s'_b + (e - s_b + o) / 2, the
list-length bound E_{r+1} <= E_r / 2 + nb and the per-thread prefix slots.  Every point must land
exactly once, in its own bucket's run, and each bucket's points must be preserved through R
rounds.  No GPU: this pins the layout the kernels and the workspace sizes rely on."""
import random

import pytest

KA = 64  # list elements per thread (KA / 2 pair slots)


def _round(lst, starts, nb, emax_r, emax_next):
    E = starts[nb]
    assert E == len(lst) <= emax_r
    cnt = []
    for b in range(nb):
        s0, mb = starts[b], starts[b + 1] - starts[b]
        o = s0 & 1
        cnt.append(0 if mb == 0 else o + (mb - o + 1) // 2)
    sn = [0]
    for c in cnt:
        sn.append(sn[-1] + c)
    assert sn[nb] <= emax_next
    nthr = (emax_r + KA - 1) // KA
    out = [None] * sn[nb]
    seen = set()
    for t in range(nthr):
        for k in range(KA // 2 - 1, -1, -1):
            e0 = 2 * (t + k * nthr)
            if e0 >= E:
                continue
            b0 = lst[e0][0]
            b1 = lst[e0 + 1][0] if e0 + 1 < E else None
            val = list(lst[e0][1])
            seen.add(e0)
            if b1 == b0:
                val += lst[e0 + 1][1]
                seen.add(e0 + 1)
            elif b1 is not None:
                s1 = starts[b1]
                q1 = sn[b1] + ((e0 + 1 - s1 + (s1 & 1)) >> 1)
                assert sn[b1] <= q1 < sn[b1 + 1] and out[q1] is None
                out[q1] = (b1, list(lst[e0 + 1][1]))
                seen.add(e0 + 1)
            s0 = starts[b0]
            q0 = sn[b0] + ((e0 - s0 + (s0 & 1)) >> 1)
            assert sn[b0] <= q0 < sn[b0 + 1] and out[q0] is None
            out[q0] = (b0, val)
    assert seen == set(range(E)) and all(o is not None for o in out)
    return out, sn


def _run(counts, rounds):
    nb = len(counts)
    emax = [sum(counts)]
    for _ in range(rounds):
        e = emax[-1]
        emax.append(min((e + 1) // 2 + nb, e))
    starts = [0]
    for c in counts:
        starts.append(starts[-1] + c)
    lst = [(b, [(b, k)]) for b, c in enumerate(counts) for k in range(c)]
    for r in range(rounds):
        lst, starts = _round(lst, starts, nb, emax[r], emax[r + 1])
    got = {}
    for b, v in lst:
        got.setdefault(b, []).extend(v)
    for b, c in enumerate(counts):
        assert sorted(got.get(b, [])) == [(b, k) for k in range(c)]


@pytest.mark.parametrize("seed", range(40))
def test_pairing_layout_random(seed):
    rng = random.Random(seed)
    nb = rng.choice([1, 2, 5, 64, 300])
    mode = seed % 3
    if mode == 0:
        counts = [rng.randint(0, 3) for _ in range(nb)]
    elif mode == 1:
        counts = [rng.randint(0, 200) for _ in range(nb)]
    else:
        counts = [0] * nb
        counts[rng.randrange(nb)] = rng.randint(1, 5000)
    _run(counts, rng.randint(1, 4))


def test_pairing_layout_edges():
    _run([0, 0, 0], 3)          # empty list
    _run([1], 4)                # one point
    _run([1, 1, 1, 1, 1], 2)    # every bucket a single
    _run([3, 2, 7, 1, 0, 9], 4)  # odd starts
