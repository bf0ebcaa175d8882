"""Device input generator vs the oracle's generator (same bytes)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_gen_fr_matches_oracle(zk, orc):
    got = zk.gen.fr(1, 5000).cpu().numpy().view(np.uint64).reshape(-1, 4)
    assert np.array_equal(got, orc.gen_fr(1, 5000))
    got = zk.gen.fr(0, 100, start=1 << 20).cpu().numpy().view(np.uint64).reshape(-1, 4)
    assert np.array_equal(got, orc.gen_fr(0, 100, start=1 << 20))


def test_gen_points_matches_oracle(zk, orc):
    got = zk.gen.points(2, 3000).cpu().numpy().view(np.uint64).reshape(-1, 8)
    assert np.array_equal(got, orc.gen_points(2, 3000))
    got = zk.gen.points(2, 50, start=(1 << 22) - 50).cpu().numpy().view(np.uint64).reshape(-1, 8)
    assert np.array_equal(got, orc.gen_points(2, 50, start=(1 << 22) - 50))
