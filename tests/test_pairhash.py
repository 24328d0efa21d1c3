"""The order-independent pair-set digest (xmatch_b200/pairhash.py) that the
full-size 50M x 50M parity check compares: same set in any order gives the
same digest; a missing, extra or altered pair changes it."""
import numpy as np

from xmatch_b200 import pairhash


def test_digest_order_independent_and_sensitive():
    rng = np.random.default_rng(3)
    p = np.stack([rng.integers(0, 1 << 40, 100_000), rng.integers(0, 1 << 40, 100_000)], 1).astype(np.int64)
    d = pairhash.pairset_digest(p)
    assert d == pairhash.pairset_digest(p[rng.permutation(len(p))])
    assert d == pairhash.pairset_digest(p, chunk=997)
    assert d["count"] == len(p)
    assert pairhash.pairset_digest(p[1:]) != d
    q = p.copy()
    q[5, 1] += 1
    assert pairhash.pairset_digest(q)["sum"] != d["sum"]
    r = p.copy()
    r[7] = r[7, ::-1]          # (idA, idB) is ordered: the swapped pair is another pair
    assert pairhash.pairset_digest(r) != d
    assert pairhash.pairset_digest(np.empty((0, 2), np.int64)) == {"count": 0, "sum": "%016x" % 0,
                                                                   "xor": "%016x" % 0}


def test_digest_of_golden_fixture_pairs(golden_dir):
    import os
    p = np.load(os.path.join(golden_dir, "pairs_test_x_test_r5.npz"))["pairs"]
    d = pairhash.pairset_digest(p)
    assert d == pairhash.pairset_digest(p[::-1].copy())
