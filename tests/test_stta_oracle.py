"""The STTA oracle (oracle/stta_oracle.py) on CPU: exact reconstruction when the sketch ranks
reach the TT ranks, linear combinations, the forward block plan, and a compression error close
to the truncated SVD's."""
import numpy as np
import pytest

from oracle import stta_oracle as so
from oracle import tt_oracle as o


def test_forward_plan_monotone_and_oversampled():
    b, p = so.forward_sketch_plan((2,) * 8, 8, [1] + [6] * 7 + [1], 4, 1.5)
    assert b == [1, 2, 4, 4, 4, 4, 4, 4, 4]
    assert p[0] == 1 and all(p[i] >= p[i + 1] for i in range(1, 8))
    b1, p1 = so.forward_sketch_plan((2,) * 8, 8, [1] + [6] * 7 + [1], 4, 1.0)
    assert p == [1] + [int(np.ceil(1.5 * v)) for v in p1[1:]]


@pytest.mark.parametrize("orth,block", [(True, 4), (False, None), (True, 2)])
def test_stta_exact_when_sketch_reaches_rank(orth, block):
    g = np.random.default_rng(3)
    x = o.rand_tt((2,) * 8, 5, g, normalise=True)
    y = so.stta(x, 8, orthogonal=orth, block_rks=block)
    assert o.rel_error(x, y) < 1e-11


def test_stta_lincomb_exact():
    g = np.random.default_rng(4)
    x1 = o.rand_tt((2,) * 8, 5, g, normalise=True)
    x2 = o.rand_tt((2,) * 8, 3, g, normalise=True)
    z = so.stta_lincomb([0.5, -2.0], [x1, x2], 10, block_rks=4)
    ref = o.tt_add(o.tt_scale(0.5, x1), o.tt_scale(-2.0, x2))
    assert o.rel_error(ref, z) < 1e-11


def test_stta_compression_near_optimal():
    """Rank-8 STTA of a rank-16 TT: its error is within a small factor of the best rank-8
    (truncated-SVD) error."""
    g = np.random.default_rng(9)
    x = o.rand_tt((2,) * 10, 16, g, normalise=True)
    y = so.stta(x, 8, block_rks=4)
    best = o.tt_rounding(x, rmax=8)
    e, eb = o.rel_error(x, y), o.rel_error(x, best)
    assert eb < e < 5 * eb
