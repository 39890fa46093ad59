"""STTA on the GPU (ttc_stta: forward and reverse sketches, overlaps, pseudo-inverses and joins
in one plan, src/tt_randtools.jl:551-641) against the oracle's restatement
(oracle/stta_oracle.py), with the same Philox sketch blocks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
from gpu_helpers import rel, to_dev, to_or  # noqa: E402
from oracle import stta_oracle as so  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402


@pytest.mark.parametrize("d,r,rk,orth,block", [(8, 5, 8, True, 4), (8, 5, 8, False, None), (10, 16, 8, True, 4),
                                               (12, 24, 12, False, 6), (16, 40, 24, True, 8), (6, 3, 5, True, 2)])
def test_stta_matches_oracle(d, r, rk, orth, block):
    g = np.random.default_rng(d * 100 + r)
    x = o.rand_tt((2,) * d, r, g, normalise=True)
    want = so.stta(x, rk, orthogonal=orth, block_rks=block, seed_left=11, seed_right=22)
    got = ttcuda.stta(to_dev(x), rk, orthogonal=orth, block_rks=block, seed_left=11, seed_right=22)
    assert list(got.ttv_rks) == list(want.ttv_rks)
    assert list(got.ttv_ot) == [0] * d
    assert rel(got, want) < 1e-9
    if rk >= r:
        assert o.rel_error(x, to_or(got)) < 1e-10           # exact when the sketches reach the rank


def test_stta_default_ranks_and_lincomb():
    g = np.random.default_rng(7)
    x1 = o.rand_tt((2,) * 10, 6, g, normalise=True)
    x2 = o.rand_tt((2,) * 10, 4, g, normalise=True)
    got = ttcuda.stta(to_dev(x1))
    want = so.stta(x1)
    assert list(got.ttv_rks) == list(want.ttv_rks) and rel(got, want) < 1e-9
    zl = ttcuda.stta_lincomb([0.5, -2.0], [to_dev(x1), to_dev(x2)], 12, block_rks=4)
    zo = so.stta_lincomb([0.5, -2.0], [x1, x2], 12, block_rks=4)
    assert list(zl.ttv_rks) == list(zo.ttv_rks) and rel(zl, zo) < 1e-9
    ref = o.tt_add(o.tt_scale(0.5, x1), o.tt_scale(-2.0, x2))
    assert o.rel_error(ref, to_or(zl)) < 1e-10


def test_stta_rejects_bad_boundary_ranks():
    g = np.random.default_rng(1)
    x = o.rand_tt((2,) * 6, 3, g)
    with pytest.raises(ttcuda.DimensionMismatch):
        ttcuda.stta(to_dev(x), [2, 4, 4, 4, 4, 4, 1])
