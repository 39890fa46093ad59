"""Randomized rounding of Hadamard products on the GPU (ttc_ttrand_rounding_hadamard, structured
Kronecker contractions for the last factor, src/tt_randtools.jl:364-473) against the oracle,
which multiplies the product out and rounds it with the same Philox sketch blocks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
from gpu_helpers import rel, to_dev, to_or  # noqa: E402
from oracle import hadamard_oracle as ho  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402


@pytest.mark.parametrize("d,ranks,rk,orth,block", [(6, (3, 2), 5, True, None), (8, (4, 3), 10, True, 4),
                                                   (7, (2, 3, 2), 8, False, 3), (6, (3, 1), 4, True, None),
                                                   (12, (8, 6), 20, True, 6), (10, (5, 4, 3), 16, True, 8),
                                                   (16, (16, 12), 48, True, 8)])
def test_hadamard_rounding_matches_oracle(d, ranks, rk, orth, block):
    g = np.random.default_rng(d * 31 + sum(ranks))
    ys = [o.rand_tt((2,) * d, r, g, normalise=True) for r in ranks]
    rks = [1] + [rk] * (d - 1) + [1]
    want = ho.ttrand_rounding_hadamard(ys, rks, orth, 77, block)
    got = ttcuda.ttrand_rounding_hadamard([to_dev(t) for t in ys], rks, orthogonal=orth, seed=77, block_rks=block)
    assert list(got.ttv_rks) == list(want.ttv_rks)
    assert list(got.ttv_ot) == [1] * (d - 1) + [0]
    assert rel(got, want) < 1e-10
    if rk >= int(np.prod(ranks)):
        prod = ys[0]
        for t in ys[1:]:
            prod = ho.hadamard(prod, t)
        assert o.rel_error(prod, to_or(got)) < 1e-10


def test_hadamard_rounding_single_factor_and_int_rmax():
    g = np.random.default_rng(3)
    x = o.rand_tt((2,) * 8, 6, g, normalise=True)
    got = ttcuda.ttrand_rounding_hadamard([to_dev(x)], 8)
    want = o.ttrand_rounding(x, 8)
    assert list(got.ttv_rks) == list(want.ttv_rks) and rel(got, want) < 1e-10
    y = o.rand_tt((2,) * 8, 3, g, normalise=True)
    got2 = ttcuda.ttrand_rounding_hadamard([to_dev(x), to_dev(y)], 12, seed=9)
    want2 = ho.ttrand_rounding_hadamard([x, y], [1] + [12] * 7 + [1], True, 9, None)
    assert list(got2.ttv_rks) == list(want2.ttv_rks) and rel(got2, want2) < 1e-10


def test_hadamard_rounding_requires_ranks():
    g = np.random.default_rng(4)
    x = o.rand_tt((2,) * 5, 2, g)
    with pytest.raises(ttcuda.ArgumentError):
        ttcuda.ttrand_rounding_hadamard([to_dev(x), to_dev(x)], None)
