"""The Rayleigh-quotient gradient with FP32 contractions and FP32 accumulation (config 4's FP32
variant): against the oracle's FP64 contraction at a small size and against the library's FP64
gradient at config 4's full size (4x4 open Hubbard, U=8, snake ordering, rank 256, environments
checkpointed every 4 sites).  FP32 accumulation over sums of a few thousand terms keeps about
six significant digits, so the bound is 1e-4 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
from gpu_helpers import op_dev, to_dev  # noqa: E402
from oracle import models_oracle as mo  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402


def _rel_grad(G, Gr):
    num = sum(float(np.sum((np.asarray(a) - np.asarray(b)) ** 2)) for a, b in zip(G, Gr)) ** 0.5
    den = sum(float(np.sum(np.asarray(b) ** 2)) for b in Gr) ** 0.5
    return num / den


@pytest.mark.parametrize("ckpt", [1, 3])
def test_fp32_gradient_against_oracle(ckpt):
    h, V = mo.hubbard_1D(4, t=1.0, U=4.0)
    H = mo.hV_to_mpo(h, V, (2,) * 8)
    x = o.rand_tt((2,) * 8, 6, np.random.default_rng(31), normalise=True)
    R, G = ttcuda.rayleigh_grad(op_dev(H), to_dev(x), ckpt_every=ckpt, precision="fp32")
    Rr, Gr = o.rayleigh_value_and_grad(H, x)
    assert abs(R - Rr) <= 1e-5 * abs(Rr)
    assert _rel_grad(G, Gr) <= 1e-4


def test_fp32_gradient_config4_full_size_against_fp64():
    h, V = mo.hubbard_2D(4, 4, t=1.0, U=8.0, w_pbc=False, L_pbc=False)
    s = mo.snake_permutation(4, 4)
    H = op_dev(mo.hV_to_mpo(h[np.ix_(s, s)], V[np.ix_(s, s, s, s)], (2,) * 32))
    x = to_dev(o.rand_tt((2,) * 32, 256, np.random.default_rng(41), normalise=True))
    R64, G64 = ttcuda.rayleigh_grad(H, x, ckpt_every=4, precision="fp64")
    R32, G32 = ttcuda.rayleigh_grad(H, x, ckpt_every=4, precision="fp32")
    assert abs(R32 - R64) <= 1e-5 * abs(R64)
    assert _rel_grad(G32, G64) <= 1e-4


def test_gradient_precision_is_validated():
    h, V = mo.hubbard_1D(2, t=1.0, U=1.0)
    H = mo.hV_to_mpo(h, V, (2,) * 4)
    x = o.rand_tt((2,) * 4, 2, np.random.default_rng(1))
    with pytest.raises(ttcuda.ArgumentError):
        ttcuda.rayleigh_grad(op_dev(H), to_dev(x), precision="bf16")
