"""The Hadamard-product oracle (oracle/hadamard_oracle.py) on CPU: the slice-wise Kronecker
product is the element-wise product of the dense tensors, and its randomized rounding with
sketch ranks at least the product ranks reproduces it."""
import numpy as np

from oracle import hadamard_oracle as ho
from oracle import tt_oracle as o


def test_hadamard_is_elementwise_product():
    g = np.random.default_rng(0)
    x = o.rand_tt((2, 3, 2, 2), 3, g)
    y = o.rand_tt((2, 3, 2, 2), 2, g)
    z = ho.hadamard(x, y)
    assert z.ttv_rks == [a * b for a, b in zip(x.ttv_rks, y.ttv_rks)]
    assert np.allclose(o.ttv_to_tensor(z), o.ttv_to_tensor(x) * o.ttv_to_tensor(y), rtol=1e-13, atol=1e-13)


def test_hadamard_rounding_exact_at_full_rank():
    g = np.random.default_rng(1)
    ys = [o.rand_tt((2,) * 7, r, g, normalise=True) for r in (3, 2, 2)]
    rks = [1] + [16] * 6 + [1]
    z = ho.ttrand_rounding_hadamard(ys, rks, seed=5, block_rks=4)
    d = o.ttv_to_tensor(ys[0]) * o.ttv_to_tensor(ys[1]) * o.ttv_to_tensor(ys[2])
    assert np.linalg.norm(o.ttv_to_tensor(z) - d) <= 1e-12 * np.linalg.norm(d)
