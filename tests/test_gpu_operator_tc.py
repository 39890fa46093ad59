"""The operator sketch on the tcgen05 tensor cores (src/sketches.jl:1648-1713 in BF16 or TF32 with
FP32 accumulation) against the FP64 oracle, and the operator-aware randomized rounding that
consumes it (src/tt_randtools.jl:285-354), including config 2's full size against its golden
fixture (the deviation of the mixed-precision result from the FP64 one is bounded by the
randomized rounding's own error, since a perturbed sketch is another random sketch)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
from gpu_helpers import op_dev, rel, to_dev, to_or  # noqa: E402
from oracle import models_oracle as mo  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))


def _case():
    h, V = mo.hubbard_1D(5, t=1.0, U=4.0)
    H = mo.hV_to_mpo(h, V, (2,) * 10)
    x = o.rand_tt((2,) * 10, 8, np.random.default_rng(23), normalise=True)
    return H, x


@pytest.mark.parametrize("precision,tol", [("bf16", 3e-2), ("tf32", 5e-3)])
def test_operator_sketch_tensor_cores_close_to_fp64(precision, tol):
    H, x = _case()
    rks = [1] + [20] * 9 + [1]
    blocks = o.make_reverse_sketch(x.ttv_dims, rks, seed=7, orthogonal=False, block_rks=20)[0]
    Wr, sr = o.tt_recursive_sketch_op(H, x, rks, orthogonal=False, block_rks=20, blocks=blocks)
    Wg, sg = ttcuda.tt_recursive_sketch(to_dev(x), rks, H=op_dev(H), orthogonal=False, block_rks=20,
                                        precision=precision, sketch_blocks=blocks)
    assert sg == sr
    num = sum(np.linalg.norm(a - b) ** 2 for a, b in zip(Wg, Wr)) ** 0.5
    den = sum(np.linalg.norm(b) ** 2 for b in Wr) ** 0.5
    assert num <= tol * den


def test_operator_sketch_tf32_closer_than_bf16_with_blocks():
    """Several sketch blocks per site (block_rks=4): every block's three GEMMs on the tensor cores."""
    H, x = _case()
    rks = [1, 3, 7, 9, 9, 9, 9, 9, 7, 3, 1]
    blocks = o.make_reverse_sketch(x.ttv_dims, rks, seed=9, orthogonal=False, block_rks=4)[0]
    Wr, sr = o.tt_recursive_sketch_op(H, x, rks, orthogonal=False, block_rks=4, blocks=blocks)
    errs = {}
    for p in ("tf32", "bf16"):
        Wg, sg = ttcuda.tt_recursive_sketch(to_dev(x), rks, H=op_dev(H), orthogonal=False, block_rks=4, precision=p,
                                            sketch_blocks=blocks)
        assert sg == sr
        errs[p] = sum(np.linalg.norm(a - b) ** 2 for a, b in zip(Wg, Wr)) ** 0.5
    den = sum(np.linalg.norm(b) ** 2 for b in Wr) ** 0.5
    assert errs["tf32"] < errs["bf16"] <= 3e-2 * den


@pytest.mark.parametrize("precision", ["bf16", "tf32"])
def test_operator_rounding_mixed_precision_error_matches_fp64(precision):
    """Rounding H x without forming it, with a sketch of rank 30 against H x of rank up to 7*8: the
    tensor-core sketch's error exceeds the FP64 sketch's by at most 1e-5 (the bound stated for the
    mixed-precision paths; the levels whose right interface is structurally rank deficient are
    contracted in FP64, which keeps the BF16 and TF32 results this close), and the FP64 range
    finder keeps the cores orthonormal."""
    H, x = _case()
    rks = [1] + [30] * 9 + [1]
    Hx = o.tto_apply(H, x)
    z64 = ttcuda.ttrand_rounding_op([1.0], op_dev(H), [to_dev(x)], rks, orthogonal=False, seed=3, block_rks=30)
    ztc = ttcuda.ttrand_rounding_op([1.0], op_dev(H), [to_dev(x)], rks, orthogonal=False, seed=3, block_rks=30,
                                    precision=precision)
    assert ztc.ttv_rks == z64.ttv_rks
    e64, etc = rel(z64, Hx), rel(ztc, Hx)
    assert etc <= e64 + 1e-5, (etc, e64)
    for c in ztc.ttv_vec[:-1]:
        Q = np.asarray(c).reshape(-1, c.shape[2], order="F")
        assert np.abs(Q.T @ Q - np.eye(Q.shape[1])).max() < 1e-12


def test_config2_full_size_tf32_operator_rounding_against_golden():
    """Config 2 at full size with the TF32 operator sketch: identical ranks, and every bond's
    singular values within 2 % of the FP64 oracle's (the relative spread of a rank-138 randomized
    rounding of a rank-896 product across sketches is larger)."""
    import golden
    import make_golden as mg
    fx = golden.load("config2_hubbard_op.json.gz")
    H = ttcuda.json_to_mpo(fx["mpo"])
    _, y = mg.config2_inputs()
    p = fx["params"]
    z = ttcuda.ttrand_rounding_op([1.0], H, [to_dev(y)], fx["rks"], orthogonal=p["orthogonal"], seed=p["sketch_seed"],
                                  block_rks=p["s"], precision="tf32")
    assert z.ttv_rks == fx["expected"]["ranks"]
    sv = o.tt_svdvals(to_or(z))
    worst = max(float(np.abs(a - np.asarray(b)).max() / max(b)) for a, b in zip(sv, fx["expected"]["svals"]))
    assert worst < 2e-2, worst
