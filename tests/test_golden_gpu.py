"""GPU parity against the golden fixtures (tests/golden/), at the configurations' full sizes.

The library runs on the fixtures' inputs through the C ABI (ttcuda); the FP64 oracle fingerprints
its outputs (ranks, ot, singular values of every bond, norm, probe inner products, distance to
the input) and golden.compare checks them against the stored oracle results.  Tolerances:
FP64 paths 1e-10; mixed-precision paths (BF16 or TF32 sketch contractions) 1e-5, the bound the
specification of this path states for them.  Ranks must be identical in every case.

The PPP benzene test builds the reference test's Hamiltonian (test/test_models.jl:24-30) with
every tt_rounding(::TToperator) step done by the library and checks the reference's known
ground-state energy.
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

ttcuda = pytest.importorskip("ttcuda")
from gpu_helpers import op_dev, to_dev, to_or  # noqa: E402
from oracle import models_oracle as mo  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402

import golden  # noqa: E402
import make_golden as mg  # noqa: E402

FP64_TOL = 1e-10
MIXED_TOL = 1e-5
PPP_BENZENE_ENERGY = -0.46752535023652453    # test/test_models.jl:29


@pytest.fixture(scope="module", autouse=True)
def ctx():
    yield ttcuda.get_context()


def _check(got_tt, x, expected, tol, check_ot=True):
    fp = golden.fingerprint(to_or(got_tt), x)
    bad = golden.compare(fp, expected, tol, check_ot=check_ot)
    assert bad == [], bad[:6]
    return fp


def test_golden_config1_tt_rounding():
    """Config 1: X = sum_j 2^-j X_j formed on the device (tt_scale, tt_add) from the terms stored
    in the reference's JSON schema, then tt_rounding(X; tol=1e-8, rmax=64)."""
    fx = golden.load("config1_sum_of_tts.json.gz")
    terms = [ttcuda.json_to_mps(t) for t in fx["terms"]]
    X = None
    for j, t in enumerate(terms, start=1):
        t = ttcuda.tt_scale(2.0 ** -j, t)
        X = t if X is None else ttcuda.tt_add(X, t)
    Xo = to_or(X)
    assert golden.checksum_ok(golden.checksum(Xo), fx["input_checksum"])
    Y = ttcuda.tt_rounding(X, tol=fx["params"]["tol"], rmax=fx["params"]["rmax"])
    _check(Y, Xo, fx["expected"], FP64_TOL)


@pytest.fixture(scope="module")
def config3():
    fx = golden.load("config3_batch3.json.gz")
    xs = mg.config3_inputs()
    for x, cs in zip(xs, fx["input_checksums"]):
        assert golden.checksum_ok(golden.checksum(x), cs)
    return fx, xs


def test_golden_config3_batched_tt_rounding(config3):
    fx, xs = config3
    xb = ttcuda.DeviceBatch.from_tts([to_dev(x) for x in xs])
    yb = ttcuda.DeviceBatch(xs[0].ttv_dims, [x.ttv_rks for x in xs])
    xb.round_det(yb, tol=fx["params"]["tol"])
    for got, x, exp in zip(yb.download(), xs, fx["expected_det"]):
        _check(got, x, exp, FP64_TOL)


@pytest.mark.parametrize("precision,uploaded", [("fp64", True), ("bf16", True), ("bf16", False), ("tf32", True)])
def test_golden_config3_randomized_then_svd_sweep(config3, precision, uploaded):
    """ttrand_rounding with the batch's heuristic ranks and orthogonal sketch blocks (uploaded from
    the host, or drawn on the device from the same Philox stream), then tt_rounding(tol=1e-8)."""
    fx, xs = config3
    rks = fx["rks"]
    N = xs[0].N
    dims = xs[0].ttv_dims
    blocks = mg.config3_blocks(rks, N, dims)[0] if uploaded else None
    s = ttcuda._sketch_ranks(dims, rks, N)
    xb = ttcuda.DeviceBatch.from_tts([to_dev(x) for x in xs])
    yb = ttcuda.DeviceBatch(dims, [ttcuda._rand_out_caps(dims, s)] * len(xs))
    xb.round_rand(yb, rks, orthogonal=True, seed=fx["params"]["sketch_seed"], block_rks=N, precision=precision,
                  after_tol=fx["params"]["tol"], sketch_blocks=blocks)
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    for got, x, exp in zip(yb.download(), xs, fx["expected_rand_then_det"]):
        _check(got, x, exp, tol)


@pytest.mark.parametrize("uploaded", [True, False])
def test_golden_config2_operator_rounding(uploaded):
    """Config 2: ttrand_rounding([1.0], H, [y], rks) without forming H y, FP64 sketch, the MPO from
    the fixture's JSON and y regenerated from its seed."""
    fx = golden.load("config2_hubbard_op.json.gz")
    H = ttcuda.json_to_mpo(fx["mpo"])
    _, y = mg.config2_inputs()
    assert golden.checksum_ok(golden.checksum(y), fx["y_checksum"])
    p = fx["params"]
    blocks = None
    if uploaded:
        blocks = o.make_reverse_sketch(y.ttv_dims, fx["rks"], seed=p["sketch_seed"], orthogonal=p["orthogonal"],
                                       block_rks=p["s"])[0]
    z = ttcuda.ttrand_rounding_op([1.0], H, [to_dev(y)], fx["rks"], orthogonal=p["orthogonal"],
                                  seed=p["sketch_seed"], block_rks=p["s"], sketch_blocks=blocks)
    # the distance to H y (rank ~900) takes minutes in the oracle: singular values, probes and the
    # norm pin the result here
    _check(z, None, fx["expected"], FP64_TOL)


def _gpu_round_tto(A, tol):
    """tt_rounding(::TToperator) (src/tt_rounding.jl:275-277) with the rounding on the device."""
    v = o.tto_to_ttv(A)
    r = ttcuda.tt_rounding(to_dev(v), tol=tol)
    return o.ttv_to_tto(to_or(r))


def test_ppp_benzene_known_answer_with_device_rounding():
    H = mo.PPP_C_NH_N(6, order=np.random.default_rng(3).permutation(12), round_tto=_gpu_round_tto)
    n = H.N
    M = o.tto_to_tensor(H).reshape(2 ** n, 2 ** n, order="F")
    idx = np.arange(2 ** n)
    sel = idx[np.array([bin(i).count("1") for i in idx]) == 6]
    e = float(np.linalg.eigvalsh(M[np.ix_(sel, sel)])[0])
    assert abs(e - PPP_BENZENE_ENERGY) <= 1e-6          # the reference's tolerance
    assert abs(e - PPP_BENZENE_ENERGY) <= 1e-11
