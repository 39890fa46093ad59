"""GPU parity of libttcuda against the FP64 oracle (same seeded inputs, same sketches).

Tolerances: FP64 paths match the oracle's represented tensor to 1e-10 relative and the
truncation ranks exactly (singular values of these inputs are separated far more than
1e-6 relative at the cut); the BF16-sketch path matches to 1e-8 when the sketch rank
covers the TT rank (the range finder then spans the exact column space).
"""
import math

import numpy as np
import pytest

from oracle import tt_oracle as o
from oracle import models_oracle as mo

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
from gpu_helpers import decaying_tt, op_dev, rel, rel_dense, sum_of_tts, to_dev, to_or  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def ctx():
    c = ttcuda.get_context()
    yield c


# ------------------------------------------------------------------ deterministic rounding
def test_tt_rounding_sum_of_tts_config1_small():
    """Config-1 shape (n=2, d=20, sum of 8 rank-8 TTs, tol 1e-8, rmax 64)."""
    X = sum_of_tts((2,) * 20, 8, 8, seed=1)
    ref = o.tt_rounding(X, tol=1e-8, rmax=64)
    got = ttcuda.tt_rounding(to_dev(X), tol=1e-8, rmax=64)
    assert got.ttv_rks == ref.ttv_rks
    assert got.ttv_ot == ref.ttv_ot
    assert rel(got, ref) < 1e-10
    assert rel(got, X) < 1e-8 * 2


@pytest.mark.parametrize("direction", ["left", "right"])
def test_tt_rounding_directions_dense(direction):
    g = np.random.default_rng(2)
    x = o.rand_tt((2,) * 8, [1, 2, 4, 8, 8, 8, 4, 2, 1], g)
    y = o.tt_add(x, o.tt_scale(0.5, x))       # rank doubles, true rank unchanged
    ref = o.tt_rounding(y, tol=1e-10, direction=direction)
    got = ttcuda.tt_rounding(to_dev(y), tol=1e-10, direction=direction)
    assert got.ttv_rks == ref.ttv_rks == [1, 2, 4, 8, 8, 8, 4, 2, 1]
    assert got.ttv_ot == ref.ttv_ot
    assert rel_dense(got, y) < 1e-12


def test_tt_rounding_truncation_and_rmax():
    x = decaying_tt((2,) * 12, [1, 2, 4, 8, 16, 32, 40, 32, 16, 8, 4, 2, 1], seed=3, decay_per=4.0)
    for tol, rmax in [(1e-3, 2 ** 14), (1e-6, 2 ** 14), (1e-6, 10), (0.0, 2 ** 14)]:
        ref = o.tt_rounding(x, tol=tol, rmax=rmax)
        got = ttcuda.tt_rounding(to_dev(x), tol=tol, rmax=rmax)
        assert got.ttv_rks == ref.ttv_rks, (tol, rmax)
        assert rel(got, ref) < 1e-10


def test_tt_rounding_left_orthogonal_input_skips_qr():
    x = o.orthogonalize(o.rand_tt((2,) * 10, 6, np.random.default_rng(4)), i=10)
    assert o.is_leftorthogonal(x)
    ref = o.tt_rounding(x, tol=1e-9)
    got = ttcuda.tt_rounding(to_dev(x), tol=1e-9)
    assert got.ttv_rks == ref.ttv_rks
    assert rel(got, ref) < 1e-11


def test_tt_rounding_zero_tensor_early_exit():
    """norm(core N) < tol returns zeros_tt with the orthogonalised ranks (src/tt_rounding.jl:179-181)."""
    x = o.rand_tt((2,) * 6, 3, np.random.default_rng(5))
    x.ttv_vec = [c * 1e-30 for c in x.ttv_vec]
    ref = o.tt_rounding(x, tol=1e-8)
    got = ttcuda.tt_rounding(to_dev(x), tol=1e-8)
    assert got.ttv_rks == ref.ttv_rks
    assert all(np.all(c == 0) for c in got.ttv_vec)
    assert got.ttv_ot == [0] * 6


def test_tt_rounding_zero_padded_ranks():
    """tt_up_rks pads with exact zeros: rank-deficient QR/SVD inputs."""
    x = o.rand_tt((2,) * 8, [1, 2, 4, 4, 4, 4, 4, 2, 1], np.random.default_rng(6))
    y = o.tt_up_rks(x, 12)
    ref = o.tt_rounding(y, tol=1e-10)
    got = ttcuda.tt_rounding(to_dev(y), tol=1e-10)
    assert got.ttv_rks == ref.ttv_rks
    assert rel_dense(got, x) < 1e-12


def test_tt_rounding_small_N():
    for N in (1, 2, 3):
        x = o.rand_tt((3,) * N, 3, np.random.default_rng(7 + N))
        ref = o.tt_rounding(x, tol=1e-12)
        got = ttcuda.tt_rounding(to_dev(x), tol=1e-12)
        assert got.ttv_rks == ref.ttv_rks
        assert rel_dense(got, x) < 1e-12


def test_invalid_direction_raises():
    x = o.rand_tt((2,) * 4, 2, np.random.default_rng(8))
    with pytest.raises(ttcuda.ArgumentError):
        ttcuda.tt_rounding(to_dev(x), direction="up")


@pytest.mark.parametrize("root", [1, 4, 8])
def test_orthogonalize(root):
    x = o.rand_tt((2,) * 8, [1, 2, 4, 8, 8, 8, 4, 2, 1], np.random.default_rng(9))
    ref = o.orthogonalize(x, i=root)
    got = ttcuda.orthogonalize(to_dev(x), i=root)
    assert got.ttv_rks == ref.ttv_rks
    assert got.ttv_ot == ref.ttv_ot
    assert rel_dense(got, x) < 1e-12
    for k in range(8):
        c = got.ttv_vec[k]
        if k < root - 1:
            assert np.allclose(sum(c[i].T @ c[i] for i in range(2)), np.eye(c.shape[2]), atol=1e-12)
        elif k > root - 1:
            assert np.allclose(sum(c[i] @ c[i].T for i in range(2)), np.eye(c.shape[1]), atol=1e-12)


def test_norm():
    x = o.rand_tt((2,) * 10, 5, np.random.default_rng(10))
    assert math.isclose(ttcuda.norm(to_dev(x)), o.norm(x), rel_tol=1e-12)


# ------------------------------------------------------------------ sketches, randomized rounding
def _blocks(x, rks, orthogonal, block_rks=None, seed=1234):
    return o.make_reverse_sketch(x.ttv_dims, rks, seed=seed, orthogonal=orthogonal, block_rks=block_rks)[0]


@pytest.mark.parametrize("orthogonal", [False, True])
@pytest.mark.parametrize("block_rks", [None, 3, 16])
def test_recursive_sketch_host_blocks(orthogonal, block_rks):
    x = o.rand_tt((2,) * 8, [1, 2, 4, 8, 8, 8, 4, 2, 1], np.random.default_rng(11))
    rks = [1, 5, 6, 7, 6, 5, 4, 2, 1]
    blocks = _blocks(x, rks, orthogonal, block_rks)
    Wr, sr = o.tt_recursive_sketch(x, rks, orthogonal=orthogonal, block_rks=block_rks, blocks=blocks)
    Wg, sg = ttcuda.tt_recursive_sketch(to_dev(x), rks, orthogonal=orthogonal, block_rks=block_rks,
                                        sketch_blocks=blocks)
    assert sg == sr
    for a, b in zip(Wg, Wr):
        assert a.shape == b.shape
        assert np.allclose(a, b, rtol=1e-11, atol=1e-11 * np.abs(b).max())


@pytest.mark.parametrize("orthogonal", [False, True])
def test_recursive_sketch_device_philox_matches_oracle(orthogonal):
    x = o.rand_tt((2,) * 10, 6, np.random.default_rng(12))
    rks = o.default_rank_heuristic(x)
    Wr, sr = o.tt_recursive_sketch(x, rks, orthogonal=orthogonal, seed=77, block_rks=16, rng_kind="philox")
    Wg, sg = ttcuda.tt_recursive_sketch(to_dev(x), rks, orthogonal=orthogonal, seed=77, block_rks=16)
    assert sg == sr
    for a, b in zip(Wg, Wr):
        assert np.allclose(a, b, rtol=1e-10, atol=1e-10 * np.abs(b).max())


def test_recursive_sketch_bf16_close():
    x = o.rand_tt((2,) * 10, 8, np.random.default_rng(13))
    rks = o.default_rank_heuristic(x)
    Wr, _ = o.tt_recursive_sketch(x, rks, orthogonal=False, seed=5, block_rks=32, rng_kind="philox")
    Wg, _ = ttcuda.tt_recursive_sketch(to_dev(x), rks, orthogonal=False, seed=5, block_rks=32, precision="bf16")
    for a, b in zip(Wg, Wr):
        assert np.linalg.norm(a - b) <= 3e-2 * np.linalg.norm(b)


@pytest.mark.parametrize("orthogonal", [False, True])
def test_ttrand_rounding_exact_reconstruction(orthogonal):
    """test/test_ttrand.jl:67-88 on the GPU: rank<=4 TT padded to 20 with 1e-8 noise."""
    g = np.random.default_rng(14)
    A_tt = o.rand_tt((2,) * 8, [1, 2, 4, 4, 4, 4, 4, 2, 1], g)
    A_pert = o.tt_up_rks(A_tt, 20, rng=g, eps_wn=1e-8)
    rks = [1, 2, 4, 6, 6, 6, 4, 2, 1]
    blocks = _blocks(A_pert, rks, orthogonal)
    ref = o.ttrand_rounding(A_pert, rks, orthogonal=orthogonal, blocks=blocks)
    got = ttcuda.ttrand_rounding(to_dev(A_pert), rks, orthogonal=orthogonal, sketch_blocks=blocks)
    assert got.ttv_rks == ref.ttv_rks
    assert got.ttv_ot == ref.ttv_ot
    assert rel(got, ref) < 1e-10
    assert rel_dense(got, A_pert) < 1e-6


def test_ttrand_rounding_device_sketch_and_default_heuristic():
    x = decaying_tt((2,) * 14, [1, 2, 4, 8, 16, 24, 24, 24, 24, 24, 16, 8, 4, 2, 1], seed=15)
    ref = o.ttrand_rounding(x, orthogonal=False, seed=99, block_rks=64, rng_kind="philox")
    got = ttcuda.ttrand_rounding(to_dev(x), orthogonal=False, seed=99, block_rks=64)
    assert got.ttv_rks == ref.ttv_rks
    assert rel(got, ref) < 1e-10
    assert rel(got, x) < 1e-11     # sketch rank covers the TT rank: exact up to rounding


def test_recursive_sketch_tf32_closer_than_bf16():
    """TF32 sketch contractions (FP32 operands, 10-bit mantissa on the tensor cores) track the
    FP64 sketch more closely than BF16 (7-bit)."""
    x = o.rand_tt((2,) * 10, 8, np.random.default_rng(13))
    rks = o.default_rank_heuristic(x)
    Wr, _ = o.tt_recursive_sketch(x, rks, orthogonal=False, seed=5, block_rks=32, rng_kind="philox")
    Wt, _ = ttcuda.tt_recursive_sketch(to_dev(x), rks, orthogonal=False, seed=5, block_rks=32, precision="tf32")
    Wb, _ = ttcuda.tt_recursive_sketch(to_dev(x), rks, orthogonal=False, seed=5, block_rks=32, precision="bf16")
    et = sum(np.linalg.norm(a - b) ** 2 for a, b in zip(Wt, Wr)) ** 0.5
    eb = sum(np.linalg.norm(a - b) ** 2 for a, b in zip(Wb, Wr)) ** 0.5
    nr = sum(np.linalg.norm(b) ** 2 for b in Wr) ** 0.5
    assert et <= 5e-3 * nr
    assert et < eb


def test_ttrand_rounding_tf32_sketch_accuracy():
    """TF32 sketch, FP64 range finder and projection: s >= r keeps the TT to 1e-8."""
    x = decaying_tt((2,) * 14, [1, 2, 4, 8, 16, 32, 32, 32, 32, 32, 16, 8, 4, 2, 1], seed=16)
    rks = o.default_rank_heuristic(x)
    got = ttcuda.ttrand_rounding(to_dev(x), rks, orthogonal=False, seed=3, block_rks=64, precision="tf32")
    assert got.ttv_rks == o.ttrand_rounding(x, rks, orthogonal=False, seed=3, block_rks=64).ttv_rks
    assert rel(got, x) < 1e-8


def test_ttrand_rounding_bf16_sketch_accuracy():
    """Mixed precision: BF16 sketch, FP64 range finder/projection; s >= r keeps 1e-8."""
    x = decaying_tt((2,) * 14, [1, 2, 4, 8, 16, 32, 32, 32, 32, 32, 16, 8, 4, 2, 1], seed=16)
    rks = o.default_rank_heuristic(x)
    got = ttcuda.ttrand_rounding(to_dev(x), rks, orthogonal=False, seed=3, block_rks=64, precision="bf16")
    assert got.ttv_rks == o.ttrand_rounding(x, rks, orthogonal=False, seed=3, block_rks=64).ttv_rks
    assert rel(got, x) < 1e-8


def test_ttrand_rounding_rmax_truncates():
    """ttrand_rounding(y, rmax) with a sketch below the TT rank (test/test_ttrand.jl:164-174 idea)."""
    g = np.random.default_rng(17)
    dims = (5,) * 8
    A = o.rand_tt(dims, 3, g, normalise=True)
    B = o.rand_tt(dims, 12, g, normalise=True)
    S = o.tt_add(A, o.tt_scale(1e-4, B))
    rks = [1] + [6] * 7 + [1]
    blocks = _blocks(S, rks, True)
    ref = o.ttrand_rounding(S, rks, blocks=blocks)
    got = ttcuda.ttrand_rounding(to_dev(S), rks, sketch_blocks=blocks)
    assert got.ttv_rks == ref.ttv_rks
    assert rel(got, ref) < 1e-9
    assert rel(got, A) < 1e-3


def test_lincomb_op_residual_rounding():
    g = np.random.default_rng(18)
    dims = (2,) * 6
    y1 = o.rand_tt(dims, 3, g)
    y2 = o.rand_tt(dims, 2, g)
    H = o.tto_decomp(g.standard_normal((2,) * 12))
    rks = [1, 6, 10, 12, 10, 6, 1]
    blocks = _blocks(y1, rks, False, block_rks=16)
    r1 = o.ttrand_rounding_lincomb([0.5, -2.0], [y1, y2], rks, orthogonal=False, block_rks=16, blocks=blocks)
    g1 = ttcuda.ttrand_rounding_lincomb([0.5, -2.0], [to_dev(y1), to_dev(y2)], rks, orthogonal=False, block_rks=16,
                                        sketch_blocks=blocks)
    assert g1.ttv_rks == r1.ttv_rks and rel(g1, r1) < 1e-10
    rks2 = [1] + [64] * 5 + [1]
    blocks2 = _blocks(y1, rks2, False, block_rks=64)
    r2 = o.ttrand_rounding_op([1.5, 0.25], H, [y1, y2], rks2, orthogonal=False, block_rks=64, blocks=blocks2)
    g2 = ttcuda.ttrand_rounding_op([1.5, 0.25], op_dev(H), [to_dev(y1), to_dev(y2)], rks2, orthogonal=False,
                                   block_rks=64, sketch_blocks=blocks2)
    assert g2.ttv_rks == r2.ttv_rks and rel(g2, r2) < 1e-10
    r3 = o.ttrand_rounding_residual(H, y1, y2, rks2, orthogonal=False, block_rks=64, blocks=blocks2)
    g3 = ttcuda.ttrand_rounding_residual(op_dev(H), to_dev(y1), to_dev(y2), rks2, orthogonal=False, block_rks=64,
                                         sketch_blocks=blocks2)
    assert g3.ttv_rks == r3.ttv_rks and rel(g3, r3) < 1e-10


def test_operator_sketch():
    g = np.random.default_rng(19)
    x = o.rand_tt((2,) * 6, 4, g)
    H = o.tto_decomp(g.standard_normal((2,) * 12))
    rks = [1, 7, 9, 9, 9, 7, 1]
    blocks = _blocks(x, rks, False, block_rks=4)
    Wr, sr = o.tt_recursive_sketch_op(H, x, rks, orthogonal=False, block_rks=4, blocks=blocks)
    Wg, sg = ttcuda.tt_recursive_sketch(to_dev(x), rks, H=op_dev(H), orthogonal=False, block_rks=4,
                                        sketch_blocks=blocks)
    assert sg == sr
    for a, b in zip(Wg, Wr):
        assert np.allclose(a, b, rtol=1e-10, atol=1e-10 * np.abs(b).max())


# ------------------------------------------------------------------ apply, dot, environments
def test_mpo_apply_hubbard():
    h, V = mo.hubbard_1D(4, t=1.0, U=4.0)
    H = mo.hV_to_mpo(h, V, (2,) * 8)
    x = o.rand_tt((2,) * 8, 6, np.random.default_rng(20))
    ref = o.tto_apply(H, x)
    got = ttcuda.mpo_apply(op_dev(H), to_dev(x))
    assert got.ttv_rks == ref.ttv_rks
    for a, b in zip(got.ttv_vec, ref.ttv_vec):
        assert np.array_equal(a, b) or np.allclose(a, b, rtol=1e-14, atol=1e-14)


def test_dot_partial_contraction_dot_operator():
    g = np.random.default_rng(21)
    dims = (2,) * 7
    A = o.rand_tt(dims, 5, g)
    B = o.rand_tt(dims, 3, g)
    assert math.isclose(ttcuda.dot(to_dev(A), to_dev(B)), o.dot(A, B), rel_tol=1e-12)
    for rev in (True, False):
        Wg = ttcuda.partial_contraction(to_dev(A), to_dev(B), reverse=rev)
        Wr = o.partial_contraction(A, B, reverse=rev)
        for a, b in zip(Wg, Wr):
            assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(b).max()))
    H = o.tto_decomp(g.standard_normal((2,) * 14))
    assert math.isclose(ttcuda.dot_operator(to_dev(A), op_dev(H), to_dev(B)), o.dot_operator(A, H, B), rel_tol=1e-10)


def test_add_scale():
    g = np.random.default_rng(22)
    x = o.rand_tt((3,) * 5, 3, g)
    y = o.rand_tt((3,) * 5, 2, g)
    s = ttcuda.tt_add(to_dev(x), to_dev(y))
    assert s.ttv_rks == o.tt_add(x, y).ttv_rks
    assert rel_dense(s, o.tt_add(x, y)) < 1e-14
    z = ttcuda.tt_scale(-2.5, to_dev(x))
    assert rel_dense(z, o.tt_scale(-2.5, x)) < 1e-14


def test_rayleigh_grad_vs_oracle_and_fd():
    h, V = mo.hubbard_1D(3, t=1.0, U=8.0)
    H = mo.hV_to_mpo(h, V, (2,) * 6)
    x = o.rand_tt((2,) * 6, 4, np.random.default_rng(23))
    Rr, Gr = o.rayleigh_value_and_grad(H, x)
    for ck in (1, 2, 4):
        Rg, Gg = ttcuda.rayleigh_grad(op_dev(H), to_dev(x), ckpt_every=ck)
        assert math.isclose(Rg, Rr, rel_tol=1e-12)
        for a, b in zip(Gg, Gr):
            assert np.allclose(a, b, rtol=1e-10, atol=1e-12 * max(1.0, np.abs(b).max()))


# ------------------------------------------------------------------ batched device rounding
def test_batched_round_det_uneven_ranks():
    g = np.random.default_rng(24)
    dims = (2,) * 12
    tts = []
    for i in range(5):
        r = [1] + [int(v) for v in g.integers(2, 24, size=11)] + [1]
        tts.append(decaying_tt(dims, o.r_and_d_to_rks(r, dims, rmax=max(r)), seed=100 + i, decay_per=3.0))
    xb = ttcuda.DeviceBatch.from_tts([to_dev(t) for t in tts])
    caps = [o.r_and_d_to_rks(t.ttv_rks, dims) for t in tts]
    yb = ttcuda.DeviceBatch(dims, [[max(a, 1) for a in c] for c in caps])
    for rep in range(2):          # second run replays the captured CUDA graph
        xb.round_det(yb, tol=1e-6)
        outs = yb.download()
        for t, got in zip(tts, outs):
            ref = o.tt_rounding(t, tol=1e-6)
            assert got.ttv_rks == ref.ttv_rks
            assert rel(got, ref) < 1e-10


def test_repeated_rounds_reuse_their_plans():
    """A repeated rounding with the same shapes reuses its execution plan (replayed as a CUDA
    graph from the second run on) and gives bitwise the same result, for the deterministic
    and the randomized rounding; new input values with the same ranks reuse it too."""
    ctx = ttcuda.get_context()
    dims = (2,) * 10
    tts = [decaying_tt(dims, o.r_and_d_to_rks([1] + [10] * 9 + [1], dims), seed=400 + i, decay_per=2.0)
           for i in range(3)]
    xb = ttcuda.DeviceBatch.from_tts([to_dev(t) for t in tts])
    rks = o.default_rank_heuristic(tts)
    cap = ttcuda._rand_out_caps(dims, ttcuda._sketch_ranks(dims, rks, 64))
    yr = ttcuda.DeviceBatch(dims, [cap] * 3)
    yd = ttcuda.DeviceBatch(dims, [t.ttv_rks for t in tts])
    runs = {"det": lambda: xb.round_det(yd, tol=1e-6),
            "rand": lambda: xb.round_rand(yr, rks, seed=9, block_rks=64, precision="bf16", after_tol=1e-6)}
    outs = {"det": yd, "rand": yr}
    for name, run in runs.items():
        run()
        first = [np.concatenate([c.ravel() for c in t.ttv_vec]) for t in outs[name].download()]
        built = ctx.stats()["plans_built"]
        for _ in range(3):
            run()
            again = [np.concatenate([c.ravel() for c in t.ttv_vec]) for t in outs[name].download()]
            assert all(np.array_equal(a, b) for a, b in zip(first, again)), name
        assert ctx.stats()["plans_built"] == built, name
    # same ranks, other values: same plans, results of the new input
    tts2 = [decaying_tt(dims, t.ttv_rks, seed=500 + i, decay_per=2.0) for i, t in enumerate(tts)]
    built = ctx.stats()["plans_built"]
    xb.upload([to_dev(t) for t in tts2])
    xb.round_det(yd, tol=1e-6)
    assert ctx.stats()["plans_built"] == built
    for t, got in zip(tts2, yd.download()):
        ref = o.tt_rounding(t, tol=1e-6)
        assert got.ttv_rks == ref.ttv_rks
        assert rel(got, ref) < 1e-10


def test_page_locked_upload_and_download_match_staged():
    """Cores in page-locked host memory skip the staging copy (uploads by DMA, downloads written
    by the layout kernel); the results equal those through the staging buffer."""
    dims = (2, 3, 2, 4, 2, 3)
    tts = [decaying_tt(dims, o.r_and_d_to_rks([1, 2, 5, 7, 6, 3, 1], dims), seed=600 + i, decay_per=2.0)
           for i in range(4)]
    dev = [to_dev(t) for t in tts]
    xs = ttcuda.DeviceBatch.from_tts(dev)
    xp = ttcuda.DeviceBatch.from_tts([ttcuda.pinned_tt(t) for t in dev])
    for a, b in zip(xs.download(), xp.download(reuse=True)):
        assert a.ttv_rks == b.ttv_rks
        assert all(np.array_equal(u, v) for u, v in zip(a.ttv_vec, b.ttv_vec))
    ys = ttcuda.DeviceBatch(dims, [t.ttv_rks for t in tts])
    xp.round_det(ys, tol=1e-4)
    staged, pinned = ys.download(), ys.download(reuse=True)
    for t, a, b in zip(tts, staged, pinned):
        assert a.ttv_rks == b.ttv_rks == o.tt_rounding(t, tol=1e-4).ttv_rks
        assert all(np.array_equal(u, v) for u, v in zip(a.ttv_vec, b.ttv_vec))


def test_batched_round_rand_then_svd():
    dims = (2,) * 10
    tts = [decaying_tt(dims, o.r_and_d_to_rks([1] + [12] * 9 + [1], dims), seed=200 + i, decay_per=2.0)
           for i in range(3)]
    rks = o.default_rank_heuristic(tts)
    xb = ttcuda.DeviceBatch.from_tts([to_dev(t) for t in tts])
    s = ttcuda._sketch_ranks(dims, rks, 64)
    cap = ttcuda._rand_out_caps(dims, s)
    yb = ttcuda.DeviceBatch(dims, [cap] * 3)
    for prec in ("fp64", "bf16", "tf32"):
        xb.round_rand(yb, rks, orthogonal=False, seed=4, block_rks=64, precision=prec, after_tol=1e-5)
        for t, got in zip(tts, yb.download()):
            ref = o.tt_rounding(o.ttrand_rounding(t, rks, orthogonal=False, seed=4, block_rks=64), tol=1e-5)
            assert got.ttv_rks == ref.ttv_rks
            assert rel(got, ref) < (1e-10 if prec == "fp64" else 1e-7)


def _range_finder_forms(dims, rep, s):
    """Forms the randomized sweep's range finder takes per bond (F: the sketch rank s is below
    both dimensions of y_k's unfolding; T: r_{k+1} is the smallest; W: n e_k is)."""
    e, forms = 1, []
    for k in range(len(dims) - 1):
        m, c = dims[k] * e, rep[k + 1]
        q = min(m, c, s[k + 1])
        forms.append("F" if q == s[k + 1] else ("T" if q == c else "W"))
        e = q
    return forms


@pytest.mark.parametrize("prec", ["fp64", "bf16"])
def test_batched_round_rand_then_svd_mixed_levels(prec):
    """A batch whose range finders take all three forms.  With the SVD sweep following, the
    compressing levels (F) read the sketch and the others take the reduced forms that keep only
    range(Q).  x = t + t/2 represents t at twice its ranks, and the sketch ranks of the F levels
    cover t's ranks, so the result is t rounded, whatever the sketch's precision."""
    dims = (2,) * 10
    rks = [1, 2, 4, 8, 8, 16, 16, 16, 8, 4, 1]
    block = 8
    s = ttcuda._sketch_ranks(dims, rks, block)
    g = np.random.default_rng(77)
    xs, forms = [], set()
    for r in (5, 6, 3):
        t = o.rand_tt(dims, o.r_and_d_to_rks([1] + [r] * 9 + [1], dims), g)
        x = o.tt_add(t, o.tt_scale(0.5, t))
        forms.update(_range_finder_forms(dims, x.ttv_rks, s))
        xs.append(x)
    assert forms == {"F", "T", "W"}
    xb = ttcuda.DeviceBatch.from_tts([to_dev(x) for x in xs])
    yb = ttcuda.DeviceBatch(dims, [ttcuda._rand_out_caps(dims, s)] * len(xs))
    xb.round_rand(yb, rks, orthogonal=False, seed=21, block_rks=block, precision=prec, after_tol=1e-10)
    for x, got in zip(xs, yb.download()):
        ref = o.tt_rounding(o.ttrand_rounding(x, rks, orthogonal=False, seed=21, block_rks=block), tol=1e-10)
        assert got.ttv_rks == ref.ttv_rks == o.tt_rounding(x, tol=1e-10).ttv_rks
        assert rel(got, ref) < 1e-10


# ------------------------------------------------------ mixed precision on non-minimal TTs
@pytest.mark.parametrize("block", [None, 8, 16, 64])
@pytest.mark.parametrize("orthogonal", [False, True])
def test_ttrand_bf16_sum_of_tts_exact(block, orthogonal):
    """Sum of three rank-4 TTs (ranks not re-clamped, so the right interfaces of the last
    bonds are rank deficient): the BF16 sketch still reconstructs the TT to FP64 accuracy,
    because rank-deficient levels are contracted in FP64."""
    g = np.random.default_rng(5)
    dims = (2,) * 10
    x = None
    for _ in range(3):
        t = o.rand_tt(dims, [1] + [4] * 9 + [1], g)
        x = t if x is None else o.tt_add(x, t)
    rks = [1] + [16] * 9 + [1]
    got = ttcuda.ttrand_rounding(to_dev(x), rks, orthogonal=orthogonal, seed=11, precision="bf16", block_rks=block)
    ref = o.ttrand_rounding(x, rks, orthogonal=orthogonal, seed=11, block_rks=block)
    assert got.ttv_rks == ref.ttv_rks
    assert rel(got, x) < 1e-11


def test_batched_round_rand_bf16_iid_ranks():
    """Independently drawn interior ranks (bonds wider than n times a neighbour), decaying
    spectrum: mixed-precision randomized rounding plus the FP64 SVD sweep meets the FP64
    deterministic rounding at tol 1e-8 with identical truncation ranks."""
    g = np.random.default_rng(31)
    dims = (2,) * 16
    tts = []
    for i in range(4):
        r = [1] + [int(v) for v in g.integers(4, 48, size=15)] + [1]
        tts.append(decaying_tt(dims, o.r_and_d_to_rks(r, dims, rmax=max(r)), seed=300 + i, decay_per=4.0))
    rks = o.default_rank_heuristic(tts)
    xb = ttcuda.DeviceBatch.from_tts([to_dev(t) for t in tts])
    block = max(rks)
    s = ttcuda._sketch_ranks(dims, rks, block)
    yb = ttcuda.DeviceBatch(dims, [ttcuda._rand_out_caps(dims, s)] * len(tts))
    xb.round_rand(yb, rks, orthogonal=False, seed=9, block_rks=block, precision="bf16", after_tol=1e-8)
    for t, got in zip(tts, yb.download()):
        ref = o.tt_rounding(t, tol=1e-8)
        assert got.ttv_rks == ref.ttv_rks
        assert rel(got, ref) < 1e-8
        # floor() keeps the discarded weight of each bond below tol^2 ||x||^2 (src/tt_rounding.jl:298-315)
        assert rel(got, t) < math.sqrt(len(dims) - 1) * 1e-8


# ------------------------------------------------------------------ full configuration sizes
def test_config2_full_size_operator_rounding_consistency():
    """Config 2 at full size: 1D Hubbard MPO (16 sites, 32 spin-orbitals, t=1, U=4) applied to a
    rank-128 TT, Gaussian sketch of rank 138 (block_rks=138: one block).  Rounding A y without
    forming it (operator sketch) and forming A y first then rounding use the same sketch, so
    they agree to FP64 rounding; <y|A|y> from the operator contraction matches dot(y, A y)."""
    h, V = mo.hubbard_1D(16, t=1.0, U=4.0)
    H = mo.hV_to_mpo(h, V, (2,) * 32)
    y = o.rand_tt((2,) * 32, 128, np.random.default_rng(40), normalise=True)
    rks = [1] + [138] * 31 + [1]
    z_op = ttcuda.ttrand_rounding_op([1.0], op_dev(H), [to_dev(y)], rks, orthogonal=False, seed=5, block_rks=138)
    Hy = ttcuda.mpo_apply(op_dev(H), to_dev(y))
    assert Hy.ttv_rks == [a * b for a, b in zip(H.tto_rks, y.ttv_rks)]
    z_apply = ttcuda.ttrand_rounding(Hy, rks, orthogonal=False, seed=5, block_rks=138)
    assert z_op.ttv_rks == z_apply.ttv_rks
    assert rel(z_op, z_apply) < 1e-10
    e1 = ttcuda.dot_operator(to_dev(y), op_dev(H), to_dev(y))
    e2 = ttcuda.dot(to_dev(y), Hy)
    assert math.isclose(e1, e2, rel_tol=1e-10)


def test_config4_full_size_gradient_finite_differences():
    """Config 4 at full size: 4x4 open-boundary Hubbard lattice (t=1, U=8) in snake ordering,
    x of rank 256, environments checkpointed every 4 sites.  The value matches
    <x|H|x>/<x|x> from the contractions and the gradient matches central finite differences
    (h = 1e-6) along 16 seeded random directions in core space."""
    h, V = mo.hubbard_2D(4, 4, t=1.0, U=8.0, w_pbc=False, L_pbc=False)
    s = mo.snake_permutation(4, 4)
    H = op_dev(mo.hV_to_mpo(h[np.ix_(s, s)], V[np.ix_(s, s, s, s)], (2,) * 32))
    g = np.random.default_rng(41)
    x = o.rand_tt((2,) * 32, 256, g, normalise=True)
    X = to_dev(x)
    R, G = ttcuda.rayleigh_grad(H, X, ckpt_every=4)

    def rq(cores):
        t = ttcuda.TTvector(x.N, cores, x.ttv_dims, x.ttv_rks, [0] * x.N)
        return ttcuda.dot_operator(t, H, t) / ttcuda.dot(t, t)

    assert math.isclose(R, rq([c.copy() for c in x.ttv_vec]), rel_tol=1e-10)
    hstep = 1e-6
    for _ in range(16):
        d = [g.standard_normal(c.shape) for c in x.ttv_vec]
        nd = math.sqrt(sum(float(np.sum(v * v)) for v in d))
        d = [v / nd for v in d]
        fp = rq([np.asfortranarray(c + hstep * v) for c, v in zip(x.ttv_vec, d)])
        fm = rq([np.asfortranarray(c - hstep * v) for c, v in zip(x.ttv_vec, d)])
        fd = (fp - fm) / (2 * hstep)
        an = sum(float(np.sum(np.asarray(gk).reshape(v.shape, order="F") * v)) for gk, v in zip(G, d))
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-3 * abs(R)), (fd, an)


def test_batch_download_reuse_matches_fresh_buffers():
    """DeviceBatch.download(reuse=True) writes into the same host buffers on every call and
    returns what a fresh download returns."""
    dims = (2,) * 10
    tts = [decaying_tt(dims, o.r_and_d_to_rks([1] + [10] * 9 + [1], dims), seed=500 + i, decay_per=3.0)
           for i in range(3)]
    xb = ttcuda.DeviceBatch.from_tts([to_dev(t) for t in tts])
    yb = ttcuda.DeviceBatch(dims, [t.ttv_rks for t in tts])
    xb.round_det(yb, tol=1e-4)
    fresh = yb.download()
    a = yb.download(reuse=True)
    b = yb.download(reuse=True)
    for f, u, v in zip(fresh, a, b):
        assert f.ttv_rks == u.ttv_rks == v.ttv_rks
        for c1, c2, c3 in zip(f.ttv_vec, u.ttv_vec, v.ttv_vec):
            assert np.array_equal(c1, c2) and np.array_equal(c2, c3)
            assert np.shares_memory(c2, c3)
