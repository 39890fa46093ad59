"""The reference's own property tests, re-expressed against the FP64 oracle.

They pin the oracle (the reference ships no golden vectors): dense equality at toy
sizes, exact reconstruction, partial_contraction == dot, rank heuristics.  Sources:
test/test_tt_tools.jl and test/test_ttrand.jl of the reference, with seeded inputs.
"""
import numpy as np
import pytest

from oracle import tt_oracle as o
from oracle import models_oracle as mo


def rng(seed=0):
    return np.random.default_rng(seed)


def test_tt_up_rks():
    """test/test_tt_tools.jl:5-14"""
    g = rng(1)
    x = g.standard_normal((4, 4, 4, 4))
    x_tt = o.ttv_decomp(x, tol=0.1)
    x = o.ttv_to_tensor(x_tt)
    y_tt = o.tt_up_rks(x_tt, 20)
    assert np.allclose(x, o.ttv_to_tensor(y_tt), atol=1e-10)
    z_tt = o.tt_up_rks(x_tt, 20, rng=g, eps_wn=1e-10)
    assert np.allclose(x, o.ttv_to_tensor(z_tt), atol=1e-6)


def test_tt_operations_dense():
    """test/test_tt_tools.jl:16-46"""
    g = rng(2)
    n, d = 3, 3
    L = g.standard_normal((n,) * 6)
    S = g.standard_normal((n,) * 6)
    L_tto, S_tto = o.tto_decomp(L), o.tto_decomp(S)
    x = g.standard_normal((n,) * 3)
    y = g.standard_normal((n,) * 3)
    x_tt, y_tt = o.ttv_decomp(x), o.ttv_decomp(y)
    a = float(g.standard_normal())
    assert np.allclose(a * x, o.ttv_to_tensor(o.tt_scale(a, x_tt)))
    z_tt = o.tt_add(x_tt, y_tt)
    assert np.allclose(o.ttv_to_tensor(z_tt), x + y)
    assert np.isclose(x.reshape(-1, order="F") @ (x + y).reshape(-1, order="F"), o.dot(x_tt, z_tt))
    assert np.allclose(o.tto_to_tensor(o.tto_add(L_tto, S_tto)), L + S)
    Lm = L.reshape(n ** d, -1, order="F")
    z = Lm @ x.reshape(-1, order="F")
    assert np.allclose(o.ttv_to_tensor(o.tto_apply(L_tto, x_tt)).reshape(-1, order="F"), z)
    A = Lm @ S.reshape(n ** d, -1, order="F")
    assert np.allclose(o.tto_to_tensor(o.tto_mul(L_tto, S_tto)).reshape(n ** d, -1, order="F"), A)


def test_orthogonalize():
    """test/test_tt_tools.jl:48-57 (every interior core checked, not one random one)."""
    dims = (2,) * 8
    rks = [1, 2, 4, 8, 8, 8, 4, 2, 1]
    x_tt = o.rand_tt(dims, rks, rng(3))
    y_tt = o.orthogonalize(x_tt)
    for i in range(1, 8):
        c = y_tt.ttv_vec[i]
        G = sum(c[k] @ c[k].T for k in range(dims[i]))
        assert np.allclose(G, np.eye(rks[i]))
        assert c.shape == (dims[i], rks[i], rks[i + 1])
    assert np.allclose(o.ttv_to_tensor(x_tt), o.ttv_to_tensor(y_tt))
    # left-orthogonal root at N
    z = o.orthogonalize(x_tt, i=8)
    for i in range(7):
        c = z.ttv_vec[i]
        assert np.allclose(sum(c[k].T @ c[k] for k in range(2)), np.eye(c.shape[2]))
    assert np.allclose(o.ttv_to_tensor(x_tt), o.ttv_to_tensor(z))


def test_tt_rounding_dense():
    """test/test_tt_tools.jl:59-71"""
    g = rng(4)
    n, d = 5, 3
    L = g.standard_normal((n,) * 6)
    x = g.standard_normal((n,) * 3)
    y = L.reshape(n ** d, -1, order="F") @ x.reshape(-1, order="F")
    y_tt = o.tto_apply(o.tto_decomp(L), o.ttv_decomp(x))
    assert np.allclose(o.ttv_to_tensor(o.tt_rounding(y_tt)).reshape(-1, order="F"), y)
    assert np.isclose(o.dot(o.ttv_decomp(x), y_tt), x.reshape(-1, order="F") @ y)
    # right-direction variant represents the same tensor
    assert np.allclose(o.ttv_to_tensor(o.tt_rounding(y_tt, direction="right")).reshape(-1, order="F"), y)


def test_partial_contraction():
    """test/test_ttrand.jl:35-46"""
    dims = (2, 2, 2, 2)
    rks = [1, 4, 4, 4, 1]
    A = o.rand_tt(dims, rks, rng(5))
    B = o.rand_tt(dims, rks, rng(6))
    W = o.partial_contraction(A, B)
    assert np.isclose(W[0][0, 0], o.dot(A, B))
    W = o.partial_contraction(A, B, reverse=False)
    assert np.isclose(W[-1][0, 0], o.dot(A, B))


def test_default_rank_heuristic():
    """test/test_ttrand.jl:48-65"""
    dims = (3, 3, 3, 3)
    A = o.rand_tt(dims, [1, 3, 5, 4, 1], rng(7), stable=False)
    h = o.default_rank_heuristic(A)
    assert len(h) == 5 and h[0] == 1 and h[-1] == 1
    assert h == [1, 3 + 3, 5 + 3, 4 + 3, 1]
    B = o.rand_tt(dims, [1, 2, 3, 2, 1], rng(8), stable=False)
    C = o.rand_tt(dims, [1, 4, 6, 3, 1], rng(9), stable=False)
    hv = o.default_rank_heuristic([A, B, C])
    assert hv[0] == 1 and hv[-1] == 1
    assert all(v >= 4 for v in hv[1:-1])


def test_tt_recursive_sketch_shapes():
    """test/test_ttrand.jl:5-33"""
    dims = (3, 3, 3, 3)
    A = o.rand_tt(dims, [1, 3, 3, 3, 1], rng(10))
    W, srk = o.tt_recursive_sketch(A, [1, 2, 2, 2, 1], seed=1234)
    assert len(W) == 5 and len(srk) == 5 and srk[0] >= 1
    for k in range(5):
        assert W[k].shape == (A.ttv_rks[k], srk[k])
    W2, srk2 = o.tt_recursive_sketch(A, 4, seed=1234)
    assert len(W2) == 5 and all(s >= 1 for s in srk2)


@pytest.mark.parametrize("orthogonal", [True, False])
def test_ttrand_rounding_exact(orthogonal):
    """test/test_ttrand.jl:67-88: rank<=4 TT padded to rank 20 with 1e-8 noise is recovered."""
    g = rng(11)
    dims = (2,) * 8
    A_tt = o.rand_tt(dims, [1, 2, 4, 4, 4, 4, 4, 2, 1], g)
    A_pert = o.tt_up_rks(A_tt, 20, rng=g, eps_wn=1e-8)
    A = o.ttv_to_tensor(A_pert)
    R = o.ttrand_rounding(A_pert, [1, 2, 4, 6, 6, 6, 4, 2, 1], orthogonal=orthogonal)
    assert np.allclose(A, o.ttv_to_tensor(R), atol=1e-6)
    R1 = o.ttrand_rounding(A_pert, [1, 2, 4, 6, 6, 6, 4, 2, 1], seed=9999, orthogonal=orthogonal)
    R2 = o.ttrand_rounding(A_pert, [1, 2, 4, 6, 6, 6, 4, 2, 1], seed=9999, orthogonal=orthogonal)
    assert np.allclose(o.ttv_to_tensor(R1), o.ttv_to_tensor(R2))
    Ra = o.ttrand_rounding(A_pert, orthogonal=orthogonal)
    assert np.allclose(A, o.ttv_to_tensor(Ra), atol=1e-6)


def test_tt_sum_rand_rounding():
    """test/test_ttrand.jl:164-174 (d=10, n=50 as in the reference)."""
    g = rng(12)
    d, n, r = 10, 50, 5
    dims = (n,) * d
    A = o.rand_tt(dims, r, g, normalise=True)
    B = o.rand_tt(dims, 20 * r, g, normalise=True)
    eps = 1e-4
    S = o.tt_add(A, o.tt_scale(eps, B))
    Ar = o.ttrand_rounding(S, 10)
    assert o.norm(o.tt_sub(A, Ar)) < 1e-3 * o.norm(A)
    As = o.tt_rounding(S, tol=eps)
    assert o.norm(o.tt_sub(A, As)) < 1e-3 * o.norm(A)


def test_lincomb_and_operator_rounding_dense():
    """Linear-combination and operator-aware rounding equal the dense sums
    (src/tt_randtools.jl:223-361, src/tt_randtools.jl:169-214)."""
    g = rng(13)
    dims = (2,) * 6
    y1 = o.rand_tt(dims, 3, g)
    y2 = o.rand_tt(dims, 2, g)
    Hd = g.standard_normal((2,) * 12)
    H = o.tto_decomp(Hd)
    Hm = Hd.reshape(64, 64, order="F")
    t1 = o.ttv_to_tensor(y1).reshape(-1, order="F")
    t2 = o.ttv_to_tensor(y2).reshape(-1, order="F")
    R = o.ttrand_rounding_lincomb([0.5, -2.0], [y1, y2], 8)
    assert np.allclose(o.ttv_to_tensor(R).reshape(-1, order="F"), 0.5 * t1 - 2.0 * t2)
    R = o.ttrand_rounding_op([1.5, 0.25], H, [y1, y2], 64)
    assert np.allclose(o.ttv_to_tensor(R).reshape(-1, order="F"), 1.5 * Hm @ t1 + 0.25 * t2)
    R = o.ttrand_rounding_residual(H, y1, y2, 64)
    assert np.allclose(o.ttv_to_tensor(R).reshape(-1, order="F"), Hm @ t1 - t2)
    # operator sketch equals the sketch of the materialised product (same blocks)
    Hy = o.tto_apply(H, y1)
    rks = [1] + [5] * 5 + [1]
    Wop, s1 = o.tt_recursive_sketch_op(H, y1, rks, orthogonal=False, block_rks=8)
    Wm, s2 = o.tt_recursive_sketch(Hy, rks, orthogonal=False, block_rks=8)
    assert s1 == s2
    for k in range(7):
        # H y rank index is (H fastest, y); the operator sketch is (y fastest, H)
        r, R_ = y1.ttv_rks[k], H.tto_rks[k]
        a = Wop[k].reshape(r, R_, -1, order="F")
        b = Wm[k].reshape(R_, r, -1, order="F").transpose(1, 0, 2)
        assert np.allclose(a, b)


def test_dot_operator_and_gradient():
    g = rng(14)
    dims = (2,) * 5
    x = o.rand_tt(dims, 3, g)
    Hd = g.standard_normal((2,) * 10)
    Hm = Hd.reshape(32, 32, order="F")
    Hm = Hm + Hm.T
    H = o.tto_decomp(Hm.reshape((2,) * 10, order="F"))
    xv = o.ttv_to_tensor(x).reshape(-1, order="F")
    assert np.isclose(o.dot_operator(x, H, x), xv @ Hm @ xv)
    xo = o.orthogonalize(x, i=3)
    assert np.isclose(o.dot_operator(xo, H, xo), xv @ Hm @ xv)
    R, grads = o.rayleigh_value_and_grad(H, x)
    assert np.isclose(R, xv @ Hm @ xv / (xv @ xv))
    # central finite differences along a random direction of core 2
    D = g.standard_normal(x.ttv_vec[2].shape)
    h = 1e-6
    xp, xm = x.copy(), x.copy()
    xp.ttv_vec[2] = x.ttv_vec[2] + h * D
    xm.ttv_vec[2] = x.ttv_vec[2] - h * D
    fd = (o.rayleigh_value_and_grad(H, xp)[0] - o.rayleigh_value_and_grad(H, xm)[0]) / (2 * h)
    assert np.isclose(fd, np.sum(grads[2] * D), rtol=1e-5, atol=1e-8)


def test_floor_rule():
    """src/tt_rounding.jl:297-315 edge cases."""
    s = np.array([1.0, 0.5, 0.25, 1e-9, 1e-10])
    assert o.floor_rank(s, 0.0) == 5
    assert o.floor_rank(s, 1e-8) == 3
    assert o.floor_rank(s, 1e-12) == 5
    assert o.floor_rank(np.array([1.0, 1.0 - 1e-6, 1e-3]), 0.5) == 2   # degenerate extension
    assert o.floor_rank(np.array([3.0]), 2.0) == 1


def test_philox_known_answer():
    """Philox4x32-10 known-answer vectors (Random123 kat_vectors: zero and all-ones inputs)."""
    c = np.zeros((1, 4), dtype=np.uint64)
    out = o.philox4x32_10(c, 0, 0)[0]
    assert [int(v) for v in out] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    c = np.full((1, 4), 0xFFFFFFFF, dtype=np.uint64)
    out = o.philox4x32_10(c, 0xFFFFFFFF, 0xFFFFFFFF)[0]
    assert [int(v) for v in out] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]


def test_hubbard_mpo_dense_small():
    """hV_to_mpo on a 2-site Hubbard chain equals the dense second-quantised H
    (cf. test/test_models.jl:6-22 for one_body_mpo)."""
    h, V = mo.hubbard_1D(2, t=1.0, U=4.0)
    dims = (2,) * 4
    H = mo.hV_to_mpo(h, V, dims)
    Hd = o.tto_to_tensor(H).reshape(16, 16, order="F")
    # dense reference from the same creation/annihilation products
    def dense(A):
        return o.tto_to_tensor(A).reshape(16, 16, order="F")
    c = [dense(mo.tto_creation(i, dims)) for i in range(1, 5)]
    a = [dense(mo.tto_annihilation(i, dims)) for i in range(1, 5)]
    ref = np.zeros((16, 16))
    for i in range(4):
        for j in range(4):
            if abs(h[i, j]) > 0 and i <= j:
                ref += h[i, j] * (c[i] @ a[j] + (c[j] @ a[i] if i < j else 0))
    for (i1, i2, i3, i4) in mo._nonzero_indices(V):
        if (i1, i2) < (i4, i3):
            v = V[i1 - 1, i2 - 1, i3 - 1, i4 - 1]
            ref += v * (c[i1 - 1] @ c[i2 - 1] @ a[i3 - 1] @ a[i4 - 1] + c[i4 - 1] @ c[i3 - 1] @ a[i2 - 1] @ a[i1 - 1])
    assert np.allclose(Hd, ref)
    assert np.allclose(Hd, Hd.T)
