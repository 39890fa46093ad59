"""The Krylov callers' oracle (oracle/krylov_oracle.py) on CPU: its sketches against the recursive
sketch, the stored-sketch expansion step against the recomputing form the GPU mirror uses, and
the eigensolvers against the dense eigenproblem of a small Hubbard chain."""
import math

import numpy as np
import pytest

from oracle import krylov_oracle as ko
from oracle import models_oracle as mo
from oracle import tt_oracle as o


@pytest.fixture(scope="module")
def hubbard3():
    h, V = mo.hubbard_1D(3, t=0.1, U=0.4)
    dims = (2,) * 6
    H = mo.hV_to_mpo(h, V, dims)
    D = o.tto_to_tensor(H).reshape(64, 64, order="F")
    ev = np.linalg.eigvalsh((D + D.T) / 2)
    b0 = o.rand_tt(dims, 4, np.random.default_rng(5), normalise=True)
    return H, ev, b0


@pytest.mark.parametrize("s,block", [(20, 8), (7, 3), (64, None)])
def test_tt_sketch_is_recursive_sketch_boundary(hubbard3, s, block):
    H, _, b0 = hubbard3
    N = b0.N
    b = o.reverse_block_ranks(b0.ttv_dims, N, N if block is None else block)
    p = math.ceil(s / b[0])
    rks = [bk * p for bk in b[:N]] + [1]
    sk, sa = ko.tt_sketch(b0, s, None, True, 77, block)
    W, srk = o.tt_recursive_sketch(b0, rks, True, 77, block)
    assert sa == srk[0] == b[0] * p
    assert np.array_equal(sk, W[0].ravel(order="F"))
    sko, _ = ko.tt_sketch(b0, s, H, True, 77, block)
    Wo, _ = o.tt_recursive_sketch_op(H, b0, rks, True, 77, block)
    assert np.array_equal(sko, Wo[0].ravel(order="F"))


def test_combined_sketch_extends_with_seed_plus_one(hubbard3):
    _, _, b0 = hubbard3
    sk, W, srk = ko.tt_combined_sketch(b0, 4, 30, None, True, 11, 2)
    rks = [4] * 6 + [1]
    rks[0] = max(rks[0], min(30, rks[1]))
    Wr, sr = o.tt_recursive_sketch(b0, rks, True, 11, 2)
    ex, _ = ko.tt_sketch(b0, 30 - sr[0], None, True, 12, 2)
    tot = sr[0] + len(ex)
    want = np.concatenate([math.sqrt(sr[0] / tot) * Wr[0].ravel(order="F"), math.sqrt(len(ex) / tot) * ex])
    assert len(sk) == tot >= 30 and np.allclose(sk, want, rtol=0, atol=1e-15)
    assert srk[0] == 1 and W[0].shape == (1, 1)
    for k in range(1, 7):
        assert np.array_equal(W[k], Wr[k])


def test_expand_basis_stored_sketches_equal_recomputed(hubbard3):
    """The reference's step reuses the window's stored sketches; rounding H b - h b with the
    sketches recomputed (what the GPU mirror does) gives the same vector."""
    H, _, b0 = hubbard3
    rmax, s = 8, 24
    sk0, W1, _ = ko.tt_combined_sketch(b0, 2 * rmax, s, None, True, 1234, 8)
    beta = np.linalg.norm(sk0)
    ko._rescale_upto_root(W1, b0, beta)
    B0 = o.tt_scale(1 / beta, b0)
    Bw, Ww, Sw = [B0], [W1], [sk0 / beta]
    for step in range(3):
        prev = list(Bw)
        skw = np.column_stack(Sw)
        bn, skb, skHb = ko.expand_basis(H, Bw, Ww, Sw, rmax, len(sk0), True, 8, 1234, 2)
        h = np.linalg.lstsq(skw, skHb, rcond=None)[0]
        y = o.ttrand_rounding_op([1.0] + list(-h), H, [prev[-1]] + prev, [2 * rmax] * 6 + [1], True, 1234, 8)
        y = o.tt_rounding(y, rmax=rmax)
        y = o.tt_scale(1 / np.linalg.norm(ko.tt_combined_sketch(y, 2 * rmax, len(sk0), None, True, 1234, 8)[0]), y)
        assert bn.ttv_rks == y.ttv_rks
        assert o.rel_error(bn, y) < 1e-12
        assert abs(np.linalg.norm(skb) - 1) < 1e-14
    assert len(Bw) == len(Ww) == len(Sw) == 2          # k_trunc window


def test_sketched_rayleigh_ritz_variational_and_converging(hubbard3):
    H, ev, b0 = hubbard3
    e, psi, hist = ko.sketched_rayleigh_ritz(H, b0, 12, 8)
    assert [h["iter"] for h in hist] == list(range(1, 13))
    assert all(h["e_true"] >= ev[0] - 1e-12 for h in hist if np.isfinite(h["e_true"]))
    assert hist[-1]["e_true"] < hist[0]["e_true"]
    assert abs(hist[-1]["e_true"] - ev[0]) < 0.1 * abs(ev[0])
    assert abs(o.norm(psi) - 1) < 1e-12


@pytest.mark.parametrize("which,sigma", [("LM", 0.0), ("SM", 0.5)])
def test_eig_arnoldi_dense_eigenvalue(hubbard3, which, sigma):
    H, ev, b0 = hubbard3
    lam, v, hist = ko.eig_arnoldi(H, 6, b0, Imax=6, rmax=16, which=which, sigma=sigma, history=True)
    want = ev[np.argmax(np.abs(ev + sigma))] if which == "LM" else ev[np.argmin(np.abs(ev + sigma))]
    assert abs(lam - want) < 1e-3 * max(1.0, abs(want))
