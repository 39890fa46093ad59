"""Krylov callers on the GPU (ttcuda.solvers, src/tt_solvers.jl, src/sketches.jl:617-1038) against
the oracle's restatement (oracle/krylov_oracle.py) and the dense eigenproblem: boundary sketches,
the sketch-orthogonal expansion step, sketched Rayleigh-Ritz and restarted Arnoldi."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
import ttcuda.solvers as ts  # noqa: E402
from gpu_helpers import op_dev, rel, to_dev  # noqa: E402
from oracle import krylov_oracle as ko  # noqa: E402
from oracle import models_oracle as mo  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402


@pytest.fixture(scope="module")
def hub():
    h, V = mo.hubbard_1D(3, t=0.1, U=0.4)
    dims = (2,) * 6
    H = mo.hV_to_mpo(h, V, dims)
    D = o.tto_to_tensor(H).reshape(64, 64, order="F")
    ev = np.linalg.eigvalsh((D + D.T) / 2)
    b0 = o.rand_tt(dims, 4, np.random.default_rng(5), normalise=True)
    return H, op_dev(H), ev, b0, to_dev(b0)


@pytest.mark.parametrize("s,block,with_op", [(20, 8, False), (7, 3, True), (64, None, False), (40, 4, True)])
def test_tt_sketch_matches_oracle(hub, s, block, with_op):
    H, Hd, _, b0, b0d = hub
    got, sa = ts.tt_sketch(b0d, s, Hd if with_op else None, True, 99, block)
    want, sw = ko.tt_sketch(b0, s, H if with_op else None, True, 99, block)
    assert sa == sw
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("with_op", [False, True])
def test_tt_combined_sketch_matches_oracle(hub, with_op):
    H, Hd, _, b0, b0d = hub
    got, Wg, sg = ts.tt_combined_sketch(b0d, 6, 50, Hd if with_op else None, True, 5, 4)
    want, Ww, sw = ko.tt_combined_sketch(b0, 6, 50, H if with_op else None, True, 5, 4)
    assert sg == sw and len(got) == len(want)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    for a, b in zip(Wg, Ww):
        assert a.shape == b.shape and np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300)


def test_expand_basis_matches_stored_sketch_form(hub):
    H, Hd, _, b0, b0d = hub
    rmax = 8
    sk0, W1, _ = ko.tt_combined_sketch(b0, 2 * rmax, 24, None, True, 1234, 8)
    beta = float(np.linalg.norm(sk0))
    ko._rescale_upto_root(W1, b0, beta)
    Bo, Wo, So = [o.tt_scale(1 / beta, b0)], [W1], [sk0 / beta]
    sk0d, W1d, _ = ts.tt_combined_sketch(b0d, 2 * rmax, 24, None, True, 1234, 8)
    ts._rescale_sketch(W1d, b0d, float(np.linalg.norm(sk0d)))
    Bd, Wd, Sd = [ttcuda.tt_scale(1 / float(np.linalg.norm(sk0d)), b0d)], [W1d], [sk0d / np.linalg.norm(sk0d)]
    for _ in range(3):
        bo, sbo, sho = ko.expand_basis(H, Bo, Wo, So, rmax, len(sk0), True, 8, 1234, 2)
        bd, sbd, shd = ts.expand_basis(Hd, Bd, Wd, Sd, rmax, len(sk0), True, 8, 1234, 2)
        assert list(bd.ttv_rks) == list(bo.ttv_rks)
        assert rel(bd, bo) < 1e-10
        assert np.abs(sbd - sbo).max() < 1e-10 and np.abs(shd - sho).max() < 1e-10 * np.abs(sho).max()
    assert len(Bd) == len(Wd) == len(Sd) == 2


def test_sketched_rayleigh_ritz_matches_oracle_and_is_variational(hub):
    H, Hd, ev, b0, b0d = hub
    eo, psio, ho = ko.sketched_rayleigh_ritz(H, b0, 10, 8)
    ed, psid, hd = ts.sketched_rayleigh_ritz(Hd, b0d, 10, 8)
    assert len(hd) == len(ho)
    for a, b in zip(hd, ho):
        assert a["iter"] == b["iter"]
        for key in ("e_sketch", "e_true", "res_sketch", "res_sample"):
            if np.isfinite(b[key]):
                assert abs(a[key] - b[key]) <= 1e-8 * max(1.0, abs(b[key])), key
            else:
                assert not np.isfinite(a[key])
        if np.isfinite(a["e_true"]):
            assert a["e_true"] >= ev[0] - 1e-12
    assert abs(ed - eo) <= 1e-8 * abs(eo)
    ov = abs(ttcuda.dot(psid, to_dev(psio)))
    assert abs(ov - 1) < 1e-8


def test_sketched_rayleigh_ritz_schedule_stages(hub):
    _, Hd, ev, _, b0d = hub
    lam, psi, stages, seeds = ts.sketched_rayleigh_ritz_schedule(Hd, b0d, [dict(d=6, rmax=8), dict(d=8, rmax=6)])
    assert seeds == [1234, 1235] and [s[0] for s in stages] == ["d=6, rmax=8", "d=8, rmax=6"]
    assert max(psi.ttv_rks) <= 6 * 4 and lam >= ev[0] - 1e-3


@pytest.mark.parametrize("which,sigma", [("LM", 0.0), ("SM", 0.5)])
def test_eig_arnoldi_matches_oracle_and_dense(hub, which, sigma):
    H, Hd, ev, b0, b0d = hub
    lo, vo, _ = ko.eig_arnoldi(H, 6, b0, Imax=6, rmax=16, which=which, sigma=sigma)
    ld, vd, hist = ts.eig_arnoldi(Hd, 6, b0d, Imax=6, rmax=16, which=which, sigma=sigma, history=True)
    assert abs(ld - lo) <= 1e-8 * max(1.0, abs(lo))
    want = ev[np.argmax(np.abs(ev + sigma))] if which == "LM" else ev[np.argmin(np.abs(ev + sigma))]
    assert abs(ld - want) < 1e-3 * max(1.0, abs(want))
    assert all(np.isfinite(hist))
