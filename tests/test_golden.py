"""CPU pins of the oracle: a known answer from the reference's own test suite, dense checks of the
MPO builders, and the golden fixtures' inputs and cheap expected values.

* PPP benzene (test/test_models.jl:24-30): the reference asserts that the ground-state energy of
  PPP_C_NH_N(6) is -0.46752535023652453 (atol 1e-6; Bendazzoli & Evangelisti 1991).  The oracle
  builds that MPO with hV_to_mpo, operator products and sums, and tt_rounding(::TToperator) -- the
  rounding path itself -- and a dense eigensolve of the 6-electron sector gives the energy.
* one_body_mpo against dense Jordan-Wigner matrices (test/test_models.jl:6-22), and hV_to_mpo /
  hV_to_mpo_tree against the dense second-quantised Hamiltonian on 4 spatial orbitals.
* The golden fixtures: regenerated inputs match the stored checksums, and the config-1 expected
  values are re-derived by the oracle.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from oracle import models_oracle as mo  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402

import golden  # noqa: E402

PPP_BENZENE_ENERGY = -0.46752535023652453    # test/test_models.jl:29


def test_ein_matches_einsum_on_the_oracle_expressions():
    g = np.random.default_rng(0)
    exprs = {
        "zaA,AB,Bzb->ab": [(2, 3, 4), (4, 5), (5, 2, 6)],
        "AB,Bzb,zaA->ab": [(4, 5), (5, 2, 6), (2, 3, 4)],
        "Aeg,zaA,Zzbe,gZc->abc": [(4, 3, 5), (2, 6, 4), (2, 2, 7, 3), (5, 2, 8)],
        "Aeg,gZc,Zzbe,zaA->abc": [(4, 3, 5), (5, 2, 8), (2, 2, 7, 3), (2, 6, 4)],
        "iab,iac,jbd->jcd": [(2, 3, 4), (2, 3, 5), (2, 4, 6)],
        "irab,irs,jac,ljbd->lscd": [(2, 3, 4, 5), (2, 3, 6), (2, 4, 7), (2, 2, 5, 3)],
        "ira,irs,jab->jsb": [(2, 3, 4), (2, 3, 5), (2, 4, 6)],
        "abc,iad,ijbe,jcf->def": [(3, 4, 5), (2, 3, 6), (2, 2, 4, 7), (2, 5, 8)],
        "ac,iad,icf->df": [(3, 4), (2, 3, 5), (2, 4, 6)],
        "def,jcf,ijbe,iad->abc": [(3, 4, 5), (2, 6, 5), (2, 2, 7, 4), (2, 8, 3)],
        "df,icf,iad->ac": [(3, 4), (2, 5, 4), (2, 6, 3)],
        "abc,jcf,ijbe,def->iad": [(3, 4, 5), (2, 5, 6), (2, 2, 4, 7), (8, 7, 6)],
        "ac,icf,df->iad": [(3, 4), (2, 4, 5), (6, 5)],
        "ac,zab,zcd->bd": [(3, 4), (2, 3, 5), (2, 4, 6)],
        "bd,zab,zcd->ac": [(5, 6), (2, 3, 5), (2, 4, 6)],
    }
    for e, shapes in exprs.items():
        ops = [g.standard_normal(s) for s in shapes]
        ref = np.einsum(e, *ops)
        assert np.allclose(o.ein(e, *ops), ref, rtol=1e-12, atol=1e-12), e


def _ground_energy(H, electrons):
    n = H.N
    M = o.tto_to_tensor(H).reshape(2 ** n, 2 ** n, order="F")
    idx = np.arange(2 ** n)
    pop = np.array([bin(i).count("1") for i in idx])
    sel = idx[pop == electrons]
    return float(np.linalg.eigvalsh(M[np.ix_(sel, sel)])[0]), float(np.abs(M - M.T).max())


def test_oracle_ppp_benzene_known_answer():
    """The reference's known answer for PPP C6H6 (test/test_models.jl:24-30), with the identity
    ordering and a permuted one (the reference test permutes the 12 spin-orbitals at random)."""
    for order in (None, np.random.default_rng(3).permutation(12)):
        H = mo.PPP_C_NH_N(6, order=order)
        e, asym = _ground_energy(H, 6)
        assert asym < 1e-12
        assert abs(e - PPP_BENZENE_ENERGY) <= 1e-6          # the reference's tolerance
        assert abs(e - PPP_BENZENE_ENERGY) <= 1e-11         # what the FP64 restatement reaches


def _dense_ops(L):
    """Dense Jordan-Wigner creation operators on L modes, mode index 1 fastest (column-major
    Kronecker order, as tto_to_tensor lays out the sites)."""
    cr = np.array([[0.0, 0.0], [1.0, 0.0]])      # mpo_core_creation: |0> -> |1>
    zs = np.diag([1.0, -1.0])
    ident = np.eye(2)
    ops = []
    for p in range(L):
        M = np.ones((1, 1))
        for s in range(L):           # later sites go to the slower (outer) Kronecker factor
            f = zs if s < p else (cr if s == p else ident)
            M = np.kron(f, M)
        ops.append(M)
    return ops


def test_one_body_mpo_matches_dense():
    """test/test_models.jl:6-15 re-expressed: a_p^dagger a_q as an MPO equals its dense matrix."""
    L = 6
    c = _dense_ops(L)
    for p, q in [(1, 1), (2, 5), (6, 3), (4, 4)]:
        A = mo.one_body_mpo(p, q, (2,) * L)
        D = o.tto_to_tensor(A).reshape(2 ** L, 2 ** L, order="F")
        assert np.abs(D - c[p - 1] @ c[q - 1].T).max() < 1e-12


def test_hV_to_mpo_tree_and_hV_to_mpo_match_dense_chemistry_hamiltonian():
    """4 spatial orbitals (8 spin-orbitals): synthetic symmetric integrals through
    one_e_two_e_integrals_to_hV; hV_to_mpo_tree (small leaves and branches, so that every phase
    runs) and hV_to_mpo with chemistry=true both equal the dense
    H = sum h_ij a_i^+ a_j + 1/2 sum V_ijkl a_i^+ a_k^+ a_l a_j (src/models.jl:263-285)."""
    h1, V1 = mo.synthetic_molecular_integrals(4, seed=11)
    h, V = mo.one_e_two_e_integrals_to_hV(h1, V1)
    L = h.shape[0]
    c = _dense_ops(L)
    a = [m.T for m in c]
    D = np.zeros((2 ** L, 2 ** L))
    for i in range(L):
        for j in range(L):
            if h[i, j] != 0:
                D += h[i, j] * c[i] @ a[j]
    nz = np.argwhere(np.abs(V) > 1e-12)
    for i, j, k, l in nz:
        D += 0.5 * V[i, j, k, l] * (c[i] @ c[k] @ a[l] @ a[j])
    assert np.abs(D - D.T).max() < 1e-10
    T = mo.hV_to_mpo_tree(h, V, (2,) * L, n_leaf=7, n_branch=3, chemistry=True)
    Dt = o.tto_to_tensor(T).reshape(2 ** L, 2 ** L, order="F")
    assert np.abs(Dt - D).max() <= 1e-7 * np.abs(D).max()
    Hs = mo.hV_to_mpo(h, V, (2,) * L, chemistry=True)
    Ds = o.tto_to_tensor(Hs).reshape(2 ** L, 2 ** L, order="F")
    assert np.abs(Ds - D).max() <= 1e-7 * np.abs(D).max()


def _fixture(name):
    p = golden.path(name)
    if not os.path.exists(p):
        pytest.fail(f"missing golden fixture {name}: run tests/golden/make_golden.py")
    return golden.load(name)


def test_golden_config1_rederived_by_the_oracle():
    import make_golden as mg
    fx = _fixture("config1_sum_of_tts.json.gz")
    terms = [o.json_to_mps(t) for t in fx["terms"]]
    fresh = mg.config1_terms()
    for a, b in zip(terms, fresh):
        assert all(np.array_equal(p, q) for p, q in zip(a.ttv_vec, b.ttv_vec))
    X = mg.config1_input(terms)
    assert golden.checksum_ok(golden.checksum(X), fx["input_checksum"])
    Y = o.tt_rounding(X, tol=fx["params"]["tol"], rmax=fx["params"]["rmax"])
    assert golden.compare(golden.fingerprint(Y, X), fx["expected"], 1e-12) == []


def test_golden_inputs_regenerate_to_their_checksums():
    import make_golden as mg
    fx3 = _fixture("config3_batch3.json.gz")
    for x, cs in zip(mg.config3_inputs(), fx3["input_checksums"]):
        assert golden.checksum_ok(golden.checksum(x), cs)
    assert mg.config3_rks() == fx3["rks"]
    fx2 = _fixture("config2_hubbard_op.json.gz")
    H, y = mg.config2_inputs()
    Hj = o.json_to_mpo(fx2["mpo"])
    assert H.tto_rks == Hj.tto_rks
    assert all(np.allclose(p, q, rtol=0, atol=1e-13) for p, q in zip(H.tto_vec, Hj.tto_vec))
    assert golden.checksum_ok(golden.checksum(y), fx2["y_checksum"])
