"""MPO construction with the roundings on the GPU (ttcuda.models, src/models.jl:180-338)
against the oracle's restatement and against the dense second-quantised Hamiltonian."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
import ttcuda.models as tm  # noqa: E402
from oracle import models_oracle as mo  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402


def _dense(A):
    Ao = o.TToperator(A.N, A.tto_vec, A.tto_dims, A.tto_rks, [0] * A.N)
    n = 2 ** A.N
    return o.tto_to_tensor(Ao).reshape(n, n, order="F")


def test_hV_to_mpo_hubbard_matches_oracle():
    h, V = tm.hubbard_1D(5, t=1.0, U=4.0)
    dims = (2,) * 10
    A = tm.hV_to_mpo(h, V, dims)
    B = mo.hV_to_mpo(h, V, dims)
    assert A.tto_rks == B.tto_rks
    D, Db = _dense(A), _dense(B)
    assert np.abs(D - Db).max() <= 1e-10 * np.abs(Db).max()


def test_hV_to_mpo_tree_chemistry_matches_oracle_and_dense():
    """4 spatial orbitals (8 spin-orbitals), small leaves and branches so that the batched leaf
    rounding and two merge levels run."""
    h1, V1 = tm.synthetic_molecular_integrals(4, seed=11)
    h, V = tm.one_e_two_e_integrals_to_hV(h1, V1)
    dims = (2,) * 8
    A = tm.hV_to_mpo_tree(h, V, dims, n_leaf=7, n_branch=3, chemistry=True)
    B = mo.hV_to_mpo_tree(h, V, dims, n_leaf=7, n_branch=3, chemistry=True)
    assert A.tto_rks == B.tto_rks
    D, Db = _dense(A), _dense(B)
    assert np.abs(D - Db).max() <= 1e-9 * np.abs(Db).max()
    # and the reference's sequential builder gives the same operator
    C = tm.hV_to_mpo(h, V, dims, chemistry=True)
    assert np.abs(_dense(C) - Db).max() <= 1e-7 * np.abs(Db).max()


def test_config4_hamiltonian_energy_expectation():
    """The config-4 MPO (4x4 open Hubbard, U=8, snake ordering) built on the GPU: <x|H|x> of a
    random rank-8 TT equals that of the oracle-built MPO."""
    h, V = tm.hubbard_2D(4, 4, t=1.0, U=8.0, w_pbc=False, L_pbc=False)
    s = tm.snake_order(4, 4)
    hs, Vs = h[np.ix_(s, s)], V[np.ix_(s, s, s, s)]
    A = tm.hV_to_mpo(hs, Vs, (2,) * 32)
    B = mo.hV_to_mpo(hs, Vs, (2,) * 32)
    assert A.tto_rks == B.tto_rks
    x = o.rand_tt((2,) * 32, 8, np.random.default_rng(3), normalise=True)
    X = ttcuda.TTvector(x.N, x.ttv_vec, x.ttv_dims, x.ttv_rks)
    ea = ttcuda.dot_operator(X, A, X)
    eb = o.dot_operator(x, B, x)
    assert abs(ea - eb) <= 1e-9 * abs(eb)
