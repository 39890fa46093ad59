"""Host side of the MPO builders in the package (ttcuda.models): the Hamiltonian coefficient
arrays and orderings against the oracle's restatement of src/models.jl, and the exact
term algebra (rank-1 operator products and block sums) against the oracle's operator products,
all without a GPU."""
import numpy as np

import ttcuda.models as tm
from oracle import models_oracle as mo
from oracle import tt_oracle as o


def test_model_arrays_match_the_oracle():
    for a, b in [(tm.hubbard_1D(6, t=1.0, U=4.0), mo.hubbard_1D(6, t=1.0, U=4.0)),
                 (tm.hubbard_1D(5, t=0.5, U=2.0, pbc=True), mo.hubbard_1D(5, t=0.5, U=2.0, pbc=True)),
                 (tm.hubbard_2D(4, 4, t=1.0, U=8.0, w_pbc=False, L_pbc=False),
                  mo.hubbard_2D(4, 4, t=1.0, U=8.0, w_pbc=False, L_pbc=False)),
                 (tm.hubbard_2D(3, 4, t=1.0, U=2.0, w_pbc=True, L_pbc=True),
                  mo.hubbard_2D(3, 4, t=1.0, U=2.0, w_pbc=True, L_pbc=True))]:
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(tm.snake_order(4, 4), mo.snake_permutation(4, 4))
    h1, V1 = mo.synthetic_molecular_integrals(3, seed=4)
    g1, W1 = tm.synthetic_molecular_integrals(3, seed=4)
    assert np.array_equal(h1, g1) and np.array_equal(V1, W1)
    a, b = tm.one_e_two_e_integrals_to_hV(h1, V1), mo.one_e_two_e_integrals_to_hV(h1, V1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_terms_and_sums_match_oracle_operator_products():
    """Each term of the package's builder equals the oracle's product of creation and
    annihilation MPOs (src/models.jl:193-224), and the block sum equals the oracle's sum."""
    L = 5
    dims = (2,) * L
    h, V = mo.hubbard_1D(3, t=1.0, U=2.0)[0][:L, :L], np.zeros((L,) * 4)
    h = h + np.diag(np.arange(1.0, L + 1))
    V[0, 2, 1, 3] = V[3, 1, 2, 0] = 0.7
    V[1, 1, 4, 4] = -0.3
    terms = tm._hV_terms(h, V, L, chemistry=False)
    crea = [mo.tto_creation(i, dims) for i in range(1, L + 1)]
    anni = [mo.tto_annihilation(i, dims) for i in range(1, L + 1)]
    ref = mo._hV_terms(h, V, crea, anni, chemistry=False)
    assert len(terms) == len(ref)
    total_p, total_o = None, None
    for t, r in zip(terms, ref):
        A = t.tto()
        Ao = o.TToperator(A.N, A.tto_vec, A.tto_dims, A.tto_rks, [0] * A.N)
        assert A.tto_rks == r.tto_rks
        assert np.allclose(o.tto_to_tensor(Ao), o.tto_to_tensor(r), atol=1e-14)
        total_p = A if total_p is None else tm.tto_add(total_p, A)
        total_o = r if total_o is None else o.tto_add(total_o, r)
    Tp = o.TToperator(total_p.N, total_p.tto_vec, total_p.tto_dims, total_p.tto_rks, [0] * L)
    assert total_p.tto_rks == total_o.tto_rks
    assert all(np.array_equal(a, b) for a, b in zip(Tp.tto_vec, total_o.tto_vec))
