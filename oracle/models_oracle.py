"""MPO builders restated from src/models.jl (TEST/SETUP INFRASTRUCTURE ONLY).

They produce the Hamiltonian MPO inputs of the Hubbard workloads on the host
(the reference builds them on the host too); the CUDA library only consumes the
resulting TToperator cores.
"""
from __future__ import annotations

import numpy as np

from . import tt_oracle as o


def _core(entries):
    out = np.zeros((2, 2, 1, 1))
    for (i, j), v in entries.items():
        out[i, j, 0, 0] = v
    return out


def mpo_core_id():            # src/models.jl:92-97
    return _core({(0, 0): 1.0, (1, 1): 1.0})


def mpo_core_ferm_sign():     # src/models.jl:99-105
    return _core({(0, 0): 1.0, (1, 1): -1.0})


def mpo_core_creation():      # src/models.jl:107-112
    return _core({(1, 0): 1.0})


def mpo_core_annihilation():  # src/models.jl:114-119
    return _core({(0, 1): 1.0})


def tto_creation(p: int, dims, fermion=True) -> o.TToperator:
    """src/models.jl:124-138 (1-based site p)."""
    N = len(dims)
    A = o.zeros_tto(dims, [1] * (N + 1))
    for i in range(p - 1):
        A.tto_vec[i] = mpo_core_ferm_sign() if fermion else mpo_core_id()
    A.tto_vec[p - 1] = mpo_core_creation()
    for i in range(p, N):
        A.tto_vec[i] = mpo_core_id()
    return A


def tto_annihilation(q: int, dims, fermion=True) -> o.TToperator:
    """src/models.jl:143-154 (1-based site q)."""
    N = len(dims)
    A = o.zeros_tto(dims, [1] * (N + 1))
    for i in range(q - 1):
        A.tto_vec[i] = mpo_core_ferm_sign() if fermion else mpo_core_id()
    A.tto_vec[q - 1] = mpo_core_annihilation()
    for i in range(q, N):
        A.tto_vec[i] = mpo_core_id()
    return A


def _mul(*ops):
    """Variadic TTO product, right-associated like `*(A, B...) = *(A, *(B...))`."""
    out = ops[-1]
    for A in reversed(ops[:-1]):
        out = o.tto_mul(A, out)
    return out


def _nonzero_indices(T, atol=1e-12):
    """Julia `findall(x -> !isapprox(x, 0.0, atol=atol), T)`: column-major order, 1-based."""
    idx = np.argwhere(np.abs(np.transpose(T, tuple(range(T.ndim))[::-1])) > atol)
    return [tuple(int(v) + 1 for v in row[::-1]) for row in idx]


def hV_to_mpo(h, V, dims, tol=1e-8, n_rnd=20, chemistry=False, round_tto=None) -> o.TToperator:
    """src/models.jl:180-231.  `round_tto(A, tol)` performs the tt_rounding(::TToperator) steps
    (src/tt_rounding.jl:275-277); the default is the oracle's own, a test may pass the device's."""
    rnd = round_tto or (lambda A, tol: o.tt_rounding_tto(A, tol=tol))
    L = h.shape[0]
    assert np.allclose(h, h.T)
    A = o.zeros_tto(dims, [1] * (L + 1))
    crea = [tto_creation(i, dims) for i in range(1, L + 1)]
    anni = [tto_annihilation(i, dims) for i in range(1, L + 1)]
    i_rnd = 1

    def maybe_round(A, i_rnd):
        if i_rnd > n_rnd:
            return rnd(A, tol), 1
        return A, i_rnd + 1

    for i in _nonzero_indices(h):
        a, b = i
        if a < b:
            H = o.tto_add(_mul(crea[a - 1], anni[b - 1]), _mul(crea[b - 1], anni[a - 1]))
            A = o.tto_add(A, o.tto_scale(h[a - 1, b - 1], H))
        elif a == b:
            H = _mul(crea[a - 1], anni[b - 1])
            A = o.tto_add(A, o.tto_scale(h[a - 1, b - 1], H))
        A, i_rnd = maybe_round(A, i_rnd)
    for i in _nonzero_indices(V):
        i1, i2, i3, i4 = i
        v = V[i1 - 1, i2 - 1, i3 - 1, i4 - 1]
        if chemistry:
            if (i1, i3) < (i2, i4):
                H = o.tto_add(_mul(crea[i1 - 1], crea[i3 - 1], anni[i4 - 1], anni[i2 - 1]),
                              _mul(crea[i2 - 1], crea[i4 - 1], anni[i3 - 1], anni[i1 - 1]))
                A = o.tto_add(A, o.tto_scale(0.5 * v, H))
            elif (i1, i3) == (i2, i4):
                H = _mul(crea[i1 - 1], crea[i3 - 1], anni[i4 - 1], anni[i2 - 1])
                A = o.tto_add(A, o.tto_scale(0.5 * v, H))
        else:
            if (i1, i2) < (i4, i3):
                H = o.tto_add(_mul(crea[i1 - 1], crea[i2 - 1], anni[i3 - 1], anni[i4 - 1]),
                              _mul(crea[i4 - 1], crea[i3 - 1], anni[i2 - 1], anni[i1 - 1]))
                A = o.tto_add(A, o.tto_scale(v, H))
            elif (i1, i2) == (i4, i3):
                H = _mul(crea[i1 - 1], crea[i2 - 1], anni[i3 - 1], anni[i4 - 1])
                A = o.tto_add(A, o.tto_scale(v, H))
        A, i_rnd = maybe_round(A, i_rnd)
    return rnd(A, tol)


def _hV_terms(h, V, crea, anni, chemistry):
    """The scaled one- and two-body terms of hV_to_mpo_tree's phase 1 (src/models.jl:263-300), in
    the order Julia's findall visits h and V (column-major)."""
    terms = []
    for a, b in _nonzero_indices(h):
        if a < b:
            terms.append(o.tto_scale(h[a - 1, b - 1], o.tto_add(_mul(crea[a - 1], anni[b - 1]),
                                                                 _mul(crea[b - 1], anni[a - 1]))))
        elif a == b:
            terms.append(o.tto_scale(h[a - 1, b - 1], _mul(crea[a - 1], anni[b - 1])))
    for i1, i2, i3, i4 in _nonzero_indices(V):
        v = V[i1 - 1, i2 - 1, i3 - 1, i4 - 1]
        if chemistry:
            if (i1, i3) < (i2, i4):
                terms.append(o.tto_scale(v / 2, o.tto_add(_mul(crea[i1 - 1], crea[i3 - 1], anni[i4 - 1], anni[i2 - 1]),
                                                          _mul(crea[i2 - 1], crea[i4 - 1], anni[i3 - 1], anni[i1 - 1]))))
            elif (i1, i3) == (i2, i4):
                terms.append(o.tto_scale(v / 2, _mul(crea[i1 - 1], crea[i3 - 1], anni[i4 - 1], anni[i2 - 1])))
        else:
            if (i1, i2) < (i4, i3):
                terms.append(o.tto_scale(v, o.tto_add(_mul(crea[i1 - 1], crea[i2 - 1], anni[i3 - 1], anni[i4 - 1]),
                                                      _mul(crea[i4 - 1], crea[i3 - 1], anni[i2 - 1], anni[i1 - 1]))))
            elif (i1, i2) == (i4, i3):
                terms.append(o.tto_scale(v, _mul(crea[i1 - 1], crea[i2 - 1], anni[i3 - 1], anni[i4 - 1])))
    return terms


def hV_to_mpo_tree(h, V, dims, tol=1e-8, n_leaf=20, n_branch=8, chemistry=False, round_tto=None) -> o.TToperator:
    """src/models.jl:254-338: every term collected (phase 1), summed in leaf groups of n_leaf and
    rounded (phase 2), then merged n_branch at a time with a rounding per merge until one MPO
    remains (phase 3).  `round_tto(A, tol)` as in hV_to_mpo."""
    rnd = round_tto or (lambda A, tol: o.tt_rounding_tto(A, tol=tol))
    L = h.shape[0]
    N = len(dims)
    assert np.allclose(h, h.T)
    crea = [tto_creation(i, dims) for i in range(1, L + 1)]
    anni = [tto_annihilation(i, dims) for i in range(1, L + 1)]
    terms = _hV_terms(h, V, crea, anni, chemistry)
    if not terms:
        return o.zeros_tto(dims, [1] * (N + 1))
    current = []
    for g0 in range(0, len(terms), n_leaf):
        A = terms[g0]
        for t in terms[g0 + 1: g0 + n_leaf]:
            A = o.tto_add(A, t)
        current.append(rnd(A, tol))
    while len(current) > 1:
        nxt = []
        for g0 in range(0, len(current), n_branch):
            A = current[g0]
            for t in current[g0 + 1: g0 + n_branch]:
                A = o.tto_add(A, t)
            nxt.append(rnd(A, tol))
        current = nxt
    return current[0]


def one_body_mpo(p: int, q: int, dims, fermion=True) -> o.TToperator:
    """src/models.jl:160-163: a_p^dagger a_q (1-based sites)."""
    return o.tto_mul(tto_creation(p, dims, fermion), tto_annihilation(q, dims, fermion))


def id_tto(d: int, n_dim: int = 2) -> o.TToperator:
    """src/tt_tools.jl:704-716: the identity as a rank-1 TToperator."""
    vec = [np.eye(n_dim).reshape(n_dim, n_dim, 1, 1).copy() for _ in range(d)]
    return o.TToperator(d, vec, (n_dim,) * d, [1] * (d + 1), [0] * d)


def PPP_C_NH_N(N: int, beta=-2.5 / 27.2113845, b=1.4 * 1.8897259886, gamma0=10.84 / 27.2113845, order=None,
               tol=1e-8, round_tto=None) -> o.TToperator:
    """src/models.jl:487-514: Pariser-Parr-Pople Hamiltonian of the cyclic polyene C_N H_N
    (2N spin-orbitals, `order` a 0-based permutation of them)."""
    rnd = round_tto or (lambda A, tol: o.tt_rounding_tto(A, tol=tol))
    order = np.arange(2 * N) if order is None else np.asarray(order)
    dims = (2,) * (2 * N)
    h = np.zeros((2 * N, 2 * N))
    for i in range(1, N):                                     # Julia i = 1..N-1, 1-based indices
        h[2 * i - 2, 2 * i] = h[2 * i, 2 * i - 2] = beta      # h[2i-1, 2i+1]
        h[2 * i - 1, 2 * i + 1] = h[2 * i + 1, 2 * i - 1] = beta  # h[2i, 2i+2]
    h[2 * N - 1, 1] = h[1, 2 * N - 1] = beta                  # h[2N, 2]
    h[2 * N - 2, 0] = h[0, 2 * N - 2] = beta                  # h[2N-1, 1]
    hs = np.triu(h) + np.triu(h, 1).T                         # Symmetric(h)
    H = hV_to_mpo(hs[np.ix_(order, order)], np.zeros((2 * N,) * 4), dims, round_tto=round_tto)
    sigma = np.argsort(order)                                 # invperm, 0-based
    ident = o.tto_scale(-1.0, id_tto(2 * N))
    for i in range(1, N + 1):
        Hi = o.tto_add(o.tto_add(one_body_mpo(sigma[2 * i - 1] + 1, sigma[2 * i - 1] + 1, dims),
                                 one_body_mpo(sigma[2 * i - 2] + 1, sigma[2 * i - 2] + 1, dims)), ident)
        for j in range(1, N + 1):
            Hj = o.tto_add(o.tto_add(one_body_mpo(sigma[2 * j - 1] + 1, sigma[2 * j - 1] + 1, dims),
                                     one_body_mpo(sigma[2 * j - 2] + 1, sigma[2 * j - 2] + 1, dims)), ident)
            Htemp = o.tto_mul(Hi, Hj)
            gij = 1.0 / (1.0 / gamma0 + b * np.sin(np.pi / N * ((i - j) % N)) / np.sin(np.pi / N))
            H = o.tto_add(H, o.tto_scale(0.5 * gij, Htemp))
        H = rnd(H, tol)
    return H


def one_e_two_e_integrals_to_hV(int1e, int2e):
    """src/models.jl:529-549: spatial-orbital integrals (L x L, L^4) to spin-orbital h (2L x 2L)
    and V (2L)^4, spin up on odd (1-based) and spin down on even spin-orbitals."""
    L = int1e.shape[0]
    h = np.zeros((2 * L, 2 * L))
    V = np.zeros((2 * L,) * 4)
    up = np.arange(L) * 2          # 1-based 2i-1
    dn = up + 1                    # 1-based 2i
    h[np.ix_(up, up)] = int1e
    h[np.ix_(dn, dn)] = int1e
    # V[2i-1,2j-1,2l-1,2k-1] = V[2i,2j,2l,2k] = V[2i,2j,2l-1,2k-1] = V[2i-1,2j-1,2l,2k] = int2e[i,j,l,k]
    for a, bb in ((up, up), (dn, dn), (dn, up), (up, dn)):
        V[np.ix_(a, a, bb, bb)] = int2e
    return h, V


def synthetic_molecular_integrals(L: int, seed: int, decay: float = 4.0):
    """Synthetic molecular integrals: h_ij = h_ji ~ N(0,1) exp(-|i-j|/decay) and V_ijkl ~ N(0,1) with
    the 8-fold permutational symmetry of real two-electron integrals, scaled by
    exp(-(|i-j| + |k-l|)/decay).  V is indexed like int2e of one_e_two_e_integrals_to_hV."""
    g = np.random.default_rng(seed)
    i = np.arange(L)
    h = g.standard_normal((L, L)) * np.exp(-np.abs(i[:, None] - i[None, :]) / decay)
    h = np.triu(h) + np.triu(h, 1).T
    V = g.standard_normal((L,) * 4)
    V = (V + V.transpose(1, 0, 2, 3) + V.transpose(0, 1, 3, 2) + V.transpose(1, 0, 3, 2)
         + V.transpose(2, 3, 0, 1) + V.transpose(3, 2, 0, 1) + V.transpose(2, 3, 1, 0) + V.transpose(3, 2, 1, 0)) / 8.0
    dij = np.abs(i[:, None] - i[None, :])
    V = V * np.exp(-(dij[:, :, None, None] + dij[None, None, :, :]) / decay)
    return h, V


def hubbard_1D(L, t=1.0, U=1.0, pbc=False):
    """src/models.jl:403-419 (returns h, V as dense arrays, 0-based storage)."""
    h = np.zeros((2 * L, 2 * L))
    V = np.zeros((2 * L,) * 4)
    for i in range(1, L):
        h[2 * i - 1, 2 * i + 1] = -t
        h[2 * i - 2, 2 * i] = -t
        V[2 * i - 2, 2 * i - 1, 2 * i - 2, 2 * i - 1] = -U
        V[2 * i - 1, 2 * i - 2, 2 * i - 1, 2 * i - 2] = -U
    V[2 * L - 2, 2 * L - 1, 2 * L - 2, 2 * L - 1] = -U
    V[2 * L - 1, 2 * L - 2, 2 * L - 1, 2 * L - 2] = -U
    if pbc:
        h[2 * L - 2, 0] = -t
        h[2 * L - 1, 1] = -t
    hs = np.triu(h) + np.triu(h, 1).T        # Symmetric(h) uses the upper triangle
    return hs, V


def hubbard_2D(w, L, t=1.0, U=1.0, w_pbc=False, L_pbc=True):
    """src/models.jl:431-476 (1-based Julia indices shifted by one)."""
    n = 2 * w * L
    h = np.zeros((n, n))
    V = np.zeros((n,) * 4)

    def setV(a, b):                # V[a,b,a,b] = -U  with 1-based a, b
        V[a - 1, b - 1, a - 1, b - 1] = -U

    def seth(a, b):
        h[a - 1, b - 1] = -t
    for i in range(0, w - 1):
        for j in range(0, L - 1):
            s = j * w + i
            setV(2 * s + 1, 2 * s + 2)
            setV(2 * s + 2, 2 * s + 1)
            seth(2 * s + 1, 2 * ((j + 1) * w + i) + 1)
            seth(2 * s + 1, 2 * (j * w + i + 1) + 1)
            seth(2 * s + 2, 2 * ((j + 1) * w + i) + 2)
            seth(2 * s + 2, 2 * (j * w + i + 1) + 2)
        s = (L - 1) * w + i
        setV(2 * s + 1, 2 * s + 2)
        setV(2 * s + 2, 2 * s + 1)
        seth(2 * s + 1, 2 * ((L - 1) * w + i + 1) + 1)
        seth(2 * s + 2, 2 * ((L - 1) * w + i + 1) + 2)
        if L_pbc and L > 2:
            seth(2 * (L * w + i - w) + 1, 2 * i + 1)
            seth(2 * (L * w + i - w) + 2, 2 * i + 2)
    for j in range(0, L - 1):
        s = j * w + w - 1
        setV(2 * s + 1, 2 * s + 2)
        setV(2 * s + 2, 2 * s + 1)
        seth(2 * s + 1, 2 * ((j + 1) * w + w - 1) + 1)
        seth(2 * s + 2, 2 * ((j + 1) * w + w - 1) + 2)
        if w_pbc and w > 2:
            seth(2 * s + 1, 2 * j * w + 1)
            seth(2 * s + 2, 2 * j * w + 2)
    setV(2 * L * w - 1, 2 * L * w)
    setV(2 * L * w, 2 * L * w - 1)
    if L_pbc and L > 2:
        seth(2 * (L * w - 1) + 1, 2 * (w - 1) + 1)
        seth(2 * (L * w - 1) + 2, 2 * (w - 1) + 2)
    if w_pbc and w > 2:
        seth(2 * (L * w - 1) + 1, 2 * (L - 1) * w + 1)
        seth(2 * (L * w - 1) + 2, 2 * (L - 1) * w + 2)
    hs = np.triu(h) + np.triu(h, 1).T
    return hs, V


def snake_permutation(w, L):
    """Spin-orbital permutation for a snake ordering of the w x L lattice labelled s = j*w + i
    (src/models.jl:436-441): columns j with odd j are traversed with i reversed.  Returns the
    0-based spin-orbital order sigma used as h[sigma][:, sigma] (examples/hubbard_2d_orderings.jl:12-15)."""
    sites = []
    for j in range(L):
        col = [j * w + i for i in range(w)]
        sites += col[::-1] if j % 2 == 1 else col
    sigma = []
    for s in sites:
        sigma += [2 * s, 2 * s + 1]
    return np.array(sigma)
