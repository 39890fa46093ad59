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


def hV_to_mpo(h, V, dims, tol=1e-8, n_rnd=20, chemistry=False) -> o.TToperator:
    """src/models.jl:180-231"""
    L = h.shape[0]
    assert np.allclose(h, h.T)
    A = o.zeros_tto(dims, [1] * (L + 1))
    crea = [tto_creation(i, dims) for i in range(1, L + 1)]
    anni = [tto_annihilation(i, dims) for i in range(1, L + 1)]
    i_rnd = 1

    def maybe_round(A, i_rnd):
        if i_rnd > n_rnd:
            return o.tt_rounding_tto(A, tol=tol), 1
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
    return o.tt_rounding_tto(A, tol=tol)


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
