"""Second-quantised Hamiltonians as TToperators (MPOs), src/models.jl of TensorTrains.

The reference builds an MPO as a sum of Jordan-Wigner operator products, rounding the running
sum with tt_rounding(::TToperator) (src/tt_rounding.jl:275-277) every few terms (hV_to_mpo,
src/models.jl:180-231) or in a tree of leaf groups and merges (hV_to_mpo_tree, :254-338).  Here
the term algebra stays on the host, where it is exact and cheap: every term is a sum of rank-1
operators whose site matrices are products of 2x2 single-mode factors, and a sum of terms is the
block-diagonal TToperator the reference's `+` builds (src/tt_operations.jl:121-148), with the
blocks in the same order.  Every rounding runs on the GPU through libttcuda: an operator is
rounded as the TTvector with mode sizes n^2 that shares its memory (tto_to_ttv,
src/tt_tools.jl:603-611), and the tree builder rounds all leaf groups of a level, and all merges
of a level, in one batched call, since they are independent.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import DeviceBatch, TToperator, TTvector, get_context, tt_rounding

# single-mode factors [i_out, j_in] (src/models.jl:92-119); mode state 1 = empty, 2 = occupied
_ID = np.eye(2)
_SIGN = np.diag([1.0, -1.0])
_CREA = np.array([[0.0, 0.0], [1.0, 0.0]])
_ANNI = np.array([[0.0, 1.0], [0.0, 0.0]])


# ------------------------------------------------------------------ rank-1 operator products
def _chain_factors(ops: Sequence[Tuple[str, int]], N: int, fermion: bool = True) -> np.ndarray:
    """Site matrices (N, 2, 2) of the product op_1 * op_2 * ... of creation ('c') and
    annihilation ('a') operators on 1-based modes: the MPO product of rank-1 operators is the
    site-wise matrix product (src/tt_operations.jl:211-237); each single-mode operator is the
    sign factor before its mode, its 2x2 matrix on it and the identity after it
    (tto_creation / tto_annihilation, src/models.jl:124-154)."""
    out = np.broadcast_to(_ID, (N, 2, 2)).copy()
    before = _SIGN if fermion else _ID
    for kind, p in ops:
        f = np.broadcast_to(_ID, (N, 2, 2)).copy()
        f[: p - 1] = before
        f[p - 1] = _CREA if kind == "c" else _ANNI
        out = np.matmul(out, f)
    return out


class _RankOneSum:
    """A sum of scaled rank-1 operators: the TToperator the reference's `+` builds from them,
    one rank per piece in order (rank 1 at the boundaries)."""

    def __init__(self, N: int):
        self.N = N
        self.coef: List[float] = []
        self.sites: List[np.ndarray] = []

    def add(self, c: float, sites: np.ndarray):
        self.coef.append(float(c))
        self.sites.append(sites)

    def extend(self, other: "_RankOneSum"):
        self.coef += other.coef
        self.sites += other.sites

    def tto(self) -> TToperator:
        N, P = self.N, len(self.coef)
        S = np.stack(self.sites)                       # (P, N, 2, 2)
        vec = []
        for k in range(N):
            R0 = 1 if k == 0 else P
            R1 = 1 if k == N - 1 else P
            core = np.zeros((2, 2, R0, R1), order="F")
            blk = S[:, k]                              # (P, 2, 2)
            if N == 1:
                core[:, :, 0, 0] = np.tensordot(self.coef, blk, axes=1)
            elif k == 0:                               # the scalar sits on the first core
                core[:, :, 0, :] = np.transpose(blk * np.asarray(self.coef)[:, None, None], (1, 2, 0))
            elif k == N - 1:
                core[:, :, :, 0] = np.transpose(blk, (1, 2, 0))
            else:
                idx = np.arange(P)
                core[:, :, idx, idx] = np.transpose(blk, (1, 2, 0))
            vec.append(core)
        rks = [1] + [P] * (N - 1) + [1]
        return TToperator(N, vec, (2,) * N, rks)


# ------------------------------------------------------------------ operator sums and rounding
def tto_add(A: TToperator, B: TToperator) -> TToperator:
    """+(A, B) for TToperators, src/tt_operations.jl:121-148 (ranks add, block diagonal)."""
    d = A.N
    rks = [a + b for a, b in zip(A.tto_rks, B.tto_rks)]
    rks[0] = rks[d] = 1
    vec = []
    for k in range(d):
        n = A.tto_dims[k]
        c = np.zeros((n, n, rks[k], rks[k + 1]), order="F")
        a, b = A.tto_vec[k], B.tto_vec[k]
        if d == 1:
            c[...] = a + b
        elif k == 0:
            c[:, :, :, : a.shape[3]] = a
            c[:, :, :, a.shape[3]:] = b
        elif k == d - 1:
            c[:, :, : a.shape[2], :] = a
            c[:, :, a.shape[2]:, :] = b
        else:
            c[:, :, : a.shape[2], : a.shape[3]] = a
            c[:, :, a.shape[2]:, a.shape[3]:] = b
        vec.append(c)
    return TToperator(d, vec, A.tto_dims, rks)


def tto_to_ttv(A: TToperator) -> TTvector:
    """src/tt_tools.jl:603-611: the TTvector with modes n^2 sharing the cores' memory order."""
    vec = [c.reshape(c.shape[0] * c.shape[1], c.shape[2], c.shape[3], order="F") for c in A.tto_vec]
    return TTvector(A.N, vec, tuple(n * n for n in A.tto_dims), A.tto_rks, A.tto_ot)


def ttv_to_tto(x: TTvector) -> TToperator:
    """src/tt_tools.jl:616-626."""
    n = [int(round(np.sqrt(m))) for m in x.ttv_dims]
    vec = [c.reshape(nk, nk, c.shape[1], c.shape[2], order="F") for c, nk in zip(x.ttv_vec, n)]
    return TToperator(x.N, vec, tuple(n), x.ttv_rks, x.ttv_ot)


def tt_rounding_tto(A: TToperator, tol: float = 1e-12, rmax: int = 2 ** 14) -> TToperator:
    """tt_rounding(::TToperator), src/tt_rounding.jl:275-277, on the GPU."""
    return ttv_to_tto(tt_rounding(tto_to_ttv(A), tol=tol, rmax=rmax))


def tt_rounding_tto_batch(As: Sequence[TToperator], tol: float = 1e-12, rmax: int = 2 ** 14) -> List[TToperator]:
    """tt_rounding of many TToperators of the same sites, in one batched device call."""
    if not As:
        return []
    if len(As) == 1:
        return [tt_rounding_tto(As[0], tol=tol, rmax=rmax)]
    vs = [tto_to_ttv(A) for A in As]
    ctx = get_context()
    xb = DeviceBatch.from_tts(vs, ctx=ctx)
    yb = DeviceBatch(vs[0].ttv_dims, [v.ttv_rks for v in vs], ctx=ctx)
    xb.round_det(yb, tol=tol, rmax=rmax)
    out = [ttv_to_tto(y) for y in yb.download()]
    xb.close()
    yb.close()
    return out


# ------------------------------------------------------------------ the Hamiltonian terms
def _nonzero_indices(T: np.ndarray, atol: float = 1e-12):
    """Julia findall(x -> !isapprox(x, 0, atol=atol), T): column-major order, 1-based."""
    idx = np.argwhere(np.abs(np.transpose(T, tuple(range(T.ndim))[::-1])) > atol)
    return [tuple(int(v) + 1 for v in row[::-1]) for row in idx]


def _hV_terms(h, V, N: int, chemistry: bool) -> List[_RankOneSum]:
    """The scaled terms of hV_to_mpo / hV_to_mpo_tree (src/models.jl:193-224, :263-300), in the
    order Julia's findall visits h then V; each a sum of one or two rank-1 operators."""
    terms = []

    def term(c, *chains):
        t = _RankOneSum(N)
        for ch in chains:
            t.add(c, _chain_factors(ch, N))
        terms.append(t)

    for a, b in _nonzero_indices(h):
        if a < b:
            term(h[a - 1, b - 1], [("c", a), ("a", b)], [("c", b), ("a", a)])
        elif a == b:
            term(h[a - 1, b - 1], [("c", a), ("a", b)])
    for i1, i2, i3, i4 in _nonzero_indices(V):
        v = V[i1 - 1, i2 - 1, i3 - 1, i4 - 1]
        if chemistry:
            if (i1, i3) < (i2, i4):
                term(v / 2, [("c", i1), ("c", i3), ("a", i4), ("a", i2)], [("c", i2), ("c", i4), ("a", i3), ("a", i1)])
            elif (i1, i3) == (i2, i4):
                term(v / 2, [("c", i1), ("c", i3), ("a", i4), ("a", i2)])
        else:
            if (i1, i2) < (i4, i3):
                term(v, [("c", i1), ("c", i2), ("a", i3), ("a", i4)], [("c", i4), ("c", i3), ("a", i2), ("a", i1)])
            elif (i1, i2) == (i4, i3):
                term(v, [("c", i1), ("c", i2), ("a", i3), ("a", i4)])
    return terms


def zeros_tto(dims, rks) -> TToperator:
    """src/tt_tools.jl:145-160."""
    N = len(dims)
    return TToperator(N, [np.zeros((dims[k], dims[k], rks[k], rks[k + 1]), order="F") for k in range(N)], dims, rks)


def hV_to_mpo(h, V, dims, tol: float = 1e-8, n_rnd: int = 20, chemistry: bool = False) -> TToperator:
    """src/models.jl:180-231: the running sum rounded after every n_rnd + 1 terms, and at the
    end, each rounding on the GPU."""
    h = np.asarray(h, dtype=np.float64)
    N = len(dims)
    if not np.allclose(h, h.T):
        raise ValueError("hV_to_mpo: h must be symmetric")
    A = zeros_tto(tuple(dims), [1] * (N + 1))
    i_rnd = 1
    for t in _hV_terms(h, V, N, chemistry):
        A = tto_add(A, t.tto())
        if i_rnd > n_rnd:
            A = tt_rounding_tto(A, tol=tol)
            i_rnd = 1
        else:
            i_rnd += 1
    return tt_rounding_tto(A, tol=tol)


def hV_to_mpo_tree(h, V, dims, tol: float = 1e-8, n_leaf: int = 20, n_branch: int = 8,
                   chemistry: bool = False) -> TToperator:
    """src/models.jl:254-338: leaf groups of n_leaf terms summed and rounded (all leaves of the
    tree in one batched device call), then merges of n_branch operators, rounded level by level
    (one batched call per level), until one MPO remains."""
    h = np.asarray(h, dtype=np.float64)
    N = len(dims)
    if not np.allclose(h, h.T):
        raise ValueError("hV_to_mpo_tree: h must be symmetric")
    terms = _hV_terms(h, V, N, chemistry)
    if not terms:
        return zeros_tto(tuple(dims), [1] * (N + 1))
    leaves = []
    for g0 in range(0, len(terms), n_leaf):
        s = _RankOneSum(N)
        for t in terms[g0: g0 + n_leaf]:
            s.extend(t)
        leaves.append(s.tto())
    current = tt_rounding_tto_batch(leaves, tol=tol)
    while len(current) > 1:
        merged = []
        for g0 in range(0, len(current), n_branch):
            A = current[g0]
            for B in current[g0 + 1: g0 + n_branch]:
                A = tto_add(A, B)
            merged.append(A)
        current = tt_rounding_tto_batch(merged, tol=tol)
    return current[0]


# ------------------------------------------------------------------ models (h, V)
def hubbard_1D(L: int, t: float = 1.0, U: float = 1.0, pbc: bool = False):
    """src/models.jl:403-419 (spin-orbitals 2i-1 up, 2i down; returns Symmetric(h), V)."""
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
    return np.triu(h) + np.triu(h, 1).T, V


def hubbard_2D(w: int, L: int, t: float = 1.0, U: float = 1.0, w_pbc: bool = False, L_pbc: bool = True):
    """src/models.jl:431-476: w x L lattice, site s = j*w + i, spin-orbitals 2s+1 (up), 2s+2."""
    n = 2 * w * L
    h = np.zeros((n, n))
    V = np.zeros((n,) * 4)

    def onsite(s):
        V[2 * s, 2 * s + 1, 2 * s, 2 * s + 1] = -U
        V[2 * s + 1, 2 * s, 2 * s + 1, 2 * s] = -U

    def hop(s, u):
        h[2 * s, 2 * u] = -t
        h[2 * s + 1, 2 * u + 1] = -t

    for i in range(w - 1):
        for j in range(L - 1):
            onsite(j * w + i)
            hop(j * w + i, (j + 1) * w + i)
            hop(j * w + i, j * w + i + 1)
        onsite((L - 1) * w + i)
        hop((L - 1) * w + i, (L - 1) * w + i + 1)
        if L_pbc and L > 2:
            hop(L * w + i - w, i)
    for j in range(L - 1):
        onsite(j * w + w - 1)
        hop(j * w + w - 1, (j + 1) * w + w - 1)
        if w_pbc and w > 2:
            hop(j * w + w - 1, j * w)
    onsite(L * w - 1)
    if L_pbc and L > 2:
        hop(L * w - 1, w - 1)
    if w_pbc and w > 2:
        hop(L * w - 1, (L - 1) * w)
    return np.triu(h) + np.triu(h, 1).T, V


def snake_order(w: int, L: int) -> np.ndarray:
    """0-based spin-orbital order of a snake traversal of the w x L lattice (columns j with odd j
    reversed in i), applied as h[sigma][:, sigma] the way the reference's examples permute
    orbitals (examples/hubbard_2d_orderings.jl:12-15)."""
    sigma = []
    for j in range(L):
        col = [j * w + i for i in range(w)]
        for s in (col[::-1] if j % 2 == 1 else col):
            sigma += [2 * s, 2 * s + 1]
    return np.array(sigma)


def one_e_two_e_integrals_to_hV(int1e, int2e):
    """src/models.jl:529-549: spatial-orbital integrals to spin-orbital h (2L x 2L) and V."""
    L = int1e.shape[0]
    h = np.zeros((2 * L, 2 * L))
    V = np.zeros((2 * L,) * 4)
    up = np.arange(L) * 2
    dn = up + 1
    h[np.ix_(up, up)] = int1e
    h[np.ix_(dn, dn)] = int1e
    for a, b in ((up, up), (dn, dn), (dn, up), (up, dn)):
        V[np.ix_(a, a, b, b)] = int2e
    return h, V


def synthetic_molecular_integrals(L: int, seed: int, decay: float = 4.0):
    """Seeded synthetic integrals of L spatial orbitals: h_ij = h_ji ~ N(0,1) exp(-|i-j|/decay),
    V_ijkl ~ N(0,1) symmetrised over the 8 permutations of real two-electron integrals and scaled
    by exp(-(|i-j| + |k-l|)/decay)."""
    g = np.random.default_rng(seed)
    i = np.arange(L)
    h = g.standard_normal((L, L)) * np.exp(-np.abs(i[:, None] - i[None, :]) / decay)
    h = np.triu(h) + np.triu(h, 1).T
    V = g.standard_normal((L,) * 4)
    V = (V + V.transpose(1, 0, 2, 3) + V.transpose(0, 1, 3, 2) + V.transpose(1, 0, 3, 2)
         + V.transpose(2, 3, 0, 1) + V.transpose(3, 2, 0, 1) + V.transpose(2, 3, 1, 0) + V.transpose(3, 2, 1, 0)) / 8.0
    dij = np.abs(i[:, None] - i[None, :])
    return h, V * np.exp(-(dij[:, :, None, None] + dij[None, None, :, :]) / decay)
