"""Krylov callers of the rounding path (src/tt_solvers.jl, src/sketches.jl:617-1038), on the GPU.

The reference's eigensolvers build Krylov bases of TTvectors whose every new vector is a
randomized rounding of a linear combination (with one operator term), and its sketched
Rayleigh-Ritz solver works on boundary sketches of those vectors.  These mirrors keep the
reference's algorithms, arguments and return values; every TT operation (operator apply, sums,
inner products, norms, sketches, both roundings) runs in libttcuda, and only the small dense
matrices (Hessenberg, sketch coefficients, Ritz problems) stay on the host, as in the reference.

Deviations, each forced by a reference behaviour that cannot be reproduced as written:
* expand_basis recomputes the sketches of the window vectors inside the operator rounding
  instead of reusing the stored ones; with the same seed and ranks both are the same sketch of
  the same vectors (the reference rescales the stored sketch levels exactly as the scalar
  division rescales the vector), so the result is the same.
* sketched_rr takes the seed of its sampled residual as an argument (the reference draws it with
  rand(Int)).  When its rounding at tol = res^2 / 2 returns the zero TT, the zero TT is returned
  with a NaN sampled residual (the reference divides by the zero norm).
* arnoldi stops at a breakdown (zero norm after rounding) instead of dividing by zero.
* eig_arnoldi restarts from the rounded Ritz vector with sketch ranks twice its ranks and
  boundary ranks 1; the reference's call passes `rks=` as a keyword that no ttrand_rounding
  method accepts, with boundary ranks 2, and re-runs Arnoldi from the previous start vector.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import (ArgumentError, TToperator, TTvector, dot, dot_operator, mpo_apply, norm, tt_add, tt_recursive_sketch,
               tt_rounding, tt_scale, ttrand_rounding, ttrand_rounding_lincomb, ttrand_rounding_op)


# ------------------------------------------------------------------------------- sketches
def _block_ranks(dims, block_rks) -> List[int]:
    """Block ranks of the reverse sketch (src/sketches.jl:652-662)."""
    N = len(dims)
    b = [block_rks] * N + [1]
    for k in range(N - 1, -1, -1):
        b[k] = min(b[k], dims[k] * b[k + 1])
    return b


def tt_sketch(A: TTvector, s: int, H: Optional[TToperator] = None, orthogonal=True, seed=1234, block_rks=None,
              precision="fp64") -> Tuple[np.ndarray, int]:
    """tt_sketch (src/sketches.jl:645-727; with H, :729-817), reverse=true: the boundary sketch of
    A (or H A) with p = ceil(s / b_1) sketch blocks on every core.  That is the recursive
    sketch whose ranks are b_k p at every bond, of which only the boundary level is kept.
    Returns (vector of b_1 p entries, b_1 p)."""
    N = A.N
    b = _block_ranks(A.ttv_dims, N if block_rks is None else block_rks)
    p = int(math.ceil(s / b[0]))
    rks = [bk * p for bk in b[:N]] + [1]
    W, srk = tt_recursive_sketch(A, rks, H=H, orthogonal=orthogonal, seed=seed, block_rks=block_rks,
                                 precision=precision)
    if srk[0] != b[0] * p:
        raise RuntimeError("tt_sketch: unexpected boundary sketch rank")
    return W[0].ravel(order="F"), b[0] * p


def tt_combined_sketch(A: TTvector, rks_or_rmax, s: int, H: Optional[TToperator] = None, orthogonal=True, seed=1234,
                       block_rks=None, precision="fp64"):
    """tt_combined_sketch (src/sketches.jl:930-1000), reverse=true: the recursive sketch at rks
    with the boundary rank raised to min(s, rks[2]), extended by a tt_sketch with seed + 1 when
    s is larger.  Returns (boundary sketch, W with W[0] = ones, sketch_rks with sketch_rks[0] = 1)."""
    N = A.N
    if isinstance(rks_or_rmax, (int, np.integer)):
        rks = [int(rks_or_rmax)] * (N + 1)
        rks[N] = 1
    else:
        rks = [int(r) for r in rks_or_rmax]
    rks[0] = max(rks[0], min(s, rks[1]))
    W, srk = tt_recursive_sketch(A, rks, H=H, orthogonal=orthogonal, seed=seed, block_rks=block_rks,
                                 precision=precision)
    sketch = W[0].ravel(order="F")
    s_rec = srk[0]
    if s > s_rec:
        extra, _ = tt_sketch(A, s - s_rec, H, orthogonal, seed + 1, block_rks, precision)
        tot = s_rec + len(extra)
        sketch = np.concatenate([math.sqrt(len(sketch) / tot) * sketch, math.sqrt(len(extra) / tot) * extra])
    W[0] = np.ones((1, 1)) if H is None else np.ones((1, 1, 1))
    srk[0] = 1
    return sketch, W, srk


def _root(x: TTvector) -> int:
    """The core that scalar multiplication scales: the first with ot == 0 (src/tt_operations.jl:428-441)."""
    ot = list(x.ttv_ot)
    if 0 not in ot:
        raise ArgumentError("the TTvector has no non-orthogonal core to scale")
    return ot.index(0)


def _rescale_sketch(W, x: TTvector, beta: float) -> None:
    """W[i] /= beta for the sketch levels that contain the scaled core (the reference's
    `for i = 2:findfirst(isequal(0), x.ttv_ot)`)."""
    for i in range(1, _root(x) + 1):
        W[i] = W[i] / beta


# ------------------------------------------------------------------------- Arnoldi
def dot_randrounding(A: TToperator, x: TTvector) -> TTvector:
    """dot_randrounding (src/tt_randtools.jl:476-480): A x formed, randomized rounding with the
    default sketch ranks, then tt_rounding(tol=1e-8)."""
    y = mpo_apply(A, x)
    y = ttrand_rounding(y)
    return tt_rounding(y, tol=1e-8)


def _sub(w: TTvector, a: float, v: TTvector) -> TTvector:
    """w - a v as the reference forms it: -(w, a v) = (-1)(a v) + w (src/tt_operations.jl:453-455)."""
    return tt_add(tt_scale(-1.0, tt_scale(a, v)), w)


def arnoldi(A: TToperator, m: int, V: Sequence[TTvector], eps_tt: float = 1e-6, rmax: int = 256
            ) -> Tuple[np.ndarray, List[TTvector], float]:
    """arnoldi (src/tt_solvers.jl:206-224): m steps of Arnoldi with modified Gram-Schmidt from
    V[0]; every new vector is rounded by ttrand_rounding (default ranks) and
    tt_rounding(tol=eps_tt, rmax).  Returns the Hessenberg matrix, the basis and H[m, m-1].  A
    breakdown after j + 1 vectors returns the (j + 1) x (j + 1) matrix, those vectors and 0."""
    Hh = np.zeros((m + 1, m + 1))
    V = [tt_scale(1.0 / norm(V[0]), V[0])]
    for j in range(m):
        w = dot_randrounding(A, V[j])
        for i in range(j + 1):
            Hh[i, j] = dot(V[i], w)                      # modified Gram-Schmidt
            w = _sub(w, Hh[i, j], V[i])
        w = ttrand_rounding(w)
        w = tt_rounding(w, tol=eps_tt, rmax=rmax)
        Hh[j + 1, j] = norm(w)
        if Hh[j + 1, j] == 0.0:
            return Hh[: j + 1, : j + 1], V, 0.0
        V.append(tt_scale(1.0 / Hh[j + 1, j], w))
    return Hh[:m, :m], V, float(Hh[m, m - 1])


def eig_arnoldi(A: TToperator, m: int, v: TTvector, Imax: int = 100, eps: float = 1e-6, eps_tt: float = 1e-4,
                rmax: int = 256, which: str = "LM", sigma: float = 0.0, history: bool = False):
    """eig_arnoldi (src/tt_solvers.jl:226-265): restarted Arnoldi for the eigenvalue of largest
    ("LM") or smallest (any other `which`) magnitude of A + sigma I.  Returns (eigenvalue, TT
    eigenvector, residual history ||A v - lambda v|| when history=True)."""
    def ritz(Hh):
        vals, vecs = np.linalg.eig(Hh + sigma * np.eye(Hh.shape[0]))
        k = int(np.argmax(np.abs(vals)) if which == "LM" else np.argmin(np.abs(vals)))
        f = vecs[:, k]
        if np.iscomplexobj(f) and np.abs(f.imag).max() > 1e-12 * max(np.abs(f.real).max(), 1e-300):
            raise ArgumentError("eig_arnoldi: complex Ritz vector (the device path is real)")
        return vals[k], np.real(f)

    def restart(V, f, v):
        rks = [1] + [2 * r for r in v.ttv_rks[1:-1]] + [1]
        u = ttrand_rounding_lincomb(list(f), V[: len(f)], rks)
        return tt_rounding(u, tol=eps_tt, rmax=rmax)

    Hh, V, h = arnoldi(A, m, [v], rmax=2 * rmax)
    lam, f = ritz(Hh)
    v = restart(V, f, v)
    hist = []
    i = 1
    while i < Imax and abs(h) > eps:
        Hh, V, h = arnoldi(A, m, [v], eps_tt=eps_tt, rmax=2 * rmax)
        lam, f = ritz(Hh)
        v = restart(V, f, v)
        if history:
            hist.append(norm(_sub(mpo_apply(A, v), float(np.real(lam)) - sigma, v)))
        i += 1
    return float(np.real(lam) - sigma), v, hist


# ---------------------------------------------------------- sketched Rayleigh-Ritz
def expand_basis(H: TToperator, B_window: List[TTvector], W_B_window: List[list], B_sketch_window: List[np.ndarray],
                 rmax: int, s: int, orthogonal=True, block_rks=8, seed=1234, k_trunc=None, precision="fp64"):
    """expand_basis! (src/tt_solvers.jl:354-452): the next vector of a sketch-orthogonal Krylov
    basis, b = H b_prev - sum_l h_l b_l with h the sketched Gram-Schmidt coefficients,
    randomized-rounded at sketch rank 2 rmax and rounded to rmax, then normalised by its sketch.
    The three windows are mutated as in the reference (appended, oldest dropped beyond k_trunc).
    Returns (b_new, sketch of b_new, sketch of H b_prev)."""
    k_trunc = len(B_window) if k_trunc is None else k_trunc
    b_prev = B_window[-1]
    N = b_prev.N
    sketch_Hb, _, _ = tt_combined_sketch(b_prev, 2 * rmax, s, H, orthogonal, seed, block_rks, precision)
    h = np.linalg.lstsq(np.column_stack(B_sketch_window), sketch_Hb, rcond=None)[0]
    rks = [2 * rmax] * N + [1]                 # the ranks of tt_combined_sketch(.., 2 rmax, s)
    y = ttrand_rounding_op([1.0] + [-float(c) for c in h], H, [b_prev] + list(B_window), rks,
                           orthogonal=orthogonal, seed=seed, block_rks=block_rks, precision=precision)
    b_new = tt_rounding(y, rmax=rmax)
    sk_new, W_new, _ = tt_combined_sketch(b_new, 2 * rmax, s, None, orthogonal, seed, block_rks, precision)
    beta = float(np.linalg.norm(sk_new))
    sk_new = sk_new / beta
    _rescale_sketch(W_new, b_new, beta)
    b_new = tt_scale(1.0 / beta, b_new)
    for win, item in ((B_window, b_new), (B_sketch_window, sk_new), (W_B_window, W_new)):
        win.append(item)
        if len(win) > k_trunc:
            win.pop(0)
    return b_new, sk_new, sketch_Hb


def _sort_eig(vals, vecs):
    """Julia's eigen order: ascending by (real, imag)."""
    idx = sorted(range(len(vals)), key=lambda i: (vals[i].real, vals[i].imag))
    return vals[idx], vecs[:, idx]


def sketched_rr(H: TToperator, B: Sequence[TTvector], C: np.ndarray, D: np.ndarray, rmax: int, orthogonal=True,
                block_rks=8, seed=1234, kappa_max=None, stable=False, sample_seed=4321, precision="fp64"):
    """sketched_rr (src/tt_solvers.jl:469-514): stable sketched Rayleigh-Ritz (Tropp and
    Nakatsukasa 2022) on the basis B with C = Omega B and D = Omega H B.  Returns (Ritz values
    ascending, Ritz vector X of the lowest, sketched residual ||D y - lambda C y||, sampled
    residual ||S(H X) - lambda S(X)|| / ||S(X)|| with a sketch of 2N entries)."""
    N = B[0].N
    if stable:
        kappa_max = 1.0 / math.sqrt(np.finfo(float).eps) if kappa_max is None else kappa_max
        U, sig, Vt = np.linalg.svd(C, full_matrices=False)
        keep = np.nonzero(sig / sig[0] > 1.0 / kappa_max)[0]
        k = int(keep[-1]) + 1 if len(keep) else 1
        Vk = Vt[:k].T
        M = U[:, :k].T @ D @ Vk
        # generalized problem M z = lambda diag(sig) z, as a standard one (diag(sig) is invertible)
        lam, Z = np.linalg.eig(M / sig[:k, None])
        lam, Z = _sort_eig(lam, Z)
        Yv = np.real(Vk @ Z)
        for j in range(k):
            Yv[:, j] /= np.linalg.norm(C @ Yv[:, j])
    else:
        M = np.linalg.lstsq(C, D, rcond=None)[0]          # C \ D (C has full column rank)
        lam, Yv = np.linalg.eig(M)
        lam, Yv = _sort_eig(lam, Yv)
        Yv = np.real(Yv)
    lam = np.real(lam)
    res_sketch = float(np.linalg.norm(D @ Yv[:, 0] - lam[0] * (C @ Yv[:, 0])))
    y = Yv[:, 0] / np.linalg.norm(Yv[:, 0])
    X = ttrand_rounding_lincomb(list(y), list(B), 4 * rmax, orthogonal=orthogonal, seed=seed, block_rks=block_rks,
                                precision=precision)
    X = tt_rounding(X, tol=res_sketch ** 2 / 2)
    nx = norm(X)
    if nx == 0.0:
        return lam, X, res_sketch, float("nan")
    X = tt_scale(1.0 / nx, X)
    S1, _ = tt_sketch(X, 2 * N, H, orthogonal, sample_seed, block_rks, precision)
    S2, _ = tt_sketch(X, 2 * N, None, orthogonal, sample_seed, block_rks, precision)
    res_sample = float(np.linalg.norm(S1 - lam[0] * S2) / np.linalg.norm(S2))
    return lam, X, res_sketch, res_sample


def sketched_rayleigh_ritz(H: TToperator, b0: TTvector, d: int, rmax: int, orthogonal=True, block_rks=8, seed=1234,
                           sketch_size=None, k_trunc=None, e_nuc=0.0, sample_seed=4321, precision="fp64"):
    """sketched_rayleigh_ritz (src/tt_solvers.jl:547-618): a d-dimensional sketch-orthogonal Krylov
    basis from b0 with a sketched Rayleigh-Ritz solve after every expansion (the j-th samples its
    residual with seed sample_seed + j).  Returns (lowest Ritz value + e_nuc, its Ritz vector,
    history of dicts iter / e_sketch / e_true / res_sketch / res_sample)."""
    sketch_size = 4 * d if sketch_size is None else sketch_size
    k_trunc = d - 1 if k_trunc is None else k_trunc
    B: List[TTvector] = [None] * d
    sk_b: List[np.ndarray] = [None] * d
    sk_Hb: List[np.ndarray] = [None] * d
    sk0, W1, _ = tt_combined_sketch(b0, 2 * rmax, sketch_size, None, orthogonal, seed, block_rks, precision)
    s = len(sk0)
    beta = float(np.linalg.norm(sk0))
    sk_b[0] = sk0 / beta
    _rescale_sketch(W1, b0, beta)
    B[0] = tt_scale(1.0 / beta, b0)
    Bw, Ww, Sw = [B[0]], [W1], [sk_b[0]]
    hist = []

    def solve(j):
        lam, psi, rs, rsam = sketched_rr(H, B[:j], np.column_stack(sk_b[:j]), np.column_stack(sk_Hb[:j]), rmax,
                                         orthogonal, block_rks, seed, sample_seed=sample_seed + j, precision=precision)
        e_true = dot_operator(psi, H, psi) + e_nuc if norm(psi) > 0.0 else float("nan")
        hist.append(dict(iter=j, e_sketch=float(lam[0]) + e_nuc, e_true=e_true, res_sketch=rs, res_sample=rsam))
        return float(lam[0]) + e_nuc, psi

    for j in range(1, d):
        B[j], sk_b[j], sk_Hb[j - 1] = expand_basis(H, Bw, Ww, Sw, rmax, s, orthogonal, block_rks, seed, k_trunc,
                                                   precision)
        solve(j)
    sk_Hb[d - 1], _, _ = tt_combined_sketch(B[d - 1], 2 * rmax, s, H, orthogonal, seed, block_rks, precision)
    e, psi = solve(d)
    return e, psi, hist


def sketched_rayleigh_ritz_schedule(H: TToperator, b0: TTvector, schedule: Sequence[dict], orthogonal=True,
                                    block_rks=8, seed=1234, e_nuc=0.0, sample_seed=4321, precision="fp64"):
    """sketched_rayleigh_ritz(H, b0, schedule) (src/tt_solvers.jl:649-688): one stage per schedule
    entry (keys d, rmax; optional seed, sketch_size, k_trunc, label), each restarted from the
    previous stage's Ritz vector rounded to the new rmax.  Returns (lambda, psi, [(label,
    history)], seeds used).  The reference's validate_seed loop, which redraws seeds with
    rand(Int), is left out."""
    psi, lam = b0, 0.0
    stages, seeds = [], []
    for i, st in enumerate(schedule):
        d, rmax = int(st["d"]), int(st["rmax"])
        s = int(st.get("seed", seed + i))
        sk = int(st.get("sketch_size", 4 * d))
        kt = int(st.get("k_trunc", d - 1))
        lbl = st.get("label", f"d={d}, rmax={rmax}")
        b_init = psi if i == 0 else tt_rounding(psi, rmax=rmax)
        seeds.append(s)
        lam, psi, hist = sketched_rayleigh_ritz(H, b_init, d, rmax, orthogonal, block_rks, s, sk, kt, e_nuc,
                                                sample_seed, precision)
        stages.append((lbl, hist))
    return lam, psi, stages, seeds
