"""FP64 CPU restatement of the Krylov callers of the rounding path -- TEST INFRASTRUCTURE.

The oracle of ttcuda.solvers: only tests/ may import it; the product never does.  Each
function restates the reference function cited beside it, on the primitives of tt_oracle:

  tt_sketch               src/sketches.jl:645-727 (TT), :729-817 (operator); reverse=true
  tt_combined_sketch      src/sketches.jl:930-1000
  expand_basis            src/tt_solvers.jl:354-452 (the reference form: stored sketches W_B)
  sketched_rr             src/tt_solvers.jl:469-514
  sketched_rayleigh_ritz  src/tt_solvers.jl:547-618
  dot_randrounding        src/tt_randtools.jl:476-480
  arnoldi, eig_arnoldi    src/tt_solvers.jl:206-265

Sketch blocks come from the same Philox streams as every other oracle sketch (SketchRNG).
The sampled-residual seed that the reference draws with rand(Int) is an argument here, so that
the GPU mirror and this restatement see the same sketch.  Parity: pinned through tt_oracle's
pins (the reference ships no tests for these functions); the tests check this restatement
against the dense eigenproblem and the GPU mirror against this restatement.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np
import scipy.linalg as sla

from . import tt_oracle as o

F = "F"


def _sort_eig(vals, vecs):
    """Julia's eigen order (LinearAlgebra eigsortby): ascending by (real, imag)."""
    idx = sorted(range(len(vals)), key=lambda i: (vals[i].real, vals[i].imag))
    return vals[idx], vecs[:, idx]


def tt_sketch(A: o.TTvector, s: int, H: Optional[o.TToperator] = None, orthogonal=True, seed=1234, block_rks=None,
              rng_kind="philox"):
    """src/sketches.jl:645-727 / :729-817 (reverse): boundary sketch only, with the block count
    p = ceil(s / b_1) on every core.  Returns (vector of length b_1 p, b_1 p)."""
    N, dims = A.N, A.ttv_dims
    b = o.reverse_block_ranks(dims, N, N if block_rks is None else block_rks)
    p = int(math.ceil(s / b[0]))
    rng = o.SketchRNG(seed, rng_kind)
    Wp = np.ones((1, 1, 1)) if H is None else np.ones((1, 1, 1, 1))
    for k in range(N - 1, -1, -1):
        B = o.generate_sketch_blocks(rng, k, b[k + 1], dims[k], b[k], p, orthogonal)
        if H is None:
            Wc = np.zeros((A.ttv_rks[k], b[k], p))
            for j in range(p):
                Wc[:, :, j] = o.contract_sketch_core_backwards(A.ttv_vec[k], B[:, :, :, j],
                                                               Wp[:, :, j if k < N - 1 else 0])
        else:
            Wc = np.zeros((A.ttv_rks[k], H.tto_rks[k], b[k], p))
            for j in range(p):
                Wc[:, :, :, j] = o.contract_sketch_core_backwards_op(A.ttv_vec[k], H.tto_vec[k], B[:, :, :, j],
                                                                     Wp[:, :, :, j if k < N - 1 else 0])
        Wp = Wc
    Wp = Wp / math.sqrt(p)
    return Wp.ravel(order=F), b[0] * p


def tt_combined_sketch(A: o.TTvector, rks_or_rmax, s: int, H: Optional[o.TToperator] = None, orthogonal=True,
                       seed=1234, block_rks=None, rng_kind="philox"):
    """src/sketches.jl:930-1000 (reverse): the recursive sketch at rks with the boundary rank
    raised to min(s, rks[2]), plus a tt_sketch with seed+1 when s exceeds it.  Returns
    (boundary sketch, W with W[0] = ones, sketch_rks with sketch_rks[0] = 1)."""
    N = A.N
    if isinstance(rks_or_rmax, (int, np.integer)):
        rks = [int(rks_or_rmax)] * (N + 1)
        rks[N] = 1
    else:
        rks = [int(r) for r in rks_or_rmax]
    rks[0] = max(rks[0], min(s, rks[1]))
    if H is None:
        W, srk = o.tt_recursive_sketch(A, rks, orthogonal, seed, block_rks, rng_kind=rng_kind)
    else:
        W, srk = o.tt_recursive_sketch_op(H, A, rks, orthogonal, seed, block_rks, rng_kind=rng_kind)
    sketch = W[0].ravel(order=F)
    s_rec = srk[0]
    if s > s_rec:
        extra, _ = tt_sketch(A, s - s_rec, H, orthogonal, seed + 1, block_rks, rng_kind)
        tot = s_rec + len(extra)
        sketch = np.concatenate([math.sqrt(len(sketch) / tot) * sketch, math.sqrt(len(extra) / tot) * extra])
    W[0] = np.ones((1, 1)) if H is None else np.ones((1, 1, 1))
    srk = list(srk)
    srk[0] = 1
    return sketch, W, srk


def _rescale_upto_root(W, x: o.TTvector, beta: float):
    """W[i] /= beta for the sketch levels 2:findfirst(ot .== 0) (Julia indices): the levels whose
    contraction includes the core that x / beta scales (src/tt_operations.jl:428-441)."""
    f = x.ttv_ot.index(0) if 0 in list(x.ttv_ot) else None
    if f is None:
        raise ValueError("the TTvector has no non-orthogonal core to scale")
    for i in range(1, f + 1):
        W[i] = W[i] / beta


def expand_basis(H: o.TToperator, B_window: List[o.TTvector], W_B_window: List[list], B_sketch_window: List[np.ndarray],
                 rmax: int, s: int, orthogonal=True, block_rks=8, seed=1234, k_trunc=None, rng_kind="philox"):
    """src/tt_solvers.jl:354-452: one sketch-orthogonal Krylov step, reusing the stored sketches
    W_B of the window; mutates the three windows.  Returns (b_new, sketch_b_new, sketch_Hb_prev)."""
    k_trunc = len(B_window) if k_trunc is None else k_trunc
    b_prev = B_window[-1]
    N, dims = b_prev.N, b_prev.ttv_dims
    sketch_Hb, WHb, s_rks = tt_combined_sketch(b_prev, 2 * rmax, s, H, orthogonal, seed, block_rks, rng_kind)
    W_HB = [WHb[k].reshape(b_prev.ttv_rks[k] * H.tto_rks[k], s_rks[k], order=F) for k in range(N + 1)]
    Cw = np.column_stack(B_sketch_window)
    h = np.linalg.lstsq(Cw, sketch_Hb, rcond=None)[0]
    m = 1 + len(B_window)
    vec = [None] * N
    out = [1] * (N + 1)
    ot = [0] * N
    b1 = b_prev.ttv_vec[0].reshape(dims[0], b_prev.ttv_rks[1], order=F)
    H1 = H.tto_vec[0].reshape(dims[0], dims[0], H.tto_rks[1], order=F)
    Ay1 = np.einsum("ijb,ja->iab", H1, b1)
    Y = [Ay1.reshape(dims[0], 1, b_prev.ttv_rks[1] * H.tto_rks[1], order=F)]
    for i, b in enumerate(B_window):
        Y.append(-h[i] * b.ttv_vec[0])
    for k in range(N - 1):
        Z = np.einsum("iab,bc->iac", Y[0], W_HB[k + 1])
        for i, W in enumerate(W_B_window):
            Z += np.einsum("iab,bc->iac", Y[1 + i], W[k + 1])
        Q, _ = o.qr_julia(Z.reshape(dims[k] * out[k], s_rks[k + 1], order=F))
        out[k + 1] = Q.shape[1]
        vec[k] = Q.reshape(dims[k], out[k], out[k + 1], order=F)
        ot[k] = 1
        y1 = Y[0].reshape(dims[k], out[k], b_prev.ttv_rks[k + 1], H.tto_rks[k + 1], order=F)
        Ay = o.ein("irab,irs,jac,ljbd->lscd", y1, vec[k], b_prev.ttv_vec[k + 1], H.tto_vec[k + 1])
        new = [Ay.reshape(dims[k + 1], out[k + 1], b_prev.ttv_rks[k + 2] * H.tto_rks[k + 2], order=F)]
        for i, b in enumerate(B_window):
            new.append(o.ein("iab,iac,jbd->jcd", Y[1 + i], vec[k], b.ttv_vec[k + 1]))
        Y = new
    vec[N - 1] = sum(Y).reshape(dims[N - 1], out[N - 1], 1, order=F)
    b_new = o.tt_rounding(o.TTvector(N, vec, tuple(dims), out, ot), rmax=rmax)
    sk_new, W_new, _ = tt_combined_sketch(b_new, 2 * rmax, s, None, orthogonal, seed, block_rks, rng_kind)
    beta = float(np.linalg.norm(sk_new))
    sk_new = sk_new / beta
    _rescale_upto_root(W_new, b_new, beta)
    b_new = o.tt_scale(1.0 / beta, b_new)
    for win, item in ((B_window, b_new), (B_sketch_window, sk_new), (W_B_window, W_new)):
        win.append(item)
        if len(win) > k_trunc:
            win.pop(0)
    return b_new, sk_new, sketch_Hb


def sketched_rr(H: o.TToperator, B: Sequence[o.TTvector], C: np.ndarray, D: np.ndarray, rmax: int, orthogonal=True,
                block_rks=8, seed=1234, kappa_max=None, stable=False, sample_seed=4321, rng_kind="philox"):
    """src/tt_solvers.jl:469-514: sketched Rayleigh-Ritz on the basis B with C = Omega B and
    D = Omega H B.  Returns (Ritz values ascending, Ritz vector X, sketched residual, sampled
    residual)."""
    d = len(B)
    N = B[0].N
    if stable:
        kappa_max = 1.0 / math.sqrt(np.finfo(float).eps) if kappa_max is None else kappa_max
        U, sig, Vt = np.linalg.svd(C, full_matrices=False)
        keep = np.nonzero(sig / sig[0] > 1.0 / kappa_max)[0]
        k = int(keep[-1]) + 1 if len(keep) else 1
        Uk, Vk, sk = U[:, :k], Vt[:k].T, sig[:k]
        M = Uk.T @ D @ Vk
        lam, Z = sla.eig(M, np.diag(sk))
        lam, Z = _sort_eig(lam, Z)
        Yv = np.real(Vk @ Z)
        for j in range(k):
            Yv[:, j] /= np.linalg.norm(C @ Yv[:, j])
    else:
        Q, R, P = sla.qr(C, mode="economic", pivoting=True)     # qr(C, ColumnNorm()); M = F \ D
        Mp = sla.solve_triangular(R, Q.T @ D)
        M = np.empty_like(Mp)
        M[P] = Mp
        lam, Yv = np.linalg.eig(M)
        lam, Yv = _sort_eig(lam, Yv)
        Yv = np.real(Yv)
    lam = np.real(lam)
    res_sketch = float(np.linalg.norm(D @ Yv[:, 0] - lam[0] * (C @ Yv[:, 0])))
    y = Yv[:, 0] / np.linalg.norm(Yv[:, 0])
    X = o.ttrand_rounding_lincomb(list(y), list(B), 4 * rmax, orthogonal, seed, block_rks, rng_kind=rng_kind)
    X = o.tt_rounding(X, tol=res_sketch ** 2 / 2)
    nx = o.norm(X)
    if nx == 0.0:
        # tol = res^2 / 2 is a relative tolerance: from res >= sqrt(2) on, the rounding returns the
        # zero TT, which the reference then divides by its zero norm (NaN cores); the zero TT is
        # returned here, with a NaN sampled residual as in the reference
        return lam, X, res_sketch, float("nan")
    X = o.tt_scale(1.0 / nx, X)
    S1, _ = tt_sketch(X, 2 * N, H, orthogonal, sample_seed, block_rks, rng_kind)
    S2, _ = tt_sketch(X, 2 * N, None, orthogonal, sample_seed, block_rks, rng_kind)
    res_sample = float(np.linalg.norm(S1 - lam[0] * S2) / np.linalg.norm(S2))
    return lam, X, res_sketch, res_sample


def sketched_rayleigh_ritz(H: o.TToperator, b0: o.TTvector, d: int, rmax: int, orthogonal=True, block_rks=8,
                           seed=1234, sketch_size=None, k_trunc=None, e_nuc=0.0, sample_seed=4321,
                           rng_kind="philox"):
    """src/tt_solvers.jl:547-618: d-dimensional sketch-orthogonal Krylov basis from b0 with a
    sketched Rayleigh-Ritz solve after every expansion.  The j-th solve samples its residual
    with seed sample_seed + j.  Returns (lowest Ritz value + e_nuc, Ritz vector, history)."""
    sketch_size = 4 * d if sketch_size is None else sketch_size
    k_trunc = d - 1 if k_trunc is None else k_trunc
    B: List[o.TTvector] = [None] * d
    sk_b: List[np.ndarray] = [None] * d
    sk_Hb: List[np.ndarray] = [None] * d
    sk0, W1, _ = tt_combined_sketch(b0, 2 * rmax, sketch_size, None, orthogonal, seed, block_rks, rng_kind)
    s = len(sk0)
    beta = float(np.linalg.norm(sk0))
    sk_b[0] = sk0 / beta
    _rescale_upto_root(W1, b0, beta)
    B[0] = o.tt_scale(1.0 / beta, b0)
    Bw, Ww, Sw = [B[0]], [W1], [sk_b[0]]
    hist = []

    def solve(j):
        C = np.column_stack(sk_b[:j])
        D = np.column_stack(sk_Hb[:j])
        lam, psi, rs, rsam = sketched_rr(H, B[:j], C, D, rmax, orthogonal, block_rks, seed,
                                         sample_seed=sample_seed + j, rng_kind=rng_kind)
        e_true = o.dot_operator(psi, H, psi) + e_nuc if o.norm(psi) > 0.0 else float("nan")
        hist.append(dict(iter=j, e_sketch=lam[0] + e_nuc, e_true=e_true, res_sketch=rs, res_sample=rsam))
        return lam[0] + e_nuc, psi

    for j in range(1, d):
        b_new, skb, skHb = expand_basis(H, Bw, Ww, Sw, rmax, s, orthogonal, block_rks, seed, k_trunc, rng_kind)
        B[j], sk_b[j], sk_Hb[j - 1] = b_new, skb, skHb
        solve(j)
    sk_Hb[d - 1], _, _ = tt_combined_sketch(B[d - 1], 2 * rmax, s, H, orthogonal, seed, block_rks, rng_kind)
    e, psi = solve(d)
    return e, psi, hist


def dot_randrounding(A: o.TToperator, x: o.TTvector) -> o.TTvector:
    """src/tt_randtools.jl:476-480"""
    y = o.tto_apply(A, x)
    y = o.ttrand_rounding(y)
    return o.tt_rounding(y, tol=1e-8)


def arnoldi(A: o.TToperator, m: int, V: List[o.TTvector], eps_tt=1e-6, rmax=256):
    """src/tt_solvers.jl:206-224.  A breakdown (the rounded w is the zero TT: its norm fell below
    eps_tt, which tt_rounding compares with the absolute norm of the last core) ends the
    iteration with the j + 1 vectors built so far, whose span is then invariant up to eps_tt;
    the reference divides by the zero norm and carries NaN cores from there on."""
    Hh = np.zeros((m + 1, m + 1))
    V = list(V[:1])
    V[0] = o.tt_scale(1.0 / o.norm(V[0]), V[0])
    for j in range(m):
        w = dot_randrounding(A, V[j])
        for i in range(j + 1):
            Hh[i, j] = o.dot(V[i], w)
            w = o.tt_sub(w, o.tt_scale(Hh[i, j], V[i]))          # w - H[i,j] V[i]
        w = o.ttrand_rounding(w)
        w = o.tt_rounding(w, tol=eps_tt, rmax=rmax)
        Hh[j + 1, j] = o.norm(w)
        if Hh[j + 1, j] == 0.0:
            return Hh[: j + 1, : j + 1], V, 0.0
        V.append(o.tt_scale(1.0 / Hh[j + 1, j], w))
    return Hh[:m, :m], V, float(Hh[m, m - 1])


def eig_arnoldi(A: o.TToperator, m: int, v: o.TTvector, Imax=100, eps=1e-6, eps_tt=1e-4, rmax=256, which="LM",
                sigma=0.0, history=False):
    """src/tt_solvers.jl:226-265, restarted from the Ritz vector with sketch ranks twice those of
    the current vector (boundary ranks 1)."""
    def ritz(Hh):
        vals, vecs = np.linalg.eig(Hh + sigma * np.eye(Hh.shape[0]))
        k = int(np.argmax(np.abs(vals)) if which == "LM" else np.argmin(np.abs(vals)))
        return vals[k], np.real(vecs[:, k])

    def restart(V, f, v):
        rks = [1] + [2 * r for r in v.ttv_rks[1:-1]] + [1]
        u = o.ttrand_rounding_lincomb(list(f), V[:len(f)], rks)
        return o.tt_rounding(u, tol=eps_tt, rmax=rmax)

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
            r = o.tt_sub(o.tto_apply(A, v), o.tt_scale(lam.real - sigma, v))
            hist.append(o.norm(r))
        i += 1
    return float(np.real(lam) - sigma), v, hist
