"""FP64 CPU restatement of the TensorTrains hot path (TEST INFRASTRUCTURE ONLY).

Every function follows the cited lines of the Julia reference
(rodrigofj99/Tensor-Train-Julia, paths relative to that project).  Arrays keep
Julia's column-major semantics: a TT core is an ndarray of shape
``(n_k, r_{k-1}, r_k)`` and every reshape uses ``order='F'``, so reshapes and
unfoldings mean exactly what they mean in Julia.  Factorisations call the same
LAPACK drivers Julia calls: ``qr`` -> geqrf+orgqr, ``lq`` -> gelqf (as QR of the
transpose), ``svd`` -> gesdd with gesvd fallback.

This module is the checker for the CUDA library.  The library never imports it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import scipy.linalg as sla

F = "F"


def ein(expr: str, *ops: np.ndarray) -> np.ndarray:
    """Contraction of `ops` by the index expression `expr` (einsum notation), performed pairwise
    from left to right -- the operands' order is the contraction order, as in the reference's
    hand-ordered `mul!` chains -- each step a BLAS tensordot over the indices no later operand
    or the output needs (an index shared by both sides and still needed later falls back to a
    two-operand einsum)."""
    ins, out = expr.split("->")
    subs = ins.split(",")
    assert len(subs) == len(ops)

    def needed(k):
        return set(out) | set("".join(subs[k + 1:]))

    def reduce_alone(s, A, keep):
        drop = [c for c in s if c not in keep and s.count(c) == 1]
        if drop:
            A = A.sum(axis=tuple(s.index(c) for c in drop))
            s = "".join(c for c in s if c not in drop)
        return s, A

    cur_s, cur = reduce_alone(subs[0], ops[0], needed(0) | set(subs[1]) if len(subs) > 1 else set(out))
    for k in range(1, len(ops)):
        s, B = subs[k], ops[k]
        later = needed(k)
        s, B = reduce_alone(s, B, later | set(cur_s))
        shared = [c for c in cur_s if c in s]
        summed = [c for c in shared if c not in later]
        batch = [c for c in shared if c in later]
        if batch:
            res = "".join(dict.fromkeys(c for c in cur_s + s if c in later))
            cur = np.einsum(f"{cur_s},{s}->{res}", cur, B)
            cur_s = res
        else:
            cur = np.tensordot(cur, B, axes=([cur_s.index(c) for c in summed], [s.index(c) for c in summed]))
            cur_s = "".join(c for c in cur_s if c not in summed) + "".join(c for c in s if c not in summed)
    cur_s, cur = reduce_alone(cur_s, cur, set(out))
    return np.ascontiguousarray(np.transpose(cur, [cur_s.index(c) for c in out]))


# --------------------------------------------------------------------------- types
@dataclass
class TTvector:
    """src/tt_tools.jl:24-34.  ttv_vec[k] has shape (n_k, r_{k-1}, r_k)."""
    N: int
    ttv_vec: List[np.ndarray]
    ttv_dims: tuple
    ttv_rks: List[int]
    ttv_ot: List[int]

    def copy(self) -> "TTvector":
        """src/tt_tools.jl:356-362"""
        return TTvector(self.N, [c.copy() for c in self.ttv_vec], tuple(self.ttv_dims),
                        list(self.ttv_rks), list(self.ttv_ot))


@dataclass
class TToperator:
    """src/tt_tools.jl:61-71.  tto_vec[k] has shape (n_k, n_k, R_{k-1}, R_k) = [i_out, j_in, a, a']."""
    N: int
    tto_vec: List[np.ndarray]
    tto_dims: tuple
    tto_rks: List[int]
    tto_ot: List[int]


# ------------------------------------------------------------------- constructors
def r_and_d_to_rks(rks, dims, rmax=1024):
    """src/tt_rounding.jl:6-24 (1-based i over eachindex(dims); new_rks[end] stays 1)."""
    rks = list(rks)
    d = len(dims)
    new = [1] * len(rks)
    for i in range(d):                       # Julia i = i+1
        right = int(np.prod(dims[i:])) if d - i > 0 else 1
        left = int(np.prod(dims[:i])) if i > 0 else 1
        if right > 0:
            if left > 0:
                new[i] = min(rks[i], left, right, rmax)
            else:
                new[i] = min(rks[i], right, rmax)
        else:
            new[i] = min(rks[i], left, rmax) if left > 0 else min(rks[i], rmax)
    return new


def zeros_tt(dims, rks, ot=None) -> TTvector:
    """src/tt_tools.jl:91-95"""
    dims = tuple(int(n) for n in dims)
    N = len(dims)
    vec = [np.zeros((dims[i], rks[i], rks[i + 1])) for i in range(N)]
    return TTvector(N, vec, dims, list(rks), list(ot) if ot is not None else [0] * N)


def zeros_tto(dims, rks) -> TToperator:
    """src/tt_tools.jl:156-160"""
    dims = tuple(int(n) for n in dims)
    N = len(dims)
    vec = [np.zeros((dims[i], dims[i], rks[i], rks[i + 1])) for i in range(N)]
    return TToperator(N, vec, dims, list(rks), [0] * N)


def rand_tt(dims, rks, rng: np.random.Generator, normalise=False, orthogonal=False,
            right=True, stable=True) -> TTvector:
    """src/tt_tools.jl:255-318 (N(0,1) cores from a numpy Generator instead of Julia's
    Xoshiro stream; Julia's stream cannot be reproduced without Julia)."""
    dims = tuple(int(n) for n in dims)
    N = len(dims)
    if isinstance(rks, (int, np.integer)):
        rks = r_and_d_to_rks([int(rks)] * (N + 1), dims, rmax=int(rks))
    elif stable:
        rks = r_and_d_to_rks(rks, dims, rmax=max(rks))
    rks = [int(r) for r in rks]
    y = zeros_tt(dims, rks)

    def randn(*shape):
        return rng.standard_normal(int(np.prod(shape))).reshape(shape, order=F)

    if orthogonal and right:
        for i in range(N - 1):
            if rks[i] > dims[i] * rks[i + 1]:
                raise ValueError(f"Cannot create right-orthogonal core {i + 1}")
            q, _ = sla.qr(randn(dims[i] * rks[i + 1], rks[i]), mode="economic")
            y.ttv_vec[i] = np.transpose(q.reshape(dims[i], rks[i + 1], rks[i], order=F), (0, 2, 1))
        y.ttv_vec[N - 1] = randn(dims[N - 1], rks[N - 1], rks[N])
        if normalise:
            y.ttv_vec[N - 1] *= 1 / math.sqrt(dims[N - 1] * rks[N])
    elif orthogonal:
        y.ttv_vec[0] = randn(dims[0], rks[0], rks[1])
        if normalise:
            y.ttv_vec[0] *= 1 / math.sqrt(dims[0] * rks[0])
        for i in range(1, N):
            if dims[i] * rks[i] > rks[i + 1]:
                raise ValueError(f"Cannot create left-orthogonal core {i + 1}")
            q, _ = sla.qr(randn(dims[i] * rks[i], rks[i + 1]), mode="economic")
            y.ttv_vec[i] = q.reshape(dims[i], rks[i], rks[i + 1], order=F)
    else:
        for i in range(N):
            y.ttv_vec[i] = randn(dims[i], rks[i], rks[i + 1])
        if normalise:
            for i in range(N):
                y.ttv_vec[i] *= 1 / math.sqrt(dims[i] * (rks[i + 1] if right else rks[i]))
    return y


def is_leftorthogonal(x: TTvector) -> bool:
    """src/tt_tools.jl:364-367"""
    return all(o == 1 for o in x.ttv_ot[: x.N - 1])


def is_rightorthogonal(x: TTvector) -> bool:
    """src/tt_tools.jl:369-372"""
    return all(o == -1 for o in x.ttv_ot[1:])


def ttv_to_tensor(x: TTvector) -> np.ndarray:
    """src/tt_tools.jl:520-535 (vectorised: same contraction)."""
    t = x.ttv_vec[0]                            # (n1, 1, r1)
    out = t.reshape(x.ttv_dims[0], x.ttv_rks[1], order=F)
    for k in range(1, x.N):
        c = x.ttv_vec[k]                        # (n, r, r')
        # out[(i1..ik-1), a] * c[ik, a, b] -> out[(i1..ik), b] with ik slowest
        out = np.einsum("Pa,iab->Pib", out, c).reshape(-1, x.ttv_rks[k + 1], order=F)
    return out.reshape(x.ttv_dims, order=F)


def tto_to_tensor(A: TToperator) -> np.ndarray:
    """src/tt_tools.jl:657-674: tensor of shape (n_1..n_d, n_1..n_d)."""
    d = A.N
    out = A.tto_vec[0].reshape(A.tto_dims[0], A.tto_dims[0], A.tto_rks[1], order=F)
    for k in range(1, d):
        c = A.tto_vec[k]
        out = np.einsum("PQa,ijab->PiQjb", out, c)
        s = out.shape
        out = out.reshape(s[0] * s[1], s[2] * s[3], s[4], order=F)
    dims = tuple(A.tto_dims)
    return out.reshape(dims + dims, order=F)


def ttv_decomp(tensor: np.ndarray, index=1, tol=1e-12) -> TTvector:
    """src/tt_tools.jl:380-443 (HSVD)."""
    dims = tensor.shape
    d = len(dims)
    vec = [None] * d
    ot = [0] * d
    for i in range(index - 1):
        ot[i] = 1
    for i in range(index, d):
        ot[i] = -1
    rks = [1] * (d + 1)
    cur = tensor
    for i in range(index - 1):
        cur = cur.reshape(rks[i] * dims[i], -1, order=F)
        u, s, vh = svd_julia(cur)
        rks[i + 1] = int(np.sum(s >= tol))
        vec[i] = np.transpose(u[:, : rks[i + 1]].reshape(rks[i], dims[i], rks[i + 1], order=F), (1, 0, 2))
        cur = np.diag(s[: rks[i + 1]]) @ vh[: rks[i + 1], :]
    for i in range(d - 1, index - 1, -1):
        cur = cur.reshape(-1, dims[i] * rks[i + 1], order=F)
        u, s, vh = svd_julia(cur)
        rks[i] = int(np.sum(s >= tol))
        vec[i] = np.transpose(vh[: rks[i], :].reshape(rks[i], dims[i], rks[i + 1], order=F), (1, 0, 2))
        cur = u[:, : rks[i]] * s[: rks[i]]
    i = index - 1
    cur = cur.reshape(dims[i] * rks[i], -1, order=F)
    vec[i] = np.transpose(cur[:, : rks[i + 1]].reshape(rks[i], dims[i], rks[i + 1], order=F), (1, 0, 2))
    return TTvector(d, vec, tuple(dims), rks, ot)


def tto_decomp(tensor: np.ndarray, index=1) -> TToperator:
    """TT-matrix decomposition of a (n_1..n_d, n_1..n_d) tensor: interleave (i_k, j_k),
    decompose as a TTvector with n_k^2 modes (src/tt_tools.jl:447-480 idea), reshape cores."""
    d = tensor.ndim // 2
    dims = tensor.shape[:d]
    perm = []
    for k in range(d):
        perm += [k, d + k]
    t = np.transpose(tensor, perm).reshape(tuple(n * n for n in dims), order=F)
    x = ttv_decomp(t, index=index)
    vec = [x.ttv_vec[k].reshape(dims[k], dims[k], x.ttv_rks[k], x.ttv_rks[k + 1], order=F) for k in range(d)]
    return TToperator(d, vec, tuple(dims), list(x.ttv_rks), list(x.ttv_ot))


def tto_to_ttv(A: TToperator) -> TTvector:
    """src/tt_tools.jl:603-611"""
    vec = [A.tto_vec[i].reshape(A.tto_dims[i] ** 2, A.tto_rks[i], A.tto_rks[i + 1], order=F) for i in range(A.N)]
    return TTvector(A.N, vec, tuple(n * n for n in A.tto_dims), list(A.tto_rks), list(A.tto_ot))


def ttv_to_tto(x: TTvector) -> TToperator:
    """src/tt_tools.jl:616-626"""
    n = [int(math.isqrt(m)) for m in x.ttv_dims]
    assert all(a * a == b for a, b in zip(n, x.ttv_dims))
    vec = [x.ttv_vec[i].reshape(n[i], n[i], x.ttv_rks[i], x.ttv_rks[i + 1], order=F) for i in range(x.N)]
    return TToperator(x.N, vec, tuple(n), list(x.ttv_rks), list(x.ttv_ot))


def tt_up_rks(x: TTvector, rk_max: int, rng: Optional[np.random.Generator] = None, eps_wn=0.0) -> TTvector:
    """src/tt_rounding.jl:26-60 (rank padding, optional noise from rand_orthogonal)."""
    d = x.N
    assert rk_max >= max(x.ttv_rks)
    rks = r_and_d_to_rks([1] + [rk_max] * (d - 1) + [1], x.ttv_dims, rmax=rk_max)
    vec = []
    for i in range(d):
        t = x.ttv_vec[i]
        n, r0, r1 = t.shape
        rkm, rk = rks[i], rks[i + 1]
        out = np.zeros((n, rkm, rk))
        out[:, :r0, :r1] = t
        if eps_wn != 0.0:
            assert rng is not None

            def rand_orth(m, k):
                q, _ = sla.qr(rng.standard_normal((max(m, k), min(m, k))), mode="economic")
                return q if m >= k else q.T
            if rkm == r0 and rk > r1:
                Q = rand_orth(n * rkm, rk - r1)
                out[:, :, r1:rk] = eps_wn * Q.reshape(n, rkm, rk - r1, order=F)
            elif rk == r1 and rkm > r0:
                Q = rand_orth(rkm - r0, n * rk)
                out[:, r0:rkm, :] = eps_wn * Q.reshape(n, rkm - r0, rk, order=F)
            elif rk > r1 and rkm > r0:
                Q = rand_orth((rkm - r0) * n, rk - r1)
                out[:, r0:rkm, r1:rk] = eps_wn * Q.reshape(n, rkm - r0, rk - r1, order=F)
        vec.append(out)
    return TTvector(d, vec, tuple(x.ttv_dims), rks, [0] * d)


# ---------------------------------------------------------------- LAPACK mirrors
def qr_julia(A: np.ndarray):
    """Julia `qr(A)`; `Matrix(F.Q)`, `F.R` -> LAPACK geqrf + orgqr (thin)."""
    Q, R = sla.qr(A, mode="economic")
    return Q, R


def lq_julia(A: np.ndarray):
    """Julia `lq(A)` -> (L, Q) with A = L Q; computed as the QR of A^T (gelqf equivalent)."""
    Qt, Rt = sla.qr(A.T, mode="economic")
    return Rt.T, Qt.T


def svd_julia(M: np.ndarray):
    """Julia `svd(M, full=false)` (gesdd) with the LAPACKException -> QRIteration (gesvd)
    fallback of src/tt_rounding.jl:191-195.  Returns (U, s, Vh)."""
    try:
        return sla.svd(M, full_matrices=False, lapack_driver="gesdd")
    except np.linalg.LinAlgError:
        return sla.svd(M, full_matrices=False, lapack_driver="gesvd")


# ------------------------------------------------------------------ TT algebra
def tt_add(x: TTvector, y: TTvector) -> TTvector:
    """src/tt_operations.jl:81-112 (direct sum, ranks not re-clamped)."""
    assert tuple(x.ttv_dims) == tuple(y.ttv_dims)
    d = x.N
    rks = [a + b for a, b in zip(x.ttv_rks, y.ttv_rks)]
    rks[0] = 1
    rks[d] = 1
    vec = [np.zeros((x.ttv_dims[k], rks[k], rks[k + 1])) for k in range(d)]
    if d == 1:
        vec[0][:, :, :] = x.ttv_vec[0] + y.ttv_vec[0]
        return TTvector(d, vec, tuple(x.ttv_dims), rks, [0] * d)
    xr, yr = x.ttv_rks, y.ttv_rks
    vec[0][:, :, : xr[1]] = x.ttv_vec[0]
    vec[0][:, :, xr[1]: rks[1]] = y.ttv_vec[0]
    for k in range(1, d - 1):
        vec[k][:, : xr[k], : xr[k + 1]] = x.ttv_vec[k]
        vec[k][:, xr[k]: rks[k], xr[k + 1]: rks[k + 1]] = y.ttv_vec[k]
    vec[d - 1][:, : xr[d - 1], 0:1] = x.ttv_vec[d - 1]
    vec[d - 1][:, xr[d - 1]: rks[d - 1], 0:1] = y.ttv_vec[d - 1]
    return TTvector(d, vec, tuple(x.ttv_dims), rks, [0] * d)


def tt_scale(a: float, A: TTvector) -> TTvector:
    """src/tt_operations.jl:428-441: scales only the first core with ot == 0."""
    if a == 0:
        return zeros_tt(A.ttv_dims, [1] * (A.N + 1))
    i = A.ttv_ot.index(0)
    vec = list(A.ttv_vec)
    vec[i] = a * vec[i]
    return TTvector(A.N, vec, tuple(A.ttv_dims), list(A.ttv_rks), list(A.ttv_ot))


def tt_sub(A: TTvector, B: TTvector) -> TTvector:
    """src/tt_operations.jl:453-455"""
    return tt_add(tt_scale(-1.0, B), A)


def tto_add(x: TToperator, y: TToperator) -> TToperator:
    """src/tt_operations.jl:121-148"""
    d = x.N
    rks = [a + b for a, b in zip(x.tto_rks, y.tto_rks)]
    rks[0] = 1
    rks[d] = 1
    n = x.tto_dims
    vec = [np.zeros((n[k], n[k], rks[k], rks[k + 1])) for k in range(d)]
    xr = x.tto_rks
    if d == 1:
        vec[0][...] = x.tto_vec[0] + y.tto_vec[0]
        return TToperator(d, vec, tuple(n), rks, [0] * d)
    vec[0][:, :, :, : xr[1]] = x.tto_vec[0]
    vec[0][:, :, :, xr[1]: rks[1]] = y.tto_vec[0]
    for k in range(1, d - 1):
        vec[k][:, :, : xr[k], : xr[k + 1]] = x.tto_vec[k]
        vec[k][:, :, xr[k]: rks[k], xr[k + 1]: rks[k + 1]] = y.tto_vec[k]
    vec[d - 1][:, :, : xr[d - 1], 0:1] = x.tto_vec[d - 1]
    vec[d - 1][:, :, xr[d - 1]: rks[d - 1], 0:1] = y.tto_vec[d - 1]
    return TToperator(d, vec, tuple(n), rks, [0] * d)


def tto_scale(a: float, A: TToperator) -> TToperator:
    """src/tt_operations.jl:444-450"""
    i = A.tto_ot.index(0)
    vec = list(A.tto_vec)
    vec[i] = a * vec[i]
    return TToperator(A.N, vec, tuple(A.tto_dims), list(A.tto_rks), list(A.tto_ot))


def tto_mul(A: TToperator, B: TToperator) -> TToperator:
    """src/tt_operations.jl:211-237: ranks A_r*B_r with the A index fastest."""
    d = A.N
    vec = []
    for k in range(d):
        a = A.tto_vec[k]
        b = B.tto_vec[k]
        n = a.shape[0]
        M = np.einsum("izab,zjcd->ijacbd", a, b)      # [i, j, aA, aB, bA, bB]
        vec.append(M.reshape(n, n, a.shape[2] * b.shape[2], a.shape[3] * b.shape[3], order=F))
    rks = [p * q for p, q in zip(A.tto_rks, B.tto_rks)]
    return TToperator(d, vec, tuple(A.tto_dims), rks, [0] * d)


def tto_apply(A: TToperator, v: TTvector) -> TTvector:
    """src/tt_operations.jl:170-194: y[i,(a,nu),(a',nu')] = sum_j A[i,j,a,a'] v[j,nu,nu'],
    combined rank index with the operator index fastest; output ot = 0."""
    assert tuple(A.tto_dims) == tuple(v.ttv_dims)
    d = v.N
    rks = [p * q for p, q in zip(A.tto_rks, v.ttv_rks)]
    vec = []
    for k in range(d):
        Y = np.einsum("ijab,jcd->iacbd", A.tto_vec[k], v.ttv_vec[k])
        vec.append(Y.reshape(v.ttv_dims[k], rks[k], rks[k + 1], order=F))
    return TTvector(d, vec, tuple(v.ttv_dims), rks, [0] * d)


def dot(A: TTvector, B: TTvector) -> float:
    """src/tt_operations.jl:302-323"""
    assert tuple(A.ttv_dims) == tuple(B.ttv_dims)
    out = np.ones((1, 1))
    for k in range(A.N):
        out = ein("ac,zab,zcd->bd", out, A.ttv_vec[k], np.conj(B.ttv_vec[k]))
    return float(out[0, 0])


def partial_contraction(A: TTvector, B: TTvector, reverse=True) -> List[np.ndarray]:
    """src/sketches.jl:1047-1070"""
    L = A.N
    W = [np.zeros((A.ttv_rks[i], B.ttv_rks[i])) for i in range(L + 1)]
    if reverse:
        W[L] = np.ones((1, 1))
        for k in range(L - 1, -1, -1):
            W[k] = ein("bd,zab,zcd->ac", W[k + 1], A.ttv_vec[k], B.ttv_vec[k])
    else:
        W[0] = np.ones((1, 1))
        for k in range(L):
            W[k + 1] = ein("ac,zab,zcd->bd", W[k], A.ttv_vec[k], B.ttv_vec[k])
    return W


def dot_operator(psi: TTvector, H: TToperator, phi: TTvector) -> float:
    """src/tt_operations.jl:390-421 (<psi|H|phi>, pivot at the canonical centre)."""
    N = psi.N

    def center(v):
        return v.ttv_ot.index(0) + 1 if 0 in v.ttv_ot else N
    c = max(center(psi), center(phi))
    L = np.ones((1, 1, 1))
    for k in range(c if c > 1 else 0):
        L = ein("abc,iad,ijbe,jcf->def", L, np.conj(psi.ttv_vec[k]), H.tto_vec[k], phi.ttv_vec[k])
    R = np.ones((1, 1, 1))
    r = c + 1 if c > 1 else 1
    for k in range(N, r - 1, -1):
        kk = k - 1
        R = ein("def,jcf,ijbe,iad->abc", R, phi.ttv_vec[kk], H.tto_vec[kk], np.conj(psi.ttv_vec[kk]))
    if c == 1:
        res = R
    elif c == N:
        res = L
    else:
        res = np.einsum("abc,abc->", L, R)
    return float(np.asarray(res).reshape(-1)[0])


# -------------------------------------------------------------- deterministic path
def orthogonalize(x: TTvector, i: int = 1) -> TTvector:
    """src/tt_rounding.jl:65-97 (1-based root i)."""
    d = x.N
    assert 1 <= i <= d
    y_rks = r_and_d_to_rks(x.ttv_rks, x.ttv_dims)
    y = zeros_tt(x.ttv_dims, y_rks)
    FR = np.ones((1, 1))
    for j in range(i - 1):                    # Julia j = j+1 in 1:i-1
        n = x.ttv_dims[j]
        # yleft[a', i, a] = FR[a', b] x[i, b, a]   (layout (r', n, r): r' fastest)
        yleft = np.einsum("ab,ibc->aic", FR, x.ttv_vec[j])
        Q, R = qr_julia(yleft.reshape(n * y.ttv_rks[j], -1, order=F))
        y.ttv_ot[j] = 1
        y.ttv_rks[j + 1] = Q.shape[1]
        y.ttv_vec[j] = np.transpose(Q.reshape(y.ttv_rks[j], n, y.ttv_rks[j + 1], order=F), (1, 0, 2))
        FR = R[: y.ttv_rks[j + 1], :]
    FL = np.ones((1, 1))
    for j in range(d - 1, i - 1, -1):          # Julia j = d..i+1
        n = x.ttv_dims[j]
        # yright[a, b', i] = x[i, a, c] FL[c, b']
        yright = np.einsum("iac,cb->abi", x.ttv_vec[j], FL)
        Lf, Q = lq_julia(yright.reshape(x.ttv_rks[j], -1, order=F))
        y.ttv_ot[j] = -1
        y.ttv_rks[j] = Q.shape[0]
        y.ttv_vec[j] = np.transpose(Q.reshape(y.ttv_rks[j], y.ttv_rks[j + 1], n, order=F), (2, 0, 1))
        FL = Lf[:, : y.ttv_rks[j]]
    c = i - 1
    y.ttv_ot[c] = 0
    y.ttv_vec[c] = np.einsum("ab,ibc,cd->iad", FR, x.ttv_vec[c], FL)
    return y


def norm(v: TTvector) -> float:
    """src/tt_rounding.jl:107-114"""
    if sum(1 for o in v.ttv_ot if o == 0) == 1:
        return float(np.linalg.norm(v.ttv_vec[v.ttv_ot.index(0)]))
    w = orthogonalize(v, i=v.N)
    return float(np.linalg.norm(w.ttv_vec[-1]))


def floor_rank(s: np.ndarray, tol: float, degen_tol: float = 1e-5) -> int:
    """src/tt_rounding.jl:297-315: returns the kept count i of `floor(s, tol)`.
    Julia `isapprox(1., r; atol=degen_tol)` has rtol=0, i.e. |1-r| <= degen_tol."""
    if tol == 0.0:
        return len(s)
    d = len(s)
    i = d
    weight = 0.0
    norm2 = float(np.dot(s, s))
    while i > 0 and weight < tol * tol * norm2:
        weight += float(s[i - 1]) ** 2
        i -= 1
    i += 1
    while i < d:
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = s[i] / s[i - 1]
        if np.isfinite(ratio) and abs(1.0 - ratio) <= degen_tol:
            i += 1
        else:
            break
    return i


def _tt_rounding(y: TTvector, tol=1e-12, rmax=2 ** 14, direction="left") -> TTvector:
    """src/tt_rounding.jl:174-269 (mutates and returns y)."""
    N = y.N
    if direction == "left":
        if np.linalg.norm(y.ttv_vec[N - 1]) < tol:
            return zeros_tt(y.ttv_dims, y.ttv_rks)
        for j in range(N - 1, 0, -1):               # Julia j = N..2 -> 0-based j
            nj, rp, rj = y.ttv_dims[j], y.ttv_rks[j], y.ttv_rks[j + 1]
            M = np.transpose(y.ttv_vec[j], (1, 0, 2)).reshape(rp, nj * rj, order=F)
            u, s, vh = svd_julia(M)
            k = floor_rank(s, tol)
            k = min(k, rmax, int(np.sum(s > 0.0)))
            y.ttv_vec[j] = np.transpose(vh[:k, :].reshape(k, nj, rj, order=F), (1, 0, 2))
            US = u[:, :k] * s[:k][None, :]
            npv, rpp = y.ttv_dims[j - 1], y.ttv_rks[j - 1]
            left = y.ttv_vec[j - 1].reshape(npv * rpp, rp, order=F)
            y.ttv_vec[j - 1] = (left @ US).reshape(npv, rpp, k, order=F)
            y.ttv_rks[j] = k
            y.ttv_ot[j] = -1
        y.ttv_ot[0] = 0
        return y
    elif direction == "right":
        if np.linalg.norm(y.ttv_vec[0]) < tol:
            return zeros_tt(y.ttv_dims, y.ttv_rks)
        for j in range(N - 1):
            nj, rp, rj = y.ttv_dims[j], y.ttv_rks[j], y.ttv_rks[j + 1]
            M = y.ttv_vec[j].reshape(nj * rp, rj, order=F)
            u, s, vh = svd_julia(M)
            k = floor_rank(s, tol)
            k = min(k, rmax, int(np.sum(s > 0.0)))
            y.ttv_vec[j] = u[:, :k].reshape(nj, rp, k, order=F)
            SVT = s[:k][:, None] * vh[:k, :]
            nn, rn = y.ttv_dims[j + 1], y.ttv_rks[j + 2]
            right = np.transpose(y.ttv_vec[j + 1], (1, 0, 2)).reshape(rj, nn * rn, order=F)
            y.ttv_vec[j + 1] = np.transpose((SVT @ right).reshape(k, nn, rn, order=F), (1, 0, 2))
            y.ttv_rks[j + 1] = k
            y.ttv_ot[j] = 1
        y.ttv_ot[N - 1] = 0
        return y
    raise ValueError("Invalid direction. Use direction=:right or direction=:left")


def tt_rounding(x: TTvector, tol=1e-12, rmax=2 ** 14, direction="left") -> TTvector:
    """src/tt_rounding.jl:146-154"""
    if direction == "left":
        y = x.copy() if is_leftorthogonal(x) else orthogonalize(x, i=x.N)
    else:
        y = x.copy() if is_rightorthogonal(x) else orthogonalize(x, i=1)
    return _tt_rounding(y, tol=tol, rmax=rmax, direction=direction)


def tt_rounding_tto(A: TToperator, tol=1e-12, rmax=2 ** 14) -> TToperator:
    """src/tt_rounding.jl:275-277"""
    return ttv_to_tto(tt_rounding(tto_to_ttv(A), tol=tol, rmax=rmax))


def tt_svdvals(x: TTvector, tol: float = 0.0) -> List[np.ndarray]:
    """src/tt_rounding.jl:282-295: singular values of the unfolding x[mu_1..mu_k; mu_{k+1}..mu_d]
    for k = 1..N-1 (orthogonalize onto site 1, then an L->R SVD sweep).  tol = 0 keeps every
    singular value (floor(s, 0) returns s); the reference's default 1e-14 applies the floor rule."""
    N = x.N
    y = orthogonalize(x, i=1)
    out = []
    cur = y.ttv_vec[0].reshape(y.ttv_dims[0] * y.ttv_rks[0], y.ttv_rks[1], order=F)
    for j in range(N - 1):
        u, s, vh = svd_julia(cur)
        k = floor_rank(s, tol) if tol > 0 else len(s)
        out.append(np.array(s[:k]))
        nxt = y.ttv_vec[j + 1]                               # (n, r_j, r_{j+1})
        SV = s[:, None] * vh                                 # (len(s), r_j)
        core = np.einsum("az,izb->iab", SV, nxt)
        cur = core.reshape(core.shape[0] * core.shape[1], core.shape[2], order=F)
    return out


# ------------------------------------------------------------- sketch generation
PHILOX_M0, PHILOX_M1 = 0xD2511F53, 0xCD9E8D57      # Salmon et al., SC'11 (Random123)
PHILOX_W0, PHILOX_W1 = 0x9E3779B9, 0xBB67AE85


def philox4x32_10(ctr: np.ndarray, key0: int, key1: int) -> np.ndarray:
    """Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  ctr: uint64 array (n, 4)
    holding 32-bit words.  Mirrors the device generator in tensor-train-julia_b200/csrc/tt_kernels.cu."""
    c = ctr.astype(np.uint64) & 0xFFFFFFFF
    k0 = np.uint64(key0 & 0xFFFFFFFF)
    k1 = np.uint64(key1 & 0xFFFFFFFF)
    mask = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(PHILOX_M0) * c[:, 0]
        p1 = np.uint64(PHILOX_M1) * c[:, 2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c = np.stack([(hi1 ^ c[:, 1] ^ k0) & mask, lo1, (hi0 ^ c[:, 3] ^ k1) & mask, lo0], axis=1)
        k0 = (k0 + np.uint64(PHILOX_W0)) & mask
        k1 = (k1 + np.uint64(PHILOX_W1)) & mask
    return c


def philox_normals(count: int, seed: int, stream: int, sub: int) -> np.ndarray:
    """N(0,1) numbers e = 0..count-1 for (seed, stream, sub): counter (e//4, stream, sub, 0),
    key = (seed lo, seed hi); Box-Muller on the word pairs (0,1) and (2,3), uniforms
    u = (w + 0.5) * 2^-32.  Element e takes normal e % 4 of its counter."""
    nctr = (count + 3) // 4
    ctr = np.zeros((nctr, 4), dtype=np.uint64)
    ctr[:, 0] = np.arange(nctr, dtype=np.uint64)
    ctr[:, 1] = stream & 0xFFFFFFFF
    ctr[:, 2] = sub & 0xFFFFFFFF
    w = philox4x32_10(ctr, seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF).astype(np.float64)
    u = (w + 0.5) * (1.0 / 4294967296.0)
    r01 = np.sqrt(-2.0 * np.log(u[:, 0]))
    r23 = np.sqrt(-2.0 * np.log(u[:, 2]))
    t01 = 2.0 * np.pi * u[:, 1]
    t23 = 2.0 * np.pi * u[:, 3]
    z = np.stack([r01 * np.cos(t01), r01 * np.sin(t01), r23 * np.cos(t23), r23 * np.sin(t23)], axis=1)
    return z.reshape(-1)[:count]


class SketchRNG:
    """Source of the raw N(0,1) sketch blocks.  'philox' reproduces the CUDA generator
    (stream = site index k, sub = 0); 'numpy' draws from a numpy Generator in call order
    (the analogue of `randn!(rng, block)` at src/sketches.jl:68)."""

    def __init__(self, seed=1234, kind="philox"):
        self.seed = int(seed)
        self.kind = kind
        self._gen = np.random.default_rng(seed) if kind == "numpy" else None

    def block(self, site: int, shape) -> np.ndarray:
        cnt = int(np.prod(shape))
        if self.kind == "philox":
            z = philox_normals(cnt, self.seed, site, 0)
        else:
            z = self._gen.standard_normal(cnt)
        return z.reshape(shape, order=F)


def generate_sketch_blocks(rng: SketchRNG, site: int, left_rank, dim, right_rank, p, orthogonal):
    """src/sketches.jl:44-84.  Returns (left_rank, dim, right_rank, p)."""
    assert (not orthogonal) or right_rank <= dim * left_rank
    use_identity = orthogonal and right_rank == dim * left_rank
    if use_identity:
        block = np.zeros((left_rank * dim, right_rank, p))
        for j in range(p):
            for i in range(right_rank):
                block[i, i, j] = 1.0
    else:
        block = rng.block(site, (left_rank * dim, right_rank, p))
        if orthogonal:
            for j in range(p):
                q, _ = qr_julia(block[:, :, j])
                block[:, :, j] = q
            block *= math.sqrt(left_rank * dim / right_rank)
        else:
            block *= 1 / math.sqrt(right_rank)
    return block.reshape(left_rank, dim, right_rank, p, order=F)


def compute_sketch_blocks_heuristic(rks, block_rks_vec, N, reverse):
    """src/sketches.jl:107-123 (code: p = ceil(rks/block_rks))."""
    p = [int(math.ceil(r / b)) for r, b in zip(rks, block_rks_vec)]
    if reverse:
        for i in range(1, N):
            p[i] = max(p[i], p[i - 1])
        p[N] = 1
    else:
        for i in range(N - 1, 0, -1):
            p[i] = max(p[i], p[i + 1])
        p[0] = 1
    return p


def default_rank_heuristic(y) -> List[int]:
    """src/tt_randtools.jl:31-50 (single TTvector or list)."""
    ys = y if isinstance(y, (list, tuple)) else [y]
    rks = list(ys[0].ttv_rks)
    for t in ys[1:]:
        rks = [max(a, b) for a, b in zip(rks, t.ttv_rks)]
    over = int(math.ceil(0.5 * max(rks)))
    N = ys[0].N
    for k in range(1, N):
        rks[k] += over
    return rks


def reverse_block_ranks(dims, N, block_rks):
    """src/sketches.jl:187-191"""
    b = [1] * (N + 1)
    for k in range(N):
        b[k] = block_rks
    for k in range(N - 1, -1, -1):
        b[k] = min(b[k], dims[k] * b[k + 1])
    return b


def sketch_plan(dims, N, rks, block_rks=None, p=None, oversampling=1):
    """Block ranks and block counts of the reverse sketch (src/sketches.jl:186-198)."""
    block_rks = N if block_rks is None else block_rks
    b = reverse_block_ranks(dims, N, block_rks)
    if p is None or (isinstance(p, int) and p == 0):
        p = compute_sketch_blocks_heuristic(list(rks), b, N, reverse=True)
    else:
        p = list(p)
    if oversampling != 1:
        for k in range(N):
            p[k] = int(math.ceil(oversampling * p[k]))
    return b, p


def make_reverse_sketch(dims, rks, seed=1234, orthogonal=True, block_rks=None, p=None,
                        rng_kind="philox"):
    """All sketch blocks of a reverse sketch, generated in the reference's order
    k = N..1 (src/sketches.jl:222-225).  Returns (blocks[k] of shape (b_{k+1}, n, b_k, p_k), b, p)."""
    N = len(dims)
    b, p = sketch_plan(dims, N, rks, block_rks, p)
    rng = SketchRNG(seed, rng_kind)
    blocks = [None] * N
    for k in range(N - 1, -1, -1):
        blocks[k] = generate_sketch_blocks(rng, k, b[k + 1], dims[k], b[k], p[k], orthogonal)
    return blocks, b, p


def contract_sketch_core_backwards(A: np.ndarray, S: np.ndarray, V: np.ndarray) -> np.ndarray:
    """src/sketches.jl:1602-1638: W[a,b] = sum A[z,a,al] S[be,z,b] V[al,be], in the order the
    reference's cost test picks: (A V) S or A (V S)."""
    z, a, al = A.shape
    be, _, b = S.shape
    if a * be * (al + b + 1) < al * (b + 1) * (a + be):
        return ein("zaA,AB,Bzb->ab", A, V, S)
    return ein("AB,Bzb,zaA->ab", V, S, A)


def contract_sketch_core_backwards_op(A, B, S, V):
    """src/sketches.jl:1648-1713: W[a,b,c] = sum A[z,a,al] B[ze,z,b,be] S[ga,ze,c] V[al,be,ga], in
    the order the reference's cost test picks: ((V A) B) S or ((V S) B) A."""
    z, a, al = A.shape
    ze, _, b, be = B.shape
    ga, _, c = S.shape
    if a * ga * (z * be * (al + ze * b) + ze * b * c) < al * c * (ze * be * (ga + z * b) + z * a * b):
        return ein("Aeg,zaA,Zzbe,gZc->abc", V, A, B, S)
    return ein("Aeg,gZc,Zzbe,zaA->abc", V, S, B, A)


def tt_recursive_sketch(A: TTvector, rks, orthogonal=True, seed=1234, block_rks=None, p=None,
                        blocks=None, rng_kind="philox"):
    """src/sketches.jl:175-305, reverse=true.  Returns (W list of (r_k, b_k*p_k), sketch_rks).
    `blocks` (from make_reverse_sketch) may be given so that both sides use identical sketches."""
    N = A.N
    dims = A.ttv_dims
    if isinstance(rks, (int, np.integer)):
        rks = [int(rks)] * (N + 1)
        rks[N] = 1
    assert rks[N] == 1 and A.ttv_rks[N] == 1
    if blocks is None:
        blocks, b, p = make_reverse_sketch(dims, rks, seed, orthogonal, block_rks, p, rng_kind)
    else:
        b, p = sketch_plan(dims, N, rks, block_rks, p)
    W = [None] * (N + 1)
    W[N] = np.ones((1, 1, 1))
    for k in range(N - 1, -1, -1):
        Wk = np.zeros((A.ttv_rks[k], b[k], p[k]))
        for j in range(p[k]):
            Wn = W[k + 1][:, :, j if k < N - 1 else 0]
            Wk[:, :, j] = contract_sketch_core_backwards(A.ttv_vec[k], blocks[k][:, :, :, j], Wn)
        W[k] = Wk
    for k in range(N + 1):
        W[k] = W[k] / math.sqrt(p[k])
    out = [W[k].reshape(A.ttv_rks[k], b[k] * p[k], order=F) for k in range(N + 1)]
    return out, [bb * pp for bb, pp in zip(b, p)]


def tt_recursive_sketch_op(H: TToperator, A: TTvector, rks, orthogonal=True, seed=1234,
                           block_rks=None, p=None, blocks=None, rng_kind="philox"):
    """src/sketches.jl:317-461, reverse=true.  Returns (W list of (r_k, R_k, b_k*p_k), sketch_rks)."""
    N = A.N
    dims = A.ttv_dims
    if isinstance(rks, (int, np.integer)):
        rks = [int(rks)] * (N + 1)
        rks[N] = 1
    assert rks[N] == 1 and A.ttv_rks[N] == 1 and H.tto_rks[N] == 1
    if blocks is None:
        blocks, b, p = make_reverse_sketch(dims, rks, seed, orthogonal, block_rks, p, rng_kind)
    else:
        b, p = sketch_plan(dims, N, rks, block_rks, p)
    W = [None] * (N + 1)
    W[N] = np.ones((1, 1, 1, 1))
    for k in range(N - 1, -1, -1):
        Wk = np.zeros((A.ttv_rks[k], H.tto_rks[k], b[k], p[k]))
        for j in range(p[k]):
            Wn = W[k + 1][:, :, :, j if k < N - 1 else 0]
            Wk[:, :, :, j] = contract_sketch_core_backwards_op(A.ttv_vec[k], H.tto_vec[k], blocks[k][:, :, :, j], Wn)
        W[k] = Wk
    for k in range(N + 1):
        W[k] = W[k] / math.sqrt(p[k])
    out = [W[k].reshape(A.ttv_rks[k], H.tto_rks[k], b[k] * p[k], order=F) for k in range(N + 1)]
    return out, [bb * pp for bb, pp in zip(b, p)]


# ------------------------------------------------------------- randomized rounding
def ttrand_rounding(y: TTvector, rks=None, orthogonal=True, seed=1234, block_rks=None,
                    blocks=None, rng_kind="philox", W=None) -> TTvector:
    """src/tt_randtools.jl:112-167 (rks may be a vector or an int rmax)."""
    N = y.N
    dims = y.ttv_dims
    if rks is None:
        rks = default_rank_heuristic(y)
    elif isinstance(rks, (int, np.integer)):
        rks = [1] + [int(rks)] * (N - 1) + [1]
    if W is None:
        W, sketch_rks = tt_recursive_sketch(y, rks, orthogonal, seed, block_rks, blocks=blocks, rng_kind=rng_kind)
    else:
        sketch_rks = [w.shape[1] for w in W]
    out_rks = [1] * (N + 1)
    ot = [0] * N
    vec = [None] * N
    yk = y.ttv_vec[0].reshape(dims[0], 1, y.ttv_rks[1], order=F)
    for k in range(N - 1):
        Z = np.einsum("iab,bc->iac", yk, W[k + 1])
        Z = Z.reshape(dims[k] * out_rks[k], sketch_rks[k + 1], order=F)
        Q, _ = qr_julia(Z)
        out_rks[k + 1] = Q.shape[1]
        vec[k] = Q.reshape(dims[k], out_rks[k], out_rks[k + 1], order=F)
        ot[k] = 1
        yk = ein("iab,iac,jbd->jcd", yk, vec[k], y.ttv_vec[k + 1])
    vec[N - 1] = yk.reshape(dims[N - 1], out_rks[N - 1], out_rks[N], order=F)
    return TTvector(N, vec, tuple(dims), out_rks, ot)


def ttrand_rounding_lincomb(alpha: Sequence[float], ys: Sequence[TTvector], rks=None, orthogonal=True,
                            seed=1234, block_rks=None, blocks=None, rng_kind="philox") -> TTvector:
    """src/tt_randtools.jl:223-283: rounding of sum_j alpha_j y_j."""
    m = len(alpha)
    N = ys[0].N
    dims = ys[0].ttv_dims
    assert len(ys) == m and all(tuple(t.ttv_dims) == tuple(dims) for t in ys)
    if rks is None:
        rks = default_rank_heuristic(list(ys))
    elif isinstance(rks, (int, np.integer)):
        rks = [1] + [int(rks)] * (N - 1) + [1]
    Ws = []
    srk = None
    for j in range(m):
        Wj, s = tt_recursive_sketch(ys[j], rks, orthogonal, seed, block_rks, blocks=blocks, rng_kind=rng_kind)
        assert srk is None or s == srk
        srk = s
        Ws.append(Wj)
    out_rks = [1] * (N + 1)
    ot = [0] * N
    vec = [None] * N
    Yk = [alpha[j] * ys[j].ttv_vec[0].reshape(dims[0], 1, ys[j].ttv_rks[1], order=F) for j in range(m)]
    for k in range(N - 1):
        Z = np.zeros((dims[k], out_rks[k], srk[k + 1]))
        for j in range(m):
            Z += np.einsum("iab,bc->iac", Yk[j], Ws[j][k + 1])
        Z = Z.reshape(dims[k] * out_rks[k], srk[k + 1], order=F)
        Q, _ = qr_julia(Z)
        out_rks[k + 1] = Q.shape[1]
        vec[k] = Q.reshape(dims[k], out_rks[k], out_rks[k + 1], order=F)
        ot[k] = 1
        Yk = [ein("iab,iac,jbd->jcd", Yk[j], vec[k], ys[j].ttv_vec[k + 1]) for j in range(m)]
    out_rks[N] = 1
    vec[N - 1] = sum(Yk)
    return TTvector(N, vec, tuple(dims), out_rks, ot)


def ttrand_rounding_op(alpha: Sequence[float], H: TToperator, ys: Sequence[TTvector], rks=None,
                       orthogonal=True, seed=1234, block_rks=None, blocks=None, rng_kind="philox") -> TTvector:
    """src/tt_randtools.jl:285-361: rounding of alpha_1 H y_1 + sum_{j>1} alpha_j y_j without
    forming H y_1.  The combined rank index of H y_1 is (y index fastest, H index)."""
    m = len(alpha)
    N = ys[0].N
    dims = ys[0].ttv_dims
    if rks is None:
        rks = default_rank_heuristic(list(ys))
    elif isinstance(rks, (int, np.integer)):
        rks = [1] + [int(rks)] * (N - 1) + [1]
    W1, srk = tt_recursive_sketch_op(H, ys[0], rks, orthogonal, seed, block_rks, blocks=blocks, rng_kind=rng_kind)
    Ws = [[W1[k].reshape(ys[0].ttv_rks[k] * H.tto_rks[k], srk[k], order=F) for k in range(N + 1)]]
    for j in range(1, m):
        Wj, s = tt_recursive_sketch(ys[j], rks, orthogonal, seed, block_rks, blocks=blocks, rng_kind=rng_kind)
        assert s == srk
        Ws.append(Wj)
    out_rks = [1] * (N + 1)
    ot = [0] * N
    vec = [None] * N
    Ay1 = np.einsum("jab,ijcd->iacbd", ys[0].ttv_vec[0], H.tto_vec[0]) * alpha[0]   # [i, a1, b1, a2, b2]
    Yk = [Ay1.reshape(dims[0], 1, ys[0].ttv_rks[1] * H.tto_rks[1], order=F)]
    for j in range(1, m):
        Yk.append(alpha[j] * ys[j].ttv_vec[0].reshape(dims[0], 1, ys[j].ttv_rks[1], order=F))
    for k in range(N - 1):
        Z = np.zeros((dims[k], out_rks[k], srk[k + 1]))
        for j in range(m):
            Z += np.einsum("iab,bc->iac", Yk[j], Ws[j][k + 1])
        Z = Z.reshape(dims[k] * out_rks[k], srk[k + 1], order=F)
        Q, _ = qr_julia(Z)
        out_rks[k + 1] = Q.shape[1]
        vec[k] = Q.reshape(dims[k], out_rks[k], out_rks[k + 1], order=F)
        ot[k] = 1
        y1k = Yk[0].reshape(dims[k], out_rks[k], ys[0].ttv_rks[k + 1], H.tto_rks[k + 1], order=F)
        Ay = ein("irab,irs,jac,ljbd->lscd", y1k, vec[k], ys[0].ttv_vec[k + 1], H.tto_vec[k + 1])
        new = [Ay.reshape(dims[k + 1], out_rks[k + 1], ys[0].ttv_rks[k + 2] * H.tto_rks[k + 2], order=F)]
        for j in range(1, m):
            new.append(ein("iab,iac,jbd->jcd", Yk[j], vec[k], ys[j].ttv_vec[k + 1]))
        Yk = new
    out_rks[N] = 1
    vec[N - 1] = sum(Yk)
    return TTvector(N, vec, tuple(dims), out_rks, ot)


def ttrand_rounding_residual(Atto: TToperator, y: TTvector, b: TTvector, rks=None, orthogonal=True,
                             seed=1234, block_rks=None, blocks=None, rng_kind="philox") -> TTvector:
    """src/tt_randtools.jl:169-214: rounding of A y - b without forming A y."""
    N = y.N
    dims = y.ttv_dims
    if rks is None:
        rks = default_rank_heuristic(y)
    elif isinstance(rks, (int, np.integer)):
        rks = [1] + [int(rks)] * (N - 1) + [1]
    WAy, srk = tt_recursive_sketch_op(Atto, y, rks, orthogonal, seed, block_rks, blocks=blocks, rng_kind=rng_kind)
    Wb, srk2 = tt_recursive_sketch(b, rks, orthogonal, seed, block_rks, blocks=blocks, rng_kind=rng_kind)
    out_rks = [1] * (N + 1)
    ot = [0] * N
    vec = [None] * N
    Ayk = np.einsum("jab,ijcd->iacbd", y.ttv_vec[0], Atto.tto_vec[0])[:, 0:1, 0, :, :]   # [i, rho, a, be]
    bk = b.ttv_vec[0].reshape(dims[0], 1, b.ttv_rks[1], order=F)
    for k in range(N - 1):
        Z = np.einsum("irab,abs->irs", Ayk, WAy[k + 1]) - np.einsum("ira,as->irs", bk, Wb[k + 1])
        Z = Z.reshape(dims[k] * out_rks[k], srk[k + 1], order=F)
        Q, _ = qr_julia(Z)
        out_rks[k + 1] = Q.shape[1]
        vec[k] = Q.reshape(dims[k], out_rks[k], out_rks[k + 1], order=F)
        ot[k] = 1
        Ayk = ein("irab,irs,jac,ljbd->lscd", Ayk, vec[k], y.ttv_vec[k + 1], Atto.tto_vec[k + 1])
        bk = ein("ira,irs,jab->jsb", bk, vec[k], b.ttv_vec[k + 1])
    vec[N - 1] = Ayk.reshape(dims[N - 1], out_rks[N - 1], 1, order=F) - bk.reshape(dims[N - 1], out_rks[N - 1], 1, order=F)
    return TTvector(N, vec, tuple(dims), out_rks, ot)


# -------------------------------------------------------------------- gradients
def rayleigh_value_and_grad(H: TToperator, x: TTvector):
    """Gradient of R(x) = <x|H|x>/<x|x> with respect to every core of x (H symmetric).
    The reference has no autodiff; this uses its environment contractions
    (src/als.jl:9-25 `init_H`/`update_H!`, src/tt_operations.jl:390-421):
    dR/dx_k = (2/<x,x>) (Heff_k x_k - R Neff_k x_k)."""
    N = x.N
    # left environments L[k] (before core k): (r, R, r)
    Lh = [None] * (N + 1)
    Ln = [None] * (N + 1)
    Lh[0] = np.ones((1, 1, 1))
    Ln[0] = np.ones((1, 1))
    for k in range(N):
        Lh[k + 1] = ein("abc,iad,ijbe,jcf->def", Lh[k], x.ttv_vec[k], H.tto_vec[k], x.ttv_vec[k])
        Ln[k + 1] = ein("ac,iad,icf->df", Ln[k], x.ttv_vec[k], x.ttv_vec[k])
    Rh = [None] * (N + 1)
    Rn = [None] * (N + 1)
    Rh[N] = np.ones((1, 1, 1))
    Rn[N] = np.ones((1, 1))
    for k in range(N - 1, -1, -1):
        Rh[k] = ein("def,jcf,ijbe,iad->abc", Rh[k + 1], x.ttv_vec[k], H.tto_vec[k], x.ttv_vec[k])
        Rn[k] = ein("df,icf,iad->ac", Rn[k + 1], x.ttv_vec[k], x.ttv_vec[k])
    e = float(Lh[N].reshape(-1)[0])
    nn = float(Ln[N].reshape(-1)[0])
    R = e / nn
    grads = []
    for k in range(N):
        hx = ein("abc,jcf,ijbe,def->iad", Lh[k], x.ttv_vec[k], H.tto_vec[k], Rh[k + 1])
        nx = ein("ac,icf,df->iad", Ln[k], x.ttv_vec[k], Rn[k + 1])
        grads.append((2.0 / nn) * (hx - R * nx))
    return R, grads


# -------------------------------------------------------------------- JSON I/O
def mps_to_json(x: TTvector) -> dict:
    """Inverse of json_to_mps (src/tt_tools.jl:765-774)."""
    return {"N": x.N, "ttv_vec": [c.reshape(-1, order=F).tolist() for c in x.ttv_vec],
            "ttv_dims": list(x.ttv_dims), "ttv_rks": list(x.ttv_rks), "ttv_ot": list(x.ttv_ot)}


def json_to_mps(j: dict) -> TTvector:
    """src/tt_tools.jl:765-774"""
    dims = tuple(int(v) for v in j["ttv_dims"])
    rks = [int(v) for v in j["ttv_rks"]]
    vec = [np.asarray(j["ttv_vec"][i], dtype=np.float64).reshape(dims[i], rks[i], rks[i + 1], order=F)
           for i in range(j["N"])]
    return TTvector(int(j["N"]), vec, dims, rks, [int(v) for v in j["ttv_ot"]])


def mpo_to_json(A: TToperator) -> dict:
    return {"N": A.N, "tto_vec": [c.reshape(-1, order=F).tolist() for c in A.tto_vec],
            "tto_dims": list(A.tto_dims), "tto_rks": list(A.tto_rks), "tto_ot": list(A.tto_ot)}


def json_to_mpo(j: dict) -> TToperator:
    """src/tt_tools.jl:776-785"""
    dims = tuple(int(v) for v in j["tto_dims"])
    rks = [int(v) for v in j["tto_rks"]]
    vec = [np.asarray(j["tto_vec"][i], dtype=np.float64).reshape(dims[i], dims[i], rks[i], rks[i + 1], order=F)
           for i in range(j["N"])]
    return TToperator(int(j["N"]), vec, dims, rks, [int(v) for v in j["tto_ot"]])


# ----------------------------------------------------------------- diagnostics
def rel_error(x: TTvector, y: TTvector) -> float:
    """||x - y|| / ||x|| without dense tensors, FP64: the norm of the difference TT
    (direct sum, then orthogonalize) keeps ~1e-15 accuracy, unlike <x,x> - 2<x,y> + <y,y>."""
    nx = norm(x)
    neg = TTvector(y.N, [-y.ttv_vec[0]] + list(y.ttv_vec[1:]), tuple(y.ttv_dims), list(y.ttv_rks), [0] * y.N)
    d = norm(tt_add(x, neg))
    return d / nx if nx > 0 else d
