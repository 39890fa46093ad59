"""FP64 CPU restatement of the streaming TT approximation (STTA) -- TEST INFRASTRUCTURE.

The oracle of the library's STTA: only tests/ may import it; the product never does.

  tt_recursive_sketch_forward   src/sketches.jl:175-185, :241-305 (reverse=false, oversampling)
  contract_sketch_core_forwards src/sketches.jl:1192-1230
  stta_sketch                   src/sketches.jl:1126-1160
  stable_inverse                src/tt_randtools.jl:485-489
  stta (single and lincomb)     src/tt_randtools.jl:551-641 (rmax variants :584-590, :635-641)

Sketch blocks come from the same Philox streams as the reverse sketch (SketchRNG, stream = the
core's 0-based index), so the GPU and this restatement draw the same blocks.  Parity is pinned
through tt_oracle's pins plus the algebraic checks in tests/test_stta_oracle.py (STTA is exact
when the sketch ranks reach the TT ranks).
"""
from __future__ import annotations

import math
from typing import List, Sequence

import numpy as np

from . import tt_oracle as o

F = "F"


def forward_block_ranks(dims, N, block_rks):
    """src/sketches.jl:244-248: b[0] = 1, b[k+1] = min(block_rks, dims[k] b[k])."""
    b = [1] * (N + 1)
    for k in range(1, N + 1):
        b[k] = block_rks
    for k in range(N):
        b[k + 1] = min(b[k + 1], dims[k] * b[k])
    return b


def forward_sketch_plan(dims, N, rks, block_rks=None, oversampling=1.0):
    """Block ranks and counts of the forward sketch (src/sketches.jl:243-258)."""
    block_rks = N if block_rks is None else block_rks
    b = forward_block_ranks(dims, N, block_rks)
    p = o.compute_sketch_blocks_heuristic(list(rks), b, N, reverse=False)
    if oversampling != 1:
        for k in range(1, N + 1):
            p[k] = int(math.ceil(oversampling * p[k]))
    return b, p


def contract_sketch_core_forwards(A: np.ndarray, S: np.ndarray, V: np.ndarray) -> np.ndarray:
    """src/sketches.jl:1192-1230: W[a,b] = sum A[z,al,a] S[be,z,b] V[al,be], in the order the
    reference's cost test picks: (V^T A) S or A (V S)."""
    z, al, a = A.shape
    be, _, b = S.shape
    if a * (be + 1) * (al + b) < al * b * (a + be + 1):
        return o.ein("Ab,zAa,bzc->ac", V, A, S)
    return o.ein("Ab,bzc,zAa->ac", V, S, A)


def tt_recursive_sketch_forward(A: o.TTvector, rks, orthogonal=True, seed=1234, block_rks=None, oversampling=1.0,
                                rng_kind="philox"):
    """src/sketches.jl:241-305 (reverse=false): W[k+1] = contraction of cores 0..k with the
    sketch blocks, left to right.  Returns (W list of (r_k, b_k p_k), sketch ranks b .* p)."""
    N, dims = A.N, A.ttv_dims
    assert rks[0] == 1 and A.ttv_rks[0] == 1
    b, p = forward_sketch_plan(dims, N, rks, block_rks, oversampling)
    rng = o.SketchRNG(seed, rng_kind)
    W = [None] * (N + 1)
    W[0] = np.ones((1, 1, 1))
    for k in range(N):
        blocks = o.generate_sketch_blocks(rng, k, b[k], dims[k], b[k + 1], p[k + 1], orthogonal)
        Wn = np.zeros((A.ttv_rks[k + 1], b[k + 1], p[k + 1]))
        for j in range(p[k + 1]):
            Wn[:, :, j] = contract_sketch_core_forwards(A.ttv_vec[k], blocks[:, :, :, j],
                                                        W[k][:, :, j if k > 0 else 0])
        W[k + 1] = Wn
    for k in range(N + 1):
        W[k] = W[k] / math.sqrt(p[k])
    return [W[k].reshape(A.ttv_rks[k], b[k] * p[k], order=F) for k in range(N + 1)], [x * y for x, y in zip(b, p)]


def stta_sketch(x: o.TTvector, rks, seed_left=1234, seed_right=5678, orthogonal=True, block_rks=None,
                rng_kind="philox"):
    """src/sketches.jl:1126-1160: left (forward, 1.5x block oversampling) and right (reverse)
    sketches, Omega[k] = W_left[k+1]^T W_right[k+1] and Psi[k] = x_k x_1 W_left[k] x_3 W_right[k+1]."""
    N = x.N
    WL, sl = tt_recursive_sketch_forward(x, rks, orthogonal, seed_left, block_rks, 1.5, rng_kind)
    WR, sr = o.tt_recursive_sketch(x, rks, orthogonal, seed_right, block_rks, rng_kind=rng_kind)
    Om = [WL[k + 1].T @ WR[k + 1] for k in range(N - 1)]
    Psi = [o.ein("iab,aA,bB->iAB", x.ttv_vec[k], WL[k], WR[k + 1]) for k in range(N)]
    return Om, Psi


def stable_inverse(A: np.ndarray, eps=1e-12) -> np.ndarray:
    """src/tt_randtools.jl:485-489: pseudo-inverse from the SVD, keeping s > max(s) eps."""
    u, s, vh = o.svd_julia(A)
    keep = s > s.max() * eps if s.size else np.zeros(0, bool)
    return vh[keep].T @ np.diag(1.0 / s[keep]) @ u[:, keep].T


def _stta_from(Om, Psi, dims) -> o.TTvector:
    """src/tt_randtools.jl:562-579 / :614-630: Psi cores joined through the pseudo-inverses of
    Omega, on the side of the smaller sketch rank."""
    N = len(Psi)
    P = [c.copy() for c in Psi]
    rks = [1] * (N + 1)
    for k in range(N - 1):
        rl, rr = Om[k].shape
        if rl < rr:
            n, a, _ = P[k].shape
            P[k] = (P[k].reshape(n * a, rr, order=F) @ stable_inverse(Om[k])).reshape(n, a, rl, order=F)
            rks[k + 1] = rl
        else:
            n, _, c = P[k + 1].shape
            M = np.transpose(P[k + 1], (1, 0, 2)).reshape(rl, n * c, order=F)
            P[k + 1] = np.transpose((stable_inverse(Om[k]) @ M).reshape(rr, n, c, order=F), (1, 0, 2))
            rks[k + 1] = rr
    return o.TTvector(N, P, tuple(dims), rks, [0] * N)


def stta(y: o.TTvector, rks=None, seed_left=1234, seed_right=5678, orthogonal=True, block_rks=None,
         rng_kind="philox") -> o.TTvector:
    """src/tt_randtools.jl:551-590 (rks vector, int rmax, or the default heuristic)."""
    N = y.N
    if rks is None:
        rks = o.default_rank_heuristic(y)
    elif isinstance(rks, (int, np.integer)):
        rks = [1] + [int(rks)] * (N - 1) + [1]
    Om, Psi = stta_sketch(y, rks, seed_left, seed_right, orthogonal, block_rks, rng_kind)
    return _stta_from(Om, Psi, y.ttv_dims)


def stta_lincomb(alpha: Sequence[float], ys: Sequence[o.TTvector], rks, seed_left=1234, seed_right=5678,
                 orthogonal=True, block_rks=None, rng_kind="philox") -> o.TTvector:
    """src/tt_randtools.jl:592-641: STTA of sum_j alpha_j ys[j] from the summed sketches."""
    N = ys[0].N
    if isinstance(rks, (int, np.integer)):
        rks = [1] + [int(rks)] * (N - 1) + [1]
    Om, Psi = None, None
    for a, y in zip(alpha, ys):
        Oj, Pj = stta_sketch(y, rks, seed_left, seed_right, orthogonal, block_rks, rng_kind)
        if Om is None:
            Om, Psi = [a * m for m in Oj], [a * c for c in Pj]
        else:
            Om = [m + a * mj for m, mj in zip(Om, Oj)]
            Psi = [c + a * cj for c, cj in zip(Psi, Pj)]
    return _stta_from(Om, Psi, ys[0].ttv_dims)
