"""Conversions between oracle and ttcuda tensors, and comparison helpers for the GPU tests."""
import math

import numpy as np

import ttcuda
from oracle import tt_oracle as o


def to_dev(x: o.TTvector) -> ttcuda.TTvector:
    return ttcuda.TTvector(x.N, x.ttv_vec, x.ttv_dims, x.ttv_rks, x.ttv_ot)


def to_or(x: ttcuda.TTvector) -> o.TTvector:
    return o.TTvector(x.N, [np.array(c) for c in x.ttv_vec], tuple(x.ttv_dims), list(x.ttv_rks), list(x.ttv_ot))


def op_dev(A: o.TToperator) -> ttcuda.TToperator:
    return ttcuda.TToperator(A.N, A.tto_vec, A.tto_dims, A.tto_rks, A.tto_ot)


def rel(a, b) -> float:
    """||a - b|| / ||b|| for two TTs (oracle or ttcuda), computed with the FP64 oracle as the
    norm of the difference TT (orthogonalisation), which is accurate to ~1e-15; the
    expansion <a,a> - 2<a,b> + <b,b> would cancel down to ~1e-8."""
    a = to_or(a) if isinstance(a, ttcuda.TTvector) else a
    b = to_or(b) if isinstance(b, ttcuda.TTvector) else b
    return o.rel_error(b, a)


def rel_dense(a, b) -> float:
    A = o.ttv_to_tensor(to_or(a) if isinstance(a, ttcuda.TTvector) else a)
    Bd = o.ttv_to_tensor(to_or(b) if isinstance(b, ttcuda.TTvector) else b)
    return float(np.linalg.norm(A - Bd) / max(np.linalg.norm(Bd), 1e-300))


def sum_of_tts(dims, r, m, seed):
    """Config-1 style input: X = sum_{j=1..m} 2^-j X_j, X_j = rand_tt(dims, r)."""
    g = np.random.default_rng(seed)
    X = None
    for j in range(1, m + 1):
        Xj = o.rand_tt(dims, r, g)
        Xj = o.tt_scale(2.0 ** -j, Xj)
        X = Xj if X is None else o.tt_add(X, Xj)
    return X


def left_orth_cores(dims, ranks, g):
    """Left-orthonormal cores with the given ranks (last core unnormalised)."""
    N = len(dims)
    vec = []
    for k in range(N):
        n, a, b = dims[k], ranks[k], ranks[k + 1]
        if k < N - 1:
            q, _ = np.linalg.qr(g.standard_normal((n * a, b)))
            vec.append(q.reshape(n, a, b, order="F") if False else np.transpose(q.reshape(a, n, b, order="F"), (1, 0, 2)))
        else:
            vec.append(g.standard_normal((n, a, b)))
    return vec


def decaying_tt(dims, ranks, seed, decay_per=32.0):
    """Synthetic TT with singular values ~10^(-i/decay_per) at every bond: left-orthonormal
    random cores, each bond's diagonal decay absorbed into the next core."""
    g = np.random.default_rng(seed)
    N = len(dims)
    vec = []
    prev = np.ones(1)
    for k in range(N):
        n, a, b = dims[k], ranks[k], ranks[k + 1]
        if k < N - 1:
            m = n * a
            q, _ = np.linalg.qr(g.standard_normal((m, max(b, 1))))
            q = q[:, :b] if q.shape[1] >= b else np.pad(q, ((0, 0), (0, b - q.shape[1])))
            core = np.transpose(q.reshape(a, n, b, order="F"), (1, 0, 2)).copy()
        else:
            core = g.standard_normal((n, a, b))
            core /= np.linalg.norm(core)
        core = core * prev[None, :, None]
        vec.append(np.asfortranarray(core))
        prev = 10.0 ** (-np.arange(b) / decay_per)
        prev /= np.sqrt(np.mean(prev ** 2))      # unit RMS: the TT norm stays O(1) along the train
    return o.TTvector(N, vec, tuple(dims), list(ranks), [0] * N)
