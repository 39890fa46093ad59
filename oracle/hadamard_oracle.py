"""FP64 CPU restatement of the randomized rounding of a Hadamard product -- TEST INFRASTRUCTURE.

The oracle of the library's ttc_ttrand_rounding_hadamard: only tests/ may import it.

  hadamard                     src/tt_operations.jl:273-287 (*(x, y): slice-wise Kronecker cores)
  ttrand_rounding_hadamard     src/tt_randtools.jl:364-473 with the Kronecker sketch of
                               src/sketches.jl:474-605 (reverse)

The reference sketches and projects the product y_1 * ... * y_M without forming it, with
Kronecker contraction kernels.  Here the product TT is formed (rank prod r_i) and rounded by
tt_oracle.ttrand_rounding: the sketch blocks are the same draws (they depend on the dimensions,
block ranks and counts only), the sketch of the product is the same tensor contraction, and each
range-finder matrix Z_k = (projected left part) x (unfolding) x (right sketch) depends on the
represented tensor only, not on the order of the combined rank index, so every Q and the result
are the reference's.  This is an independent computation of what the device's structured kernels
compute.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import tt_oracle as o


def hadamard(x: o.TTvector, y: o.TTvector) -> o.TTvector:
    """src/tt_operations.jl:273-287: core k slice i = kron(x_k[i], y_k[i]) (y's index fastest)."""
    N = x.N
    rks = [a * b for a, b in zip(x.ttv_rks, y.ttv_rks)]
    vec = []
    for k in range(N):
        n = x.ttv_dims[k]
        c = np.zeros((n, rks[k], rks[k + 1]))
        for i in range(n):
            c[i] = np.kron(x.ttv_vec[k][i], y.ttv_vec[k][i])
        vec.append(c)
    return o.TTvector(N, vec, tuple(x.ttv_dims), rks, [0] * N)


def ttrand_rounding_hadamard(ys: Sequence[o.TTvector], rks, orthogonal=True, seed=1234, block_rks=None,
                             rng_kind="philox") -> o.TTvector:
    """ttrand_rounding(y::NTuple, rks; ...) (src/tt_randtools.jl:364-473), M = len(ys) >= 1."""
    P = ys[0]
    for t in ys[1:]:
        P = hadamard(P, t)
    return o.ttrand_rounding(P, rks, orthogonal, seed, block_rks, rng_kind=rng_kind)
