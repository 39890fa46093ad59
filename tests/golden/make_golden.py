"""Writes the golden fixtures of tests/golden/ from the FP64 oracle.

    python tests/golden/make_golden.py            # all fixtures (a few minutes on 8 cores)

Each fixture holds the inputs (in the reference's JSON schema when small, else the seeds of the
committed generators plus checksums of the regenerated tensors), the call's arguments, and the
oracle's results as fingerprints (golden.py).  The GPU tests (tests/test_golden_gpu.py) run the
library on the same inputs and compare; the CPU tests (tests/test_golden.py) re-derive the cheap
fixtures from the oracle and check that the generators still reproduce the stored inputs.

Fixtures:
  config1_sum_of_tts.json.gz  X = sum_{j=1..8} 2^-j X_j, X_j rank-8 N(0,1) TTs, n=2, d=20;
                              tt_rounding(X; tol=1e-8, rmax=64)            (src/tt_rounding.jl:146)
  config3_batch3.json.gz      the first 3 TTs of the 64-TT batched-rounding workload (d=32, n=2,
                              ranks U[16,256], sigma_i = 10^(-i/32)); tt_rounding(tol=1e-8), and
                              ttrand_rounding with the batch's default_rank_heuristic ranks and
                              the given sketch blocks, then tt_rounding(tol=1e-8)
                              (src/tt_randtools.jl:112-154, :476-480)
  config2_hubbard_op.json.gz  1D Hubbard MPO (16 sites, t=1, U=4) by hV_to_mpo, applied to a
                              seeded rank-128 TT without forming the product: Gaussian sketch of
                              rank 138 (block_rks=138), ttrand_rounding([1.0], H, [y], rks)
                              (src/tt_randtools.jl:285-354)
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import bench  # noqa: E402  the config-3 workload generator (bench.workload)
import golden  # noqa: E402
from oracle import models_oracle as mo  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402

CONFIG1 = {"dims": [2] * 20, "terms": 8, "term_rank": 8, "seed": 101, "tol": 1e-8, "rmax": 64}
CONFIG3 = {"workload_seed": 7, "count": 3, "tol": 1e-8, "sketch_seed": 1234, "orthogonal": True}
CONFIG2 = {"sites": 16, "t": 1.0, "U": 4.0, "y_rank": 128, "y_seed": 40, "s": 138, "sketch_seed": 5,
           "orthogonal": False}


def config1_terms():
    g = np.random.default_rng(CONFIG1["seed"])
    dims = tuple(CONFIG1["dims"])
    return [o.rand_tt(dims, CONFIG1["term_rank"], g) for _ in range(CONFIG1["terms"])]


def config1_input(terms):
    X = None
    for j, t in enumerate(terms, start=1):
        t = o.tt_scale(2.0 ** -j, t)
        X = t if X is None else o.tt_add(X, t)
    return X


def config3_inputs():
    dims, tts = bench.workload(seed=CONFIG3["workload_seed"], batch=CONFIG3["count"])
    return [o.TTvector(len(d), [np.asfortranarray(c) for c in v], tuple(d), list(r), [0] * len(d)) for d, r, v in tts]


def config3_rks():
    """default_rank_heuristic of the whole 64-TT batch (the ranks the benchmark rounds with)."""
    g = np.random.default_rng(CONFIG3["workload_seed"])
    dims = (bench.NPHYS,) * bench.D
    ranks = []
    for _ in range(bench.BATCH):
        r = [1] + [int(v) for v in g.integers(bench.RMIN, bench.RMAX + 1, size=bench.D - 1)] + [1]
        ranks.append(bench.r_and_d(r, dims, max(r)))
    return bench.heuristic(ranks)


def config3_blocks(rks, N, dims):
    return o.make_reverse_sketch(dims, rks, seed=CONFIG3["sketch_seed"], orthogonal=CONFIG3["orthogonal"],
                                 block_rks=N)


def config2_inputs():
    h, V = mo.hubbard_1D(CONFIG2["sites"], t=CONFIG2["t"], U=CONFIG2["U"])
    N = 2 * CONFIG2["sites"]
    H = mo.hV_to_mpo(h, V, (2,) * N)
    y = o.rand_tt((2,) * N, CONFIG2["y_rank"], np.random.default_rng(CONFIG2["y_seed"]), normalise=True)
    return H, y


def make_config1():
    terms = config1_terms()
    X = config1_input(terms)
    Y = o.tt_rounding(X, tol=CONFIG1["tol"], rmax=CONFIG1["rmax"])
    golden.save("config1_sum_of_tts.json.gz", {
        "description": "tt_rounding(X; tol=1e-8, rmax=64) of X = sum_j 2^-j X_j (terms in the reference's "
                       "JSON schema, src/tt_tools.jl:765-785; X formed with +(TT,TT) and *(a,TT))",
        "params": CONFIG1,
        "terms": [o.mps_to_json(t) for t in terms],
        "input_checksum": golden.checksum(X),
        "expected": golden.fingerprint(Y, X),
    })


def make_config3():
    xs = config3_inputs()
    rks = config3_rks()
    N = xs[0].N
    blocks, b, p = config3_blocks(rks, N, xs[0].ttv_dims)
    det, mixed, sums = [], [], []
    for x in xs:
        yd = o.tt_rounding(x, tol=CONFIG3["tol"])
        z = o.ttrand_rounding(x, rks, orthogonal=CONFIG3["orthogonal"], block_rks=N, blocks=blocks)
        ym = o.tt_rounding(z, tol=CONFIG3["tol"])
        fd = golden.fingerprint(yd, x)
        fm = golden.fingerprint(ym, x)
        # both roundings approximate x to the same tolerance with the same ranks
        assert fd["ranks"] == fm["ranks"], "oracle: randomized and deterministic ranks differ"
        det.append(fd)
        mixed.append(fm)
        sums.append(golden.checksum(x))
    golden.save("config3_batch3.json.gz", {
        "description": "first 3 TTs of the batched-rounding workload (bench.workload(seed=7)); "
                       "tt_rounding(tol=1e-8) and ttrand_rounding(rks; orthogonal sketch blocks from the "
                       "Philox4x32-10 stream of seed 1234, block_rks=N) followed by tt_rounding(tol=1e-8)",
        "params": CONFIG3, "rks": rks, "sketch_block_ranks": b, "sketch_block_counts": p,
        "input_checksums": sums, "expected_det": det, "expected_rand_then_det": mixed,
    })


def make_config2():
    H, y = config2_inputs()
    N = y.N
    s = CONFIG2["s"]
    rks = [1] + [s] * (N - 1) + [1]
    z = o.ttrand_rounding_op([1.0], H, [y], rks, orthogonal=CONFIG2["orthogonal"], seed=CONFIG2["sketch_seed"],
                             block_rks=s)
    Hy = o.tto_apply(H, y)
    golden.save("config2_hubbard_op.json.gz", {
        "description": "ttrand_rounding([1.0], H, [y], rks) with H the 1D Hubbard MPO (hV_to_mpo, 32 "
                       "spin-orbitals, t=1, U=4; stored in the reference's JSON schema), y a seeded N(0,1) "
                       "rank-128 TT (normalised), Gaussian sketch blocks of rank 138 from the Philox4x32-10 "
                       "stream of seed 5 (block_rks=138, one block per site)",
        "params": CONFIG2, "rks": rks, "mpo": o.mpo_to_json(H), "y_checksum": golden.checksum(y),
        "expected": golden.fingerprint(z, Hy),
    })


if __name__ == "__main__":
    which = sys.argv[1:] or ["config1", "config2", "config3"]
    for name, fn in (("config1", make_config1), ("config2", make_config2), ("config3", make_config3)):
        if name in which:
            t0 = time.time()
            fn()
            print(f"{name}: {time.time() - t0:.1f} s", flush=True)
