"""Golden fixtures of the TT rounding path: gauge-invariant fingerprints of rounded TTs.

A rounded TT is fixed only up to its gauge (signs and rotations of the cores), so fixtures do not
store cores.  They store what two correct roundings of the same input must share:

* the ranks and orthogonality flags;
* the singular values of every bond (``tt_svdvals``, src/tt_rounding.jl:282-295, all values);
* the norm;
* inner products with a fixed set of seeded rank-2 probe TTs (linear functionals of the
  represented tensor);
* the relative distance to the input, ``||x - y|| / ||x||``.

Inputs that are small are stored in the reference's JSON schema (src/tt_tools.jl:765-785); large
ones (config-3 TTs, the rank-128 vector of config 2) are regenerated from their seeds by the
committed generators, and the fixture stores a checksum of each regenerated input so that a
generator that drifted is caught before any comparison.

Test infrastructure only: the FP64 oracle computes every expected value (``make_golden.py``) and,
in the tests, the fingerprint of the device's output.
"""
from __future__ import annotations

import gzip
import json
import os
from typing import Dict, List, Optional

import numpy as np

from oracle import tt_oracle as o

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE_SEED = 20251204
PROBE_COUNT = 8


def path(name: str) -> str:
    return os.path.join(HERE, name)


def save(name: str, obj: dict) -> None:
    with gzip.open(path(name), "wt", encoding="utf-8") as f:
        json.dump(obj, f)


def load(name: str) -> dict:
    with gzip.open(path(name), "rt", encoding="utf-8") as f:
        return json.load(f)


def probes(dims, count: int = PROBE_COUNT, seed: int = PROBE_SEED) -> List[o.TTvector]:
    """Seeded rank-2 probe TTs with N(0,1) cores (rank-clamped like rand_tt)."""
    g = np.random.default_rng(seed)
    N = len(dims)
    return [o.rand_tt(tuple(dims), [1] + [2] * (N - 1) + [1], g) for _ in range(count)]


def checksum(x: o.TTvector) -> Dict[str, float]:
    """Order-sensitive checksum of a TT's cores (sum, sum of squares, weighted sum)."""
    flat = np.concatenate([np.asarray(c).reshape(-1, order="F") for c in x.ttv_vec])
    w = np.cos(np.arange(flat.size, dtype=np.float64))
    return {"sum": float(flat.sum()), "sumsq": float(flat @ flat), "wsum": float(flat @ w), "size": int(flat.size)}


def checksum_ok(got: Dict[str, float], exp: Dict[str, float], rtol: float = 1e-12) -> bool:
    if got["size"] != exp["size"]:
        return False
    scale = max(1.0, abs(exp["sumsq"]))
    return all(abs(got[k] - exp[k]) <= rtol * scale * 10 for k in ("sum", "sumsq", "wsum"))


def fingerprint(y: o.TTvector, x: Optional[o.TTvector] = None, probe_set=None) -> dict:
    P = probe_set if probe_set is not None else probes(y.ttv_dims)
    sv = o.tt_svdvals(y, tol=0.0)
    return {
        "ranks": [int(r) for r in y.ttv_rks],
        "ot": [int(v) for v in y.ttv_ot],
        "norm": float(o.norm(y)),
        "svals": [[float(v) for v in s] for s in sv],
        "probes": [float(o.dot(y, p)) for p in P],
        "probe_norms": [float(o.norm(p)) for p in P],
        "rel_err_vs_input": None if x is None else float(o.rel_error(x, y)),
    }


def compare(got: dict, exp: dict, tol: float, check_ot: bool = True) -> List[str]:
    """Differences between two fingerprints beyond `tol`: ranks (and ot) must be identical;
    singular values within tol * (largest singular value of the bond); probe values within
    tol * ||y|| * ||probe||; the norm within tol relative; the distance to the input within tol
    (absolute, it is itself a relative quantity)."""
    bad = []
    if got["ranks"] != exp["ranks"]:
        bad.append(f"ranks {got['ranks']} != {exp['ranks']}")
        return bad
    if check_ot and got["ot"] != exp["ot"]:
        bad.append(f"ot {got['ot']} != {exp['ot']}")
    for k, (a, b) in enumerate(zip(got["svals"], exp["svals"])):
        a, b = np.asarray(a), np.asarray(b)
        if a.shape != b.shape:
            bad.append(f"bond {k + 1}: {a.size} singular values, expected {b.size}")
            continue
        if b.size:
            d = float(np.abs(a - b).max() / max(b.max(), 1e-300))
            if d > tol:
                bad.append(f"bond {k + 1}: singular values differ by {d:.3e} (relative to the largest)")
    nrm = exp["norm"]
    if abs(got["norm"] - nrm) > tol * max(nrm, 1e-300):
        bad.append(f"norm {got['norm']!r} != {nrm!r}")
    for j, (a, b, pn) in enumerate(zip(got["probes"], exp["probes"], exp["probe_norms"])):
        if abs(a - b) > tol * max(nrm, 1e-300) * pn:
            bad.append(f"probe {j}: {a!r} != {b!r}")
    if exp.get("rel_err_vs_input") is not None and got.get("rel_err_vs_input") is not None:
        if abs(got["rel_err_vs_input"] - exp["rel_err_vs_input"]) > tol:
            bad.append(f"distance to the input {got['rel_err_vs_input']:.6e} != {exp['rel_err_vs_input']:.6e}")
    return bad
