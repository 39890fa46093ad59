"""The reference's JSON schema for TT vectors and operators (src/tt_tools.jl:765-785).

A TTvector is a JSON object with the fields of the Julia struct: `N`, `ttv_dims`, `ttv_rks`,
`ttv_ot` and `ttv_vec`, where core k is a flat list of its n_k * r_{k-1} * r_k entries in
Julia's column-major order (physical index fastest); a TToperator has `N`, `tto_dims`,
`tto_rks`, `tto_ot` and `tto_vec`, core k a flat list of n_k * n_k * R_{k-1} * R_k entries.
`json_to_mps` / `json_to_mpo` read a parsed object into the host types of this package, as the
reference's functions of the same names do; `mps_to_json` / `mpo_to_json` write the same
schema, so tensors move between the reference and this library as files.  Entries are real
(FP64): a complex object is refused, since the device path computes in FP64.
"""
from __future__ import annotations

import json
from typing import Any, Dict

import numpy as np

from . import ArgumentError, DimensionMismatch, TToperator, TTvector


def _field(x: Dict[str, Any], name: str):
    if name not in x:
        raise ArgumentError(f"JSON tensor train: missing field {name!r}")
    return x[name]


def _real_core(flat, shape, what: str) -> np.ndarray:
    a = np.asarray(flat)
    if a.dtype.kind == "c" or a.dtype == object:
        raise ArgumentError(f"{what}: entries must be real numbers")
    a = a.astype(np.float64).ravel()
    if a.size != int(np.prod(shape)):
        raise DimensionMismatch(f"{what}: {a.size} entries for a core of shape {tuple(shape)}")
    return a.reshape(shape, order="F")


def json_to_mps(x: Dict[str, Any]) -> TTvector:
    """src/tt_tools.jl:765-774: a parsed TTvector object -> TTvector."""
    N = int(_field(x, "N"))
    dims = [int(v) for v in _field(x, "ttv_dims")]
    rks = [int(v) for v in _field(x, "ttv_rks")]
    ot = [int(v) for v in _field(x, "ttv_ot")]
    vec = _field(x, "ttv_vec")
    if len(dims) != N or len(rks) != N + 1 or len(ot) != N or len(vec) != N:
        raise DimensionMismatch("JSON TTvector: N, ttv_dims, ttv_rks, ttv_ot and ttv_vec disagree")
    cores = [_real_core(vec[i], (dims[i], rks[i], rks[i + 1]), f"ttv_vec[{i + 1}]") for i in range(N)]
    return TTvector(N, cores, dims, rks, ot)


def json_to_mpo(x: Dict[str, Any]) -> TToperator:
    """src/tt_tools.jl:776-785: a parsed TToperator object -> TToperator."""
    N = int(_field(x, "N"))
    dims = [int(v) for v in _field(x, "tto_dims")]
    rks = [int(v) for v in _field(x, "tto_rks")]
    ot = [int(v) for v in _field(x, "tto_ot")]
    vec = _field(x, "tto_vec")
    if len(dims) != N or len(rks) != N + 1 or len(ot) != N or len(vec) != N:
        raise DimensionMismatch("JSON TToperator: N, tto_dims, tto_rks, tto_ot and tto_vec disagree")
    cores = [_real_core(vec[i], (dims[i], dims[i], rks[i], rks[i + 1]), f"tto_vec[{i + 1}]") for i in range(N)]
    return TToperator(N, cores, dims, rks, ot)


def mps_to_json(x: TTvector) -> Dict[str, Any]:
    """TTvector -> an object of the schema json_to_mps reads (flat column-major cores)."""
    return {"N": x.N, "ttv_dims": list(x.ttv_dims), "ttv_rks": list(x.ttv_rks), "ttv_ot": list(x.ttv_ot),
            "ttv_vec": [np.asarray(c).ravel(order="F").tolist() for c in x.ttv_vec]}


def mpo_to_json(A: TToperator) -> Dict[str, Any]:
    """TToperator -> an object of the schema json_to_mpo reads."""
    return {"N": A.N, "tto_dims": list(A.tto_dims), "tto_rks": list(A.tto_rks), "tto_ot": list(A.tto_ot),
            "tto_vec": [np.asarray(c).ravel(order="F").tolist() for c in A.tto_vec]}


def load_json(path: str):
    """Read a file of the schema: a TTvector object, a TToperator object, or a list of them."""
    with open(path) as f:
        obj = json.load(f)

    def one(o):
        return json_to_mpo(o) if "tto_vec" in o else json_to_mps(o)
    return [one(o) for o in obj] if isinstance(obj, list) else one(obj)


def save_json(path: str, t) -> None:
    """Write a TTvector, a TToperator or a list of them in the schema."""
    def one(o):
        return mpo_to_json(o) if isinstance(o, TToperator) else mps_to_json(o)
    with open(path, "w") as f:
        json.dump([one(o) for o in t] if isinstance(t, (list, tuple)) else one(t), f)
