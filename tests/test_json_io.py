"""The reference's JSON schema for TT vectors and operators (src/tt_tools.jl:765-785):
json_to_mps / json_to_mpo read it, mps_to_json / mpo_to_json write it (host code, no GPU)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import models_oracle as mo
from oracle import tt_oracle as o


@pytest.fixture(scope="module")
def ttcuda():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if not os.path.exists(os.path.join(root, "tensor-train-julia_b200", "ttcuda", "libttcuda.so")):
        subprocess.check_call([sys.executable, os.path.join(root, "tensor-train-julia_b200", "build.py")])
    import ttcuda as t
    return t


def test_column_major_flat_cores(ttcuda):
    """Core k is a flat list in Julia's column-major order: entry (i, a, b) at i + n (a + r0 b)."""
    x = ttcuda.json_to_mps({"N": 2, "ttv_dims": [2, 2], "ttv_rks": [1, 2, 1], "ttv_ot": [1, 0],
                            "ttv_vec": [[1.0, 2.0, 3.0, 4.0], [5.0, 6.0, 7.0, 8.0]]})
    assert x.ttv_vec[0].shape == (2, 1, 2) and x.ttv_vec[1].shape == (2, 2, 1)
    assert x.ttv_vec[0][1, 0, 0] == 2.0 and x.ttv_vec[0][0, 0, 1] == 3.0
    assert x.ttv_vec[1][1, 0, 0] == 6.0 and x.ttv_vec[1][0, 1, 0] == 7.0
    assert x.ttv_ot == [1, 0]
    A = ttcuda.json_to_mpo({"N": 1, "tto_dims": [2], "tto_rks": [1, 1], "tto_ot": [0],
                            "tto_vec": [[1.0, 2.0, 3.0, 4.0]]})
    assert A.tto_vec[0][1, 0, 0, 0] == 2.0 and A.tto_vec[0][0, 1, 0, 0] == 3.0   # [i_out, j_in, a, a']


def test_round_trip_through_text(ttcuda, tmp_path):
    g = np.random.default_rng(3)
    x = o.rand_tt((2, 3, 2, 4, 2), [1, 2, 5, 4, 2, 1], g, stable=False)
    xt = ttcuda.TTvector(x.N, x.ttv_vec, x.ttv_dims, x.ttv_rks, [1, 1, 0, -1, 0])
    back = ttcuda.json_to_mps(json.loads(json.dumps(ttcuda.mps_to_json(xt))))
    assert back.ttv_dims == xt.ttv_dims and back.ttv_rks == xt.ttv_rks and back.ttv_ot == xt.ttv_ot
    assert all(np.array_equal(a, b) for a, b in zip(back.ttv_vec, xt.ttv_vec))
    H = mo.hubbard_1D(4, t=1.0, U=4.0) if hasattr(mo, "hubbard_1D") else None
    if H is None:
        pytest.skip("no Hubbard builder in the oracle")
    h, V = H
    Ho = mo.hV_to_mpo(h, V, (2,) * h.shape[0])
    A = ttcuda.TToperator(Ho.N, Ho.tto_vec, Ho.tto_dims, Ho.tto_rks)
    path = tmp_path / "tts.json"
    ttcuda.save_json(str(path), [xt, A])
    x2, A2 = ttcuda.load_json(str(path))
    assert all(np.array_equal(a, b) for a, b in zip(x2.ttv_vec, xt.ttv_vec))
    assert A2.tto_rks == A.tto_rks and all(np.array_equal(a, b) for a, b in zip(A2.tto_vec, A.tto_vec))


def test_schema_errors(ttcuda):
    good = {"N": 1, "ttv_dims": [2], "ttv_rks": [1, 1], "ttv_ot": [0], "ttv_vec": [[1.0, 2.0]]}
    ttcuda.json_to_mps(good)
    with pytest.raises(ttcuda.DimensionMismatch):
        ttcuda.json_to_mps(dict(good, ttv_vec=[[1.0, 2.0, 3.0]]))
    with pytest.raises(ttcuda.DimensionMismatch):
        ttcuda.json_to_mps(dict(good, ttv_rks=[1, 1, 1]))
    with pytest.raises(ttcuda.ArgumentError):
        ttcuda.json_to_mps({k: v for k, v in good.items() if k != "ttv_ot"})
    with pytest.raises(ttcuda.ArgumentError):
        ttcuda.json_to_mps(dict(good, ttv_vec=[[1 + 2j, 2.0]]))
