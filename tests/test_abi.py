"""CPU checks of the C-ABI boundary: the library loads and exports every entry point
declared in include/ttcuda.h; the host-side helpers mirror the reference."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ttcuda.h")
LIB = os.path.join(ROOT, "tensor-train-julia_b200", "ttcuda", "libttcuda.so")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ttc_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def built_lib():
    if not os.path.exists(LIB):
        import subprocess
        import sys
        subprocess.check_call([sys.executable, os.path.join(ROOT, "tensor-train-julia_b200", "build.py")])
    return ctypes.CDLL(LIB)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["ttc_tt_rounding", "ttc_ttrand_rounding", "ttc_recursive_sketch", "ttc_mpo_apply",
                 "ttc_batch_round_det", "ttc_batch_round_rand", "ttc_dot_operator", "ttc_rayleigh_grad"]:
        assert must in names


def test_library_exports_every_declared_symbol(built_lib):
    missing = [n for n in declared_functions() if not hasattr(built_lib, n)]
    assert not missing, f"symbols declared in include/ttcuda.h but not exported: {missing}"


def test_python_binding_loads_and_reports_version(built_lib):
    import ttcuda
    assert "sm_100a" in ttcuda.version()


def test_host_helpers_match_oracle():
    import ttcuda
    from oracle import tt_oracle as o
    dims = (2,) * 10
    assert ttcuda.r_and_d_to_rks([1] + [64] * 9 + [1], dims) == o.r_and_d_to_rks([1] + [64] * 9 + [1], dims)
    import numpy as np
    g = np.random.default_rng(0)
    x = o.rand_tt(dims, [1, 2, 4, 8, 5, 7, 8, 4, 3, 2, 1], g, stable=False)
    xt = ttcuda.TTvector(x.N, x.ttv_vec, x.ttv_dims, x.ttv_rks, x.ttv_ot)
    assert ttcuda.default_rank_heuristic(xt) == o.default_rank_heuristic(x)
    assert ttcuda._sketch_ranks(dims, o.default_rank_heuristic(x), 32) == \
        [b * p for b, p in zip(*o.sketch_plan(dims, 10, o.default_rank_heuristic(x), 32))]


def test_no_gpu_calls_fail_cleanly_without_device(built_lib):
    """Without a GPU, creating a context must fail with a status, not crash."""
    import ttcuda
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(Exception):
        ttcuda.Context(0)


def test_sketch_precision_names(built_lib):
    """precision is 'fp64', 'bf16' or 'tf32' (TTC_PREC_FP64/_BF16/_TF32); anything else is an
    ArgumentError before any device work."""
    import ttcuda
    keep = ttcuda._Keep()
    assert [ttcuda._sketch_opts(True, 1, None, p, None, keep).precision for p in ("fp64", "bf16", "tf32")] == [0, 1, 2]
    with pytest.raises(ttcuda.ArgumentError):
        ttcuda._sketch_opts(True, 1, None, "fp16", None, keep)


def test_ttvector_marshalling_cache(built_lib):
    """The ctypes view of a TTvector is cached while its core arrays and dims/ranks/ot are the
    same (in-place core updates keep the pointers valid); replacing a core or changing the ranks
    rebuilds it, and copies do not carry it."""
    import copy

    import numpy as np
    import ttcuda
    t = ttcuda.TTvector(3, [np.ones((2, 1, 2), order="F"), np.ones((2, 2, 2), order="F"),
                            np.ones((2, 2, 1), order="F")], (2, 2, 2), [1, 2, 2, 1])
    keep = ttcuda._Keep()
    a = ttcuda._ttv(t, keep)
    cached = t._marshal
    t.ttv_vec[1][0, 0, 0] = 5.0                     # in place: same arrays, same view
    ttcuda._ttv(t, keep)
    assert t._marshal is cached
    assert C_addr(a.cores, 1) == t.ttv_vec[1].__array_interface__["data"][0]
    t.ttv_vec[1] = np.zeros((2, 2, 2), order="F")   # replaced core: rebuilt, new pointer
    b = ttcuda._ttv(t, keep)
    assert t._marshal is not cached
    addr = C_addr(b.cores, 1)
    assert addr == t.ttv_vec[1].__array_interface__["data"][0]
    t.ttv_rks[1] = 2                                # same values: still cached
    ttcuda._ttv(t, keep)
    assert t._marshal[0][2] == (1, 2, 2, 1)
    assert not hasattr(copy.copy(t), "_marshal") and not hasattr(copy.deepcopy(t), "_marshal")
    c_ord = ttcuda.TTvector(1, [np.ones((2, 1, 1))], (2,), [1, 1])   # non-Fortran input is converted
    assert c_ord.ttv_vec[0].flags.f_contiguous


def test_marshalling_of_converted_core_sees_in_place_edits(built_lib):
    """A core that is not a Fortran-ordered float64 array (here a C-ordered one assigned after
    construction) is marshalled as a converted copy: that copy is not cached, so an in-place
    edit of the user's array reaches the next call instead of a stale copy."""
    import numpy as np
    import ttcuda
    t = ttcuda.TTvector(2, [np.ones((2, 1, 2), order="F"), np.ones((2, 2, 1), order="F")], (2, 2), [1, 2, 1])
    keep = ttcuda._Keep()
    ttcuda._ttv(t, keep)
    assert hasattr(t, "_marshal")
    core = np.ascontiguousarray(np.arange(4.0).reshape(2, 2, 1))       # C-ordered
    t.ttv_vec[1] = core
    a = ttcuda._ttv(t, keep)
    assert not hasattr(t, "_marshal")
    first = np.ctypeslib.as_array(ctypes.cast(a.cores[1], ctypes.POINTER(ctypes.c_double)), shape=(4,)).copy()
    core[1, 0, 0] = 42.0                                                # in-place edit of the user's array
    b = ttcuda._ttv(t, keep)
    second = np.ctypeslib.as_array(ctypes.cast(b.cores[1], ctypes.POINTER(ctypes.c_double)), shape=(4,)).copy()
    assert first[1] == 2.0 and second[1] == 42.0         # column-major (2,2,1): element (1,0,0) is second
    assert not hasattr(t, "_marshal")


def C_addr(pp, i):
    import ctypes
    return ctypes.cast(pp[i], ctypes.c_void_p).value
