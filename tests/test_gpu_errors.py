"""Error paths of the library on the GPU, each made to happen on purpose in a safe form, and the
context checked to stay usable afterwards:

* a NaN in an input core -> TTC_ENONFINITE (ArgumentError in the host mirror), raised from the
  device flag the Householder QR sets;
* the Jacobi SVD sweep cap lowered through a test hook so that the sweep runs out of sweeps ->
  TTC_ENOCONV on the asynchronous path (reported by ttc_synchronize), and on the synchronous path
  the library's single retry at four times the cap (the reference retries a failed gesdd with QR
  iteration, src/tt_rounding.jl:191-195), which then succeeds and is counted in ttc_stats;
* a kernel descriptor pointing outside every device allocation of the library -> TTC_EINTERNAL
  from the host-side registry check, before anything is launched;
* the tensor-core GEMM's bounded mbarrier waits set to give up at once through a test hook -> DFLAG_TIMEOUT, reported as TTC_EINTERNAL after the kernel drained the MMAs it
  issued and returned.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
from gpu_helpers import decaying_tt, rel, to_dev  # noqa: E402
from oracle import tt_oracle as o  # noqa: E402
from ttcuda._lib import lib  # noqa: E402

lib.ttc_test_set_jacobi_max_sweeps.argtypes = [C.c_void_p, C.c_int]
lib.ttc_test_set_jacobi_max_sweeps.restype = C.c_int
lib.ttc_test_bad_descriptor.argtypes = [C.c_void_p, C.c_longlong]
lib.ttc_test_bad_descriptor.restype = C.c_int
lib.ttc_test_set_tc_wait_limit.argtypes = [C.c_void_p, C.c_longlong]
lib.ttc_test_set_tc_wait_limit.restype = C.c_int
lib.ttc_test_tc_gemm_bench.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
lib.ttc_test_tc_gemm_bench.restype = C.c_int


@pytest.fixture()
def ctx():
    c = ttcuda.get_context()
    yield c
    c.check(lib.ttc_test_set_jacobi_max_sweeps(c.h, 40))
    c.check(lib.ttc_test_set_tc_wait_limit(c.h, 1 << 24))


def _still_usable():
    x = decaying_tt((2,) * 10, o.r_and_d_to_rks([1] + [12] * 9 + [1], (2,) * 10), seed=77, decay_per=3.0)
    ref = o.tt_rounding(x, tol=1e-6)
    got = ttcuda.tt_rounding(to_dev(x), tol=1e-6)
    assert got.ttv_rks == ref.ttv_rks
    assert rel(got, ref) < 1e-10


def test_nan_core_raises_nonfinite_and_context_recovers(ctx):
    x = decaying_tt((2,) * 10, o.r_and_d_to_rks([1] + [12] * 9 + [1], (2,) * 10), seed=5, decay_per=3.0)
    x.ttv_vec[3] = x.ttv_vec[3].copy()
    x.ttv_vec[3][1, 2, 3] = np.nan
    with pytest.raises(ttcuda.ArgumentError, match="NaN or Inf"):
        ttcuda.tt_rounding(to_dev(x), tol=1e-8)
    _still_usable()
    xb = ttcuda.DeviceBatch.from_tts([to_dev(x)])
    s = ttcuda._sketch_ranks(x.ttv_dims, [1] + [20] * 9 + [1], 10)
    yb = ttcuda.DeviceBatch(x.ttv_dims, [ttcuda._rand_out_caps(x.ttv_dims, s)])
    with pytest.raises(ttcuda.ArgumentError, match="NaN or Inf"):
        xb.round_rand(yb, [1] + [20] * 9 + [1], precision="bf16", after_tol=1e-8)
    _still_usable()


def _hard_batch():
    dims = (2,) * 12
    tts = [decaying_tt(dims, o.r_and_d_to_rks([1] + [40] * 11 + [1], dims), seed=90 + i, decay_per=8.0)
           for i in range(2)]
    return dims, tts


def test_sweep_cap_exhausted_async_reports_noconv(ctx):
    dims, tts = _hard_batch()
    ctx.check(lib.ttc_test_set_jacobi_max_sweeps(ctx.h, 1))
    xb = ttcuda.DeviceBatch.from_tts([to_dev(t) for t in tts])
    yb = ttcuda.DeviceBatch(dims, [t.ttv_rks for t in tts])
    before = ctx.stats()["svd_retries"]
    xb.round_det(yb, tol=1e-8, sync=False)          # the asynchronous path does not retry
    with pytest.raises(ttcuda.LAPACKException, match="sweep cap"):
        ctx.synchronize()
    assert ctx.stats()["svd_retries"] == before
    ctx.check(lib.ttc_test_set_jacobi_max_sweeps(ctx.h, 40))
    _still_usable()


def test_sweep_cap_exhausted_sync_retries_and_succeeds(ctx):
    dims, tts = _hard_batch()
    ctx.check(lib.ttc_test_set_jacobi_max_sweeps(ctx.h, 2))     # too few; the retry runs 8
    xb = ttcuda.DeviceBatch.from_tts([to_dev(t) for t in tts])
    yb = ttcuda.DeviceBatch(dims, [t.ttv_rks for t in tts])
    before = ctx.stats()["svd_retries"]
    xb.round_det(yb, tol=1e-8)
    assert ctx.stats()["svd_retries"] == before + 1
    for t, got in zip(tts, yb.download()):
        ref = o.tt_rounding(t, tol=1e-8)
        assert got.ttv_rks == ref.ttv_rks
        assert rel(got, ref) < 1e-10
    # the one-shot entry point retries the same way
    got = ttcuda.tt_rounding(to_dev(tts[0]), tol=1e-8)
    assert ctx.stats()["svd_retries"] == before + 2
    assert rel(got, o.tt_rounding(tts[0], tol=1e-8)) < 1e-10


def test_descriptor_outside_allocations_is_refused_before_launch(ctx):
    st = lib.ttc_test_bad_descriptor(ctx.h, 1 << 40)
    assert st == 7                                   # TTC_EINTERNAL
    assert b"outside device allocations" in lib.ttc_last_error(ctx.h)
    _still_usable()


def test_tensor_core_wait_timeout_is_reported_and_context_recovers(ctx):
    """The tcgen05 GEMM's mbarrier wait limit set to zero polls (one try_wait may itself block for a
    while, so a limit of one is not certain to run out): every wait of a GEMM with 128 K-steps
    gives up, the kernel flags the timeout, waits with the full limit for the MMAs it issued,
    frees its tensor memory and returns; the host reports TTC_EINTERNAL.  With the limit restored
    the same GEMM and a BF16-sketch rounding run normally."""
    ms = C.c_double()
    ctx.check(lib.ttc_test_set_tc_wait_limit(ctx.h, 0))
    st = lib.ttc_test_tc_gemm_bench(ctx.h, 256, 512, 8192, 0, 2, C.byref(ms))
    assert st == 7                                   # TTC_EINTERNAL
    assert b"bounded device wait" in lib.ttc_last_error(ctx.h)
    ctx.check(lib.ttc_test_set_tc_wait_limit(ctx.h, 1 << 24))
    ctx.check(lib.ttc_test_tc_gemm_bench(ctx.h, 256, 512, 8192, 0, 2, C.byref(ms)))
    assert ms.value > 0
    x = decaying_tt((2,) * 10, o.r_and_d_to_rks([1] + [12] * 9 + [1], (2,) * 10), seed=8, decay_per=3.0)
    got = ttcuda.ttrand_rounding(to_dev(x), [1] + [20] * 9 + [1], orthogonal=False, seed=3, precision="bf16")
    assert rel(got, x) < 1e-10
