"""GPU test of ttc_qr_noalloc, the allocation-free QR entry point.

ttc_qr_noalloc is for callers that cannot allocate device memory when they need a
factorisation (code running inside a memory pool or arena that owns the device budget):
it keeps its scratch in a fixed device array inside the library.  This file checks it
through the C ABI against the library's existing QR path (ttc_orthogonalize of the two-site
TT whose first core is A and whose second core is the identity: the orthogonalised first
core is Q and the second core becomes R), on two calls in a row so that a second call
cannot pass on the first call's leftovers, and checks that a matrix beyond the fixed
scratch is refused.  Test buffers are allocated by torch; the entry point itself allocates
nothing.  The file name makes pytest collect it after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ttcuda = pytest.importorskip("ttcuda")
torch = pytest.importorskip("torch")
from ttcuda._lib import lib  # noqa: E402

lib.ttc_qr_noalloc.restype = C.c_int32
lib.ttc_qr_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                               C.c_int64, C.c_void_p, C.c_void_p]
lib.ttc_last_error.restype = C.c_char_p


def _reference_qr(A):
    """Q, R from the existing entry point: orthogonalize the TT (A, I) onto its second site."""
    m, n = A.shape
    core1 = np.asfortranarray(A.reshape(m, 1, n))
    core2 = np.asfortranarray(np.eye(n).reshape(n, n, 1))
    x = ttcuda.TTvector(2, [core1, core2], (m, n), [1, n, 1], [0, 0])
    y = ttcuda.orthogonalize(x, 2)
    K = y.ttv_rks[1]
    Q = np.asarray(y.ttv_vec[0]).reshape(m, K)
    R = np.asarray(y.ttv_vec[1])[:, :, 0].T.copy()     # core2'[i2, b] = R[b, i2]
    return Q, R


def _noalloc_qr(A, lda=None, want_q=True, want_r=True, want_status=True):
    """Calls the entry point on device copies of A (leading dimension lda >= m, padding rows
    filled with NaN so that a read beyond row m would show) and returns Q, R (None when not
    requested), the status word (None without one) and A's device copy after the call."""
    m, n = A.shape
    K = min(m, n)
    lda = lda or m
    dev = torch.device("cuda:0")
    Ap = np.full((lda, n), np.nan)
    Ap[:m] = A
    Ad = torch.from_numpy(Ap.ravel(order="F").copy()).to(dev)
    Qd = torch.full((m * K,), np.nan, dtype=torch.float64, device=dev) if want_q else None
    Rd = torch.full((K * n,), np.nan, dtype=torch.float64, device=dev) if want_r else None
    st = torch.full((1,), -1, dtype=torch.int32, device=dev) if want_status else None
    torch.cuda.synchronize()
    rc = lib.ttc_qr_noalloc(m, n, Ad.data_ptr(), lda, Qd.data_ptr() if want_q else None, m,
                            Rd.data_ptr() if want_r else None, K, st.data_ptr() if want_status else None, None)
    assert rc == 0, lib.ttc_last_error(None).decode()
    torch.cuda.synchronize()
    Q = Qd.cpu().numpy().reshape((m, K), order="F") if want_q else None
    R = Rd.cpu().numpy().reshape((K, n), order="F") if want_r else None
    status = int(st.cpu().item()) if want_status else None
    return Q, R, status, Ad.cpu().numpy().reshape((lda, n), order="F")[:m]


def test_qr_noalloc_matches_existing_qr_two_calls():
    ttcuda.get_context()
    g = np.random.default_rng(123)
    for (m, n) in [(300, 120), (512, 256)]:         # two calls in a row on the shared scratch
        A = g.standard_normal((m, n)) * np.logspace(0, -6, n)
        Q, R, status, A_after = _noalloc_qr(A)
        Qr, Rr = _reference_qr(A)
        assert status == 0
        assert np.array_equal(A_after, A)                                 # input untouched
        assert np.allclose(np.tril(R, -1), 0.0)
        # same Householder kernel and sign convention as the existing path: FP64 agreement
        assert np.abs(Q - Qr).max() <= 1e-12
        assert np.abs(R - Rr).max() <= 1e-12 * np.abs(Rr).max()
        assert np.abs(Q.T @ Q - np.eye(Q.shape[1])).max() <= 1e-13 * m
        assert np.linalg.norm(Q @ R - A) <= 1e-13 * np.linalg.norm(A)


def test_qr_noalloc_rejects_matrix_beyond_scratch():
    m, n = 1536, 400                                  # m*n > 524288
    rc = lib.ttc_qr_noalloc(m, n, C.c_void_p(8), m, None, m, None, n, None, None)
    assert rc == 2                                    # TTC_EDIM, nothing launched
    assert b"exceeds the fixed scratch" in lib.ttc_last_error(None)


def _check_against_reference(A, Q, R):
    Qr, Rr = _reference_qr(A)
    if Q is not None:
        assert np.abs(Q - Qr).max() <= 1e-12
    if R is not None:
        assert np.allclose(np.tril(R, -1), 0.0)
        assert np.abs(R - Rr).max() <= 1e-12 * np.abs(Rr).max()


def test_qr_noalloc_optional_outputs_padded_lda_and_wide_matrix():
    """Q = NULL, R = NULL, status = NULL (the flags then go to the scratch's own slot), a leading
    dimension larger than m, and a wide matrix (m < n), each against the existing QR path."""
    ttcuda.get_context()
    g = np.random.default_rng(7)
    A = g.standard_normal((200, 90))
    _, R, status, _ = _noalloc_qr(A, want_q=False)
    assert status == 0
    _check_against_reference(A, None, R)
    Q, _, status, _ = _noalloc_qr(A, want_r=False)
    assert status == 0
    _check_against_reference(A, Q, None)
    Q, R, status, _ = _noalloc_qr(A, want_status=False)
    assert status is None
    _check_against_reference(A, Q, R)
    Q, R, status, A_after = _noalloc_qr(A, lda=256)
    assert status == 0 and np.array_equal(A_after, A)
    _check_against_reference(A, Q, R)
    W = g.standard_normal((64, 300))                  # wide: K = m, R is 64 x 300
    Q, R, status, _ = _noalloc_qr(W)
    assert status == 0
    _check_against_reference(W, Q, R)
    assert np.linalg.norm(Q @ R - W) <= 1e-13 * np.linalg.norm(W)


def test_qr_noalloc_flags_non_finite_input():
    """A NaN in A sets flag 2 in the caller's status word; the next call starts from zero."""
    ttcuda.get_context()
    A = np.random.default_rng(8).standard_normal((128, 32))
    A[5, 3] = np.nan
    _, _, status, _ = _noalloc_qr(A)
    assert status & 2
    _, _, status, _ = _noalloc_qr(np.random.default_rng(9).standard_normal((128, 32)))
    assert status == 0


def test_qr_noalloc_rejects_leading_dimension_beyond_int32():
    """Leading dimensions are stored as 32-bit integers in the kernel descriptor: larger ones are
    refused before anything runs (no pointer is dereferenced on that path)."""
    big = 2 ** 31
    rc = lib.ttc_qr_noalloc(64, 32, C.c_void_p(8), 64, C.c_void_p(8), big, None, 32, None, None)
    assert rc == 1                                    # TTC_EARG
    assert b"2^31" in lib.ttc_last_error(None)
    rc = lib.ttc_qr_noalloc(64, 32, C.c_void_p(8), 64, None, 64, C.c_void_p(8), big, None, None)
    assert rc == 1
    rc = lib.ttc_qr_noalloc(64, 32, C.c_void_p(8), big, None, 64, None, 32, None, None)
    assert rc == 1
