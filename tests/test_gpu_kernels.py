"""Kernel-level GPU tests: grouped FP64 GEMM (split strides), Householder QR, one-sided
Jacobi SVD and the tcgen05 BF16 GEMM, each against numpy on the same inputs."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ttcuda = pytest.importorskip("ttcuda")
lib = ttcuda.lib

P = C.POINTER(C.c_double)
PL = C.POINTER(C.c_longlong)
PI = C.POINTER(C.c_int)
lib.ttc_test_gemm.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                              P, C.c_longlong, PL, P, C.c_longlong, PL, P, C.c_longlong, PL, C.c_double, C.c_double]
lib.ttc_test_qr.argtypes = [C.c_void_p, C.c_int, C.c_int, P, P, P]
lib.ttc_test_jacobi.argtypes = [C.c_void_p, C.c_int, C.c_int, P, C.c_int, P, P, PI, PI]
lib.ttc_test_bf16_gemm.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, P, P, P, C.c_double]
lib.ttc_test_tf32_gemm.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, P, P, P, C.c_double]


def ptr(a):
    return a.ctypes.data_as(P)


def lptr(v):
    a = np.asarray(v, dtype=np.int64)
    return a, a.ctypes.data_as(PL)


@pytest.fixture(scope="module")
def ctx():
    return ttcuda.get_context()


def gemm(ctx, m, n, k, batch, m0, n0, k0e, A, ast, B, bst, Cm, cst, alpha=1.0, beta=0.0):
    a_s, ap = lptr(ast)
    b_s, bp = lptr(bst)
    c_s, cp = lptr(cst)
    ctx.check(lib.ttc_test_gemm(ctx.h, m, n, k, batch, m0, n0, k0e, ptr(A), A.size, ap, ptr(B), B.size, bp,
                                ptr(Cm), Cm.size, cp, alpha, beta))


def ref_gemm(m, n, k, batch, m0, n0, k0e, A, ast, B, bst, Cm, cst, alpha, beta):
    out = Cm.copy()
    for b in range(batch):
        for i in range(m):
            ia = (i % m0) * ast[0] + (i // m0) * ast[1] + b * ast[4]
            ic = (i % m0) * cst[0] + (i // m0) * cst[1] + b * cst[4]
            for j in range(n):
                jb = (j % n0) * bst[2] + (j // n0) * bst[3] + b * bst[4]
                jc = (j % n0) * cst[2] + (j // n0) * cst[3]
                s = 0.0
                for kk in range(k):
                    s += A[ia + (kk % k0e) * ast[2] + (kk // k0e) * ast[3]] * B[jb + (kk % k0e) * bst[0] + (kk // k0e) * bst[1]]
                out[ic + jc] = alpha * s + (beta * Cm[ic + jc] if beta != 0 else 0.0)
    return out


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (5, 3, 7), (64, 64, 16), (70, 65, 33), (130, 3, 200)])
def test_gemm_plain(ctx, m, n, k):
    g = np.random.default_rng(m * 1000 + n * 10 + k)
    A = g.standard_normal((m, k))
    B = g.standard_normal((k, n))
    Cm = g.standard_normal((m, n))
    Af, Bf, Cf = A.ravel(order="F").copy(), B.ravel(order="F").copy(), Cm.ravel(order="F").copy()
    gemm(ctx, m, n, k, 1, m, n, k, Af, [1, 0, m, 0, 0], Bf, [1, 0, k, 0, 0], Cf, [1, 0, m, 0, 0], 0.5, 2.0)
    assert np.allclose(Cf.reshape((m, n), order="F"), 0.5 * A @ B + 2.0 * Cm, rtol=1e-13, atol=1e-12)


def test_gemm_transposed_and_split(ctx):
    g = np.random.default_rng(3)
    # A^T (A stored k x m), B row-major, C written transposed; rows split m0, K split k0e, batch 3
    m, n, k, batch, m0, n0, k0e = 12, 9, 10, 3, 4, 3, 5
    A = g.standard_normal(4000)
    B = g.standard_normal(4000)
    Cm = g.standard_normal(4000)
    ast = [7, 29, 1, 3, 600]
    bst = [2, 11, 37, 5, 700]
    cst = [13, 1, 53, 3, 800]
    ref = ref_gemm(m, n, k, batch, m0, n0, k0e, A, ast, B, bst, Cm, cst, 1.25, 0.0)
    got = Cm.copy()
    gemm(ctx, m, n, k, batch, m0, n0, k0e, A, ast, B, bst, got, cst, 1.25, 0.0)
    assert np.allclose(got, ref, rtol=1e-13, atol=1e-12)


lib.ttc_test_gemm_runs.argtypes = lib.ttc_test_gemm.argtypes + [C.c_int, PI]


def ref_gemm_vec(m, n, k, batch, m0, n0, k0e, A, ast, B, bst, Cm, cst, alpha, beta):
    """ref_gemm with numpy index arrays (for long K)."""
    out = Cm.copy()
    i, j, kk = np.arange(m), np.arange(n), np.arange(k)
    ko_a = (kk % k0e) * ast[2] + (kk // k0e) * ast[3]
    ko_b = (kk % k0e) * bst[0] + (kk // k0e) * bst[1]
    for b in range(batch):
        Am = A[((i % m0) * ast[0] + (i // m0) * ast[1] + b * ast[4])[:, None] + ko_a[None, :]]
        Bm = B[ko_b[:, None] + ((j % n0) * bst[2] + (j // n0) * bst[3] + b * bst[4])[None, :]]
        ic = ((i % m0) * cst[0] + (i // m0) * cst[1] + b * cst[4])[:, None] + ((j % n0) * cst[2] + (j // n0) * cst[3])[None, :]
        out[ic] = alpha * (Am @ Bm) + (beta * Cm[ic] if beta != 0 else 0.0)
    return out


@pytest.mark.parametrize("m,n,k,beta", [(70, 65, 3000, 0.0), (130, 3, 4100, 0.0), (64, 64, 1024, 0.0),
                                        (70, 65, 3000, 2.0), (200, 150, 700, 0.0)])
def test_gemm_split_k(ctx, m, n, k, beta):
    """Few output tiles and long K: the planner splits K over several CTAs per tile, the last of
    which adds the partial tiles in split order; three runs of one plan (beta == 0) check that
    the tile counters are left zero for the next launch."""
    g = np.random.default_rng(m + n + k)
    A = g.standard_normal((m, k))
    B = g.standard_normal((k, n))
    Cm = g.standard_normal((m, n))
    Af, Bf, Cf = A.ravel(order="F").copy(), B.ravel(order="F").copy(), Cm.ravel(order="F").copy()
    a_s, ap = lptr([1, 0, m, 0, 0])
    b_s, bp = lptr([1, 0, k, 0, 0])
    c_s, cp = lptr([1, 0, m, 0, 0])
    ks = C.c_int(0)
    runs = 3 if beta == 0.0 else 1
    ctx.check(lib.ttc_test_gemm_runs(ctx.h, m, n, k, 1, m, n, k, ptr(Af), Af.size, ap, ptr(Bf), Bf.size, bp, ptr(Cf),
                                     Cf.size, cp, 0.5, beta, runs, C.byref(ks)))
    want = 0.5 * A @ B + beta * Cm
    assert ks.value > 1 or (m, n, k) == (200, 150, 700)
    assert np.abs(Cf.reshape((m, n), order="F") - want).max() <= 1e-12 * np.abs(want).max()


def test_gemm_split_k_mixed_radix_batched(ctx):
    """Split K over a K index of two strides (k0e = 7) with split rows and columns and a batch."""
    g = np.random.default_rng(8)
    m, n, k, batch, m0, n0, k0e = 12, 9, 2100, 3, 4, 3, 7
    ast = [7, 29, 1, 97, 70000]
    bst = [2, 31, 5000, 5, 80000]
    cst = [13, 1, 53, 3, 800]
    A = g.standard_normal(300000)
    B = g.standard_normal(300000)
    Cm = g.standard_normal(4000)
    ref = ref_gemm_vec(m, n, k, batch, m0, n0, k0e, A, ast, B, bst, Cm, cst, 1.25, 0.0)
    got = Cm.copy()
    a_s, ap = lptr(ast)
    b_s, bp = lptr(bst)
    c_s, cp = lptr(cst)
    ks = C.c_int(0)
    ctx.check(lib.ttc_test_gemm_runs(ctx.h, m, n, k, batch, m0, n0, k0e, ptr(A), A.size, ap, ptr(B), B.size, bp,
                                     ptr(got), got.size, cp, 1.25, 0.0, 2, C.byref(ks)))
    assert ks.value > 1
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-11)


@pytest.mark.parametrize("m,n", [(1, 1), (7, 3), (3, 7), (64, 64), (100, 37), (512, 256), (300, 300), (768, 384),
                                 (700, 690), (1044, 522)])
def test_householder_qr(ctx, m, n):
    g = np.random.default_rng(m + n)
    A = g.standard_normal((m, n))
    if n > 4:
        A[:, 2] = 0.0                 # exact zero column
        A[:, 3] = A[:, 1] * 3.0       # exact dependency
    K = min(m, n)
    Q = np.zeros(m * K)
    R = np.zeros(K * n)
    Af = A.ravel(order="F").copy()
    ctx.check(lib.ttc_test_qr(ctx.h, m, n, ptr(Af), ptr(Q), ptr(R)))
    Q = Q.reshape((m, K), order="F")
    R = R.reshape((K, n), order="F")
    assert np.allclose(Q.T @ Q, np.eye(K), atol=1e-13 * max(1, m))
    assert np.allclose(Q @ R, A, atol=1e-13 * max(1, m) * np.abs(A).max())
    assert np.allclose(np.tril(R, -1), 0.0)


@pytest.mark.parametrize("m,n,accw", [(1, 1, 0), (6, 6, 0), (17, 17, 0), (32, 9, 0), (32, 32, 0), (40, 40, 0),
                                      (64, 64, 0), (96, 80, 0),
                                      (256, 256, 0), (384, 384, 0), (512, 512, 0), (10, 4, 1), (64, 64, 1)])
def test_jacobi(ctx, m, n, accw):
    g = np.random.default_rng(m * 7 + n)
    U, _ = np.linalg.qr(g.standard_normal((m, n)))
    V, _ = np.linalg.qr(g.standard_normal((n, n)))
    s = 10.0 ** (-np.arange(n) / max(1, n / 12))
    X = (U * s) @ V.T
    if m >= 128:
        # the sweep drivers hand the kernel the QR-LQ preconditioned factor R2^T
        # (X = Q1 R1, R1^T = Q2 R2), which has the singular values of X
        R1 = np.linalg.qr(X, mode="r")
        X = np.linalg.qr(R1.T, mode="r").T
    Xf = X.ravel(order="F").copy()
    W = np.zeros(n * n)
    sig = np.zeros(n)
    perm = np.zeros(n, dtype=np.int32)
    sweeps = np.zeros(1, dtype=np.int32)
    ctx.check(lib.ttc_test_jacobi(ctx.h, m, n, ptr(Xf), accw, ptr(W), ptr(sig), perm.ctypes.data_as(PI),
                                  sweeps.ctypes.data_as(PI)))
    Bm = Xf.reshape((m, n), order="F")
    G = Bm.T @ Bm
    nrm = np.sqrt(np.diag(G))
    rel_off = np.abs(G - np.diag(np.diag(G))) / np.outer(nrm, nrm)
    assert sweeps[0] > 0, f"no convergence after {-sweeps[0]} sweeps; max relative off-diagonal {rel_off.max():.3e}"
    ss = sig[perm]
    assert np.all(np.diff(ss) <= 0)
    assert np.allclose(ss, s, rtol=1e-10, atol=1e-14)
    off = G - np.diag(np.diag(G))
    assert np.abs(off).max() <= 2 * max(m, 16) * 2.3e-16    # the kernel's rotation threshold
    if accw:
        Wm = W.reshape((n, n), order="F")
        assert np.allclose(Wm.T @ Wm, np.eye(n), atol=1e-13)
        assert np.allclose(X @ Wm, Bm, atol=1e-13)


def bf16_round(x):
    """Round FP64 values directly to BF16 (8 significant bits, round half to even), as the
    device's FP64 -> BF16 conversion does (normal range only)."""
    m, e = np.frexp(np.asarray(x, dtype=np.float64))
    return np.ldexp(np.round(m * 256.0) / 256.0, e)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 128, 64), (200, 130, 100), (513, 257, 264), (40, 300, 8),
                                   (2048, 2400, 200)])
def test_bf16_tcgen05_gemm(ctx, m, n, k):
    g = np.random.default_rng(m + 3 * n + 7 * k)
    A = g.standard_normal((m, k))
    B = g.standard_normal((n, k))
    Cm = np.zeros(m * n)
    ctx.check(lib.ttc_test_bf16_gemm(ctx.h, m, n, k, ptr(np.ascontiguousarray(A)), ptr(np.ascontiguousarray(B)),
                                     ptr(Cm), 1.0))
    ref = bf16_round(A) @ bf16_round(B).T
    got = Cm.reshape((m, n), order="F")
    # exact BF16 products, FP32 accumulation: error ~ sqrt(k) * 2^-24 * sum|a||b|
    bound = 4 * np.sqrt(k) * 2.0 ** -24 * (np.abs(bf16_round(A)) @ np.abs(bf16_round(B)).T)
    ratio = np.abs(got - ref) / (bound + 1e-30)
    worst = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, f"worst element {worst}: got {got[worst]}, ref {ref[worst]}, bound {bound[worst]}"
    assert np.linalg.norm(got - ref) <= 1e-6 * np.linalg.norm(ref)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 128, 32), (200, 130, 100), (513, 257, 266), (40, 300, 4),
                                   (2048, 2400, 200)])
def test_tf32_tcgen05_gemm(ctx, m, n, k):
    """kind::tf32: FP32 operands read with a 10-bit mantissa (each operand's relative error
    below 2^-10, so a product's below 2^-9), FP32 accumulation."""
    g = np.random.default_rng(m + 5 * n + 11 * k)
    A = g.standard_normal((m, k))
    B = g.standard_normal((n, k))
    Cm = np.zeros(m * n)
    ctx.check(lib.ttc_test_tf32_gemm(ctx.h, m, n, k, ptr(np.ascontiguousarray(A)), ptr(np.ascontiguousarray(B)),
                                     ptr(Cm), 1.0))
    ref = A @ B.T
    got = Cm.reshape((m, n), order="F")
    mag = np.abs(A) @ np.abs(B).T
    bound = (2.0 ** -9 + 4 * np.sqrt(k) * 2.0 ** -24) * mag
    ratio = np.abs(got - ref) / (bound + 1e-30)
    worst = np.unravel_index(np.argmax(ratio), ratio.shape)
    assert ratio.max() <= 1.0, f"worst element {worst}: got {got[worst]}, ref {ref[worst]}, bound {bound[worst]}"
    assert np.linalg.norm(got - ref) <= 2e-3 * np.linalg.norm(ref)


@pytest.mark.parametrize("n,rank", [(24, 16), (96, 64), (300, 200)])
def test_jacobi_rank_deficient(ctx, n, rank):
    """Rank-deficient square factors (n - rank numerically zero columns after mixing) converge, the
    zero singular values come out at the rounding level and the others match: sizes <= 32 run one
    problem per warp, larger ones the Gram-block cluster kernel."""
    g = np.random.default_rng(5 + n)
    m = n
    U, _ = np.linalg.qr(g.standard_normal((m, n)))
    V, _ = np.linalg.qr(g.standard_normal((n, n)))
    s = np.concatenate([10.0 ** (-np.arange(rank) / max(4.0, rank / 6)), np.zeros(n - rank)])
    X = (U * s) @ V.T
    Xf = X.ravel(order="F").copy()
    W = np.zeros(n * n)
    sig = np.zeros(n)
    perm = np.zeros(n, dtype=np.int32)
    sweeps = np.zeros(1, dtype=np.int32)
    ctx.check(lib.ttc_test_jacobi(ctx.h, m, n, ptr(Xf), 0, ptr(W), ptr(sig), perm.ctypes.data_as(PI),
                                  sweeps.ctypes.data_as(PI)))
    assert sweeps[0] > 0
    ss = sig[perm]
    assert sorted(perm.tolist()) == list(range(n))
    assert np.allclose(ss[:rank], s[:rank], rtol=1e-10, atol=1e-14)
    assert np.all(ss[rank:] <= 1e-13 * max(1, n / 32))
