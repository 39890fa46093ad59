"""ttcuda -- B200 (sm_100a) drop-in for the TT rounding path of TensorTrains.jl.

Host-side mirror of the reference's types and methods (rodrigofj99/Tensor-Train-Julia):
``TTvector``/``TToperator`` keep the reference's field names and column-major core
layout (``ttv_vec[k]`` has shape ``(n_k, r_{k-1}, r_k)``); the functions keep the
reference's names, argument meaning and errors.  Every computation runs in
libttcuda.so on the GPU; this module only marshals arrays across the C ABI.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import List, Optional, Sequence
import weakref

import numpy as np

from . import _lib as L
from ._lib import lib

__all__ = [
    "TTvector", "TToperator", "Context", "DeviceBatch", "ArgumentError", "DimensionMismatch", "LAPACKException",
    "CudaError", "r_and_d_to_rks", "default_rank_heuristic", "tt_rounding", "tt_rounding_", "orthogonalize", "norm",
    "tt_recursive_sketch", "ttrand_rounding", "ttrand_rounding_lincomb", "ttrand_rounding_op",
    "ttrand_rounding_residual", "mpo_apply", "dot", "partial_contraction", "dot_operator", "tt_add", "tt_scale",
    "rayleigh_grad", "is_leftorthogonal", "is_rightorthogonal", "version",
]


# ------------------------------------------------------------------------- errors
class ArgumentError(ValueError):
    """Julia ArgumentError (status TTC_EARG)."""


class DimensionMismatch(ValueError):
    """Julia DimensionMismatch / failed @assert on sizes (status TTC_EDIM)."""


class LAPACKException(RuntimeError):
    """Factorisation did not converge (status TTC_ENOCONV); the reference retries gesvd."""


class CudaError(RuntimeError):
    """CUDA runtime failure, allocation failure or internal error."""


_EXC = {1: ArgumentError, 2: DimensionMismatch, 3: LAPACKException, 4: LAPACKException, 5: CudaError,
        6: MemoryError, 7: CudaError, 8: ArgumentError}


# -------------------------------------------------------------------------- types
class TTvector:
    """src/tt_tools.jl:24-34.  ttv_vec[k]: float64 array (n_k, r_{k-1}, r_k), column-major."""

    def __init__(self, N, ttv_vec, ttv_dims, ttv_rks, ttv_ot=None):
        self.N = int(N)
        self.ttv_vec = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in ttv_vec]
        self.ttv_dims = tuple(int(n) for n in ttv_dims)
        self.ttv_rks = [int(r) for r in ttv_rks]
        self.ttv_ot = [int(o) for o in (ttv_ot if ttv_ot is not None else [0] * self.N)]
        if len(self.ttv_vec) != self.N or len(self.ttv_dims) != self.N or len(self.ttv_rks) != self.N + 1:
            raise DimensionMismatch("TTvector: inconsistent N, cores, dims and ranks")
        for k, c in enumerate(self.ttv_vec):
            if c.shape != (self.ttv_dims[k], self.ttv_rks[k], self.ttv_rks[k + 1]):
                raise DimensionMismatch(f"TTvector: core {k + 1} has shape {c.shape}")

    def __getstate__(self):   # copies and pickles leave out the cached ctypes marshalling
        return {k: v for k, v in self.__dict__.items() if k != "_marshal"}

    def copy(self) -> "TTvector":
        return TTvector(self.N, [c.copy(order="F") for c in self.ttv_vec], self.ttv_dims, self.ttv_rks, self.ttv_ot)


class TToperator:
    """src/tt_tools.jl:61-71.  tto_vec[k]: float64 array (n_k, n_k, R_{k-1}, R_k) = [i_out, j_in, a, a']."""

    def __init__(self, N, tto_vec, tto_dims, tto_rks, tto_ot=None):
        self.N = int(N)
        self.tto_vec = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in tto_vec]
        self.tto_dims = tuple(int(n) for n in tto_dims)
        self.tto_rks = [int(r) for r in tto_rks]
        self.tto_ot = [int(o) for o in (tto_ot if tto_ot is not None else [0] * self.N)]
        for k, c in enumerate(self.tto_vec):
            n = self.tto_dims[k]
            if c.shape != (n, n, self.tto_rks[k], self.tto_rks[k + 1]):
                raise DimensionMismatch(f"TToperator: core {k + 1} has shape {c.shape}")

    def __matmul__(self, v: TTvector) -> TTvector:
        return mpo_apply(self, v)

    __mul__ = __matmul__


def is_leftorthogonal(x: TTvector) -> bool:
    """src/tt_tools.jl:364-367"""
    return all(o == 1 for o in x.ttv_ot[: x.N - 1])


def is_rightorthogonal(x: TTvector) -> bool:
    """src/tt_tools.jl:369-372"""
    return all(o == -1 for o in x.ttv_ot[1:])


def r_and_d_to_rks(rks, dims, rmax=1024):
    """src/tt_rounding.jl:6-24 (integer rank clamp; host arithmetic)."""
    rks = list(rks)
    d = len(dims)
    new = [1] * len(rks)
    for i in range(d):
        right = int(np.prod(dims[i:])) if d - i > 0 else 1
        left = int(np.prod(dims[:i])) if i > 0 else 1
        new[i] = min(rks[i], left, right, rmax)
    return new


def default_rank_heuristic(y) -> List[int]:
    """src/tt_randtools.jl:31-50: ranks + ceil(0.5*max(ranks)) on interior bonds
    (elementwise max over a list of TTvectors)."""
    ys = y if isinstance(y, (list, tuple)) else [y]
    rks = list(ys[0].ttv_rks)
    for t in ys[1:]:
        rks = [max(a, b) for a, b in zip(rks, t.ttv_rks)]
    over = int(math.ceil(0.5 * max(rks)))
    for k in range(1, ys[0].N):
        rks[k] += over
    return rks


def version() -> str:
    return lib.ttc_version().decode()


# ------------------------------------------------------------------------ context
class Context:
    """A libttcuda context (device, stream, workspace, plan cache)."""

    def __init__(self, device: int = 0):
        h = L.vp()
        st = lib.ttc_create(C.byref(h), int(device))
        if st != 0:
            raise _EXC.get(st, CudaError)(lib.ttc_last_error(None).decode())
        self.h = h
        self.device = device

    def check(self, st: int):
        if st != 0:
            raise _EXC.get(st, CudaError)(f"{L.STATUS.get(st, st)}: {lib.ttc_last_error(self.h).decode()}")

    def stats(self) -> dict:
        s = L.Stats()
        self.check(lib.ttc_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in L.Stats._fields_}

    def synchronize(self):
        self.check(lib.ttc_synchronize(self.h))

    def set_stream(self, cuda_stream_handle: int):
        """Run subsequent calls on an existing CUDA stream (e.g. torch's cuda_stream handle)."""
        self.check(lib.ttc_set_stream(self.h, C.c_void_p(cuda_stream_handle)))

    def set_profiling(self, on: bool):
        self.check(lib.ttc_set_profiling(self.h, 1 if on else 0))

    def kernel_profile(self) -> dict:
        """Per-kernel-family (device ms, launches, algorithmic FLOPs) of the last call (profiling on)."""
        s = L.Stats()
        self.check(lib.ttc_get_stats(self.h, C.byref(s)))
        return {name: (s.kind_ms[i], int(s.kind_launches[i]), s.kind_flops[i])
                for i, name in enumerate(L.KERNEL_KINDS)}

    def close(self):
        if self.h:
            lib.ttc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_CTX: Optional[Context] = None


def get_context() -> Context:
    global _CTX
    if _CTX is None:
        _CTX = Context(0)
    return _CTX


# -------------------------------------------------------------------- marshalling
class _Keep(list):
    """Keeps the numpy buffers referenced by a ctypes structure alive."""


def _i64(v, keep: _Keep):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int64))
    keep.append(a)
    return a.ctypes.data_as(L.P_i64)


def _ptrs(arrays, keep: _Keep):
    keep.extend(arrays)
    arr = (C.c_void_p * len(arrays))(*[a.__array_interface__["data"][0] for a in arrays])
    keep.append(arr)
    return C.cast(arr, L.PP_f64)


def _f64_fortran(c):
    """c itself when it is already a Fortran-ordered float64 array, else a converted copy."""
    if isinstance(c, np.ndarray) and c.dtype == np.float64 and c.flags.f_contiguous:
        return c
    return np.asfortranarray(c, dtype=np.float64)


def _ttv(x: TTvector, keep: _Keep) -> L.TTV:
    # the marshalled arrays are cached on x while its core arrays (held by the cache, so their
    # ids stay unique) and its dims/ranks/ot are the same; in-place core updates keep them valid.
    # Only views of the user's own arrays are cached: a core that has to be converted (not a
    # Fortran-ordered float64 array, e.g. one assigned to ttv_vec[k] after construction) is a
    # private copy that an in-place edit of the user's array would leave stale, so such a TT is
    # converted afresh on every call.
    key = (tuple(map(id, x.ttv_vec)), tuple(x.ttv_dims), tuple(x.ttv_rks), tuple(x.ttv_ot))
    cached = getattr(x, "_marshal", None)
    if cached is None or cached[0] != key:
        ck = _Keep()
        cores = [_f64_fortran(c) for c in x.ttv_vec]
        args = (_i64(x.ttv_dims, ck), _i64(x.ttv_rks, ck), _i64(x.ttv_ot, ck), _ptrs(cores, ck))
        cached = (key, args, ck, list(x.ttv_vec))
        if all(a is c for a, c in zip(cores, x.ttv_vec)):
            x._marshal = cached
        elif hasattr(x, "_marshal"):
            del x._marshal
    keep.append(cached)
    return L.TTV(x.N, *cached[1])


def _tto(A: TToperator, keep: _Keep) -> L.TTO:
    cores = [_f64_fortran(c) for c in A.tto_vec]
    return L.TTO(A.N, _i64(A.tto_dims, keep), _i64(A.tto_rks, keep), _ptrs(cores, keep))


def host_empty(n: int, dtype=np.float64) -> np.ndarray:
    """A 1-D array of n elements in page-locked host memory mapped into the device address space
    (ttc_host_alloc), freed when the array and its views are gone.  TT cores in such memory are
    uploaded by DMA without the staging copy and written directly by the download kernel."""
    nbytes = max(1, int(n) * np.dtype(dtype).itemsize)
    p = C.c_void_p()
    st = lib.ttc_host_alloc(C.c_size_t(nbytes), C.byref(p))
    if st != 0:
        raise MemoryError(f"ttc_host_alloc({nbytes}): {lib.ttc_last_error(None).decode()}")
    buf = (C.c_char * nbytes).from_address(p.value)
    weakref.finalize(buf, lib.ttc_host_free, C.c_void_p(p.value))
    return np.frombuffer(buf, dtype=dtype, count=int(n))


def pinned_tt(x: "TTvector") -> "TTvector":
    """A copy of x whose cores lie in one page-locked block (host_empty): one DMA per upload."""
    sizes = [int(np.prod(c.shape)) for c in x.ttv_vec]
    flat = host_empty(sum(sizes))
    vec, o = [], 0
    for c, s in zip(x.ttv_vec, sizes):
        v = flat[o:o + s].reshape(c.shape, order="F")
        v[...] = c
        vec.append(v)
        o += s
    return TTvector(x.N, vec, x.ttv_dims, x.ttv_rks, x.ttv_ot)


class _Out:
    """Caller-allocated output buffers at the stated capacities (ttc_ttv_out); `pinned` puts the
    cores in one page-locked block, which the download kernel writes directly."""

    def __init__(self, dims, caps, pinned: bool = False):
        self.N = len(dims)
        self.dims = tuple(int(n) for n in dims)
        self.keep = _Keep()
        self.caps = np.asarray(caps, dtype=np.int64)
        self.rks = np.zeros(self.N + 1, dtype=np.int64)
        self.ot = np.zeros(self.N, dtype=np.int64)
        sizes = [int(self.dims[k] * self.caps[k] * self.caps[k + 1]) for k in range(self.N)]
        if pinned:
            flat = host_empty(sum(sizes))
            offs = np.concatenate([[0], np.cumsum(sizes)])
            self.bufs = [flat[offs[k]:offs[k + 1]] for k in range(self.N)]
        else:
            self.bufs = [np.empty(sizes[k], dtype=np.float64) for k in range(self.N)]
        self.s = L.TTVOut(self.N, self.caps.ctypes.data_as(L.P_i64), self.rks.ctypes.data_as(L.P_i64),
                          self.ot.ctypes.data_as(L.P_i64), _ptrs(self.bufs, self.keep))

    def tt(self) -> TTvector:
        r = [int(v) for v in self.rks]
        vec = [self.bufs[k][: self.dims[k] * r[k] * r[k + 1]].reshape((self.dims[k], r[k], r[k + 1]), order="F")
               for k in range(self.N)]
        return TTvector(self.N, vec, self.dims, r, [int(v) for v in self.ot])


def _sketch_opts(orthogonal, seed, block_rks, precision, sketch_blocks, keep) -> L.SketchOpts:
    prec = {"fp64": 0, "bf16": 1, "tf32": 2, 0: 0, 1: 1, 2: 2}.get(precision)
    if prec is None:
        raise ArgumentError(f"precision must be 'fp64', 'bf16' or 'tf32', not {precision!r}")
    sb = None
    if sketch_blocks is not None:
        sb = _ptrs([np.asfortranarray(b, dtype=np.float64) for b in sketch_blocks], keep)
    return L.SketchOpts(1 if orthogonal else 0, int(seed) & 0xFFFFFFFFFFFFFFFF, int(block_rks or 0), prec, sb)


def _rks_arg(rks, N, dflt):
    if rks is None:
        return list(dflt())
    if isinstance(rks, (int, np.integer)):
        return [1] + [int(rks)] * (N - 1) + [1]
    return [int(r) for r in rks]


def _sketch_ranks(dims, rks, block_rks):
    """Sketch block structure (src/sketches.jl:186-198): returns s = b .* p."""
    N = len(dims)
    b = [1] * (N + 1)
    for k in range(N):
        b[k] = block_rks if block_rks else N
    for k in range(N - 1, -1, -1):
        b[k] = min(b[k], dims[k] * b[k + 1])
    p = [int(math.ceil(r / bb)) for r, bb in zip(rks, b)]
    for i in range(1, N):
        p[i] = max(p[i], p[i - 1])
    p[N] = 1
    return [bb * pp for bb, pp in zip(b, p)]


# ------------------------------------------------------------------------ methods
def tt_rounding(x: TTvector, tol=1e-12, rmax=2 ** 14, direction="left") -> TTvector:
    """src/tt_rounding.jl:146-154"""
    if direction not in ("left", "right"):
        raise ArgumentError("Invalid direction. Use direction=:right or direction=:left")
    ctx = get_context()
    keep = _Keep()
    xs = _ttv(x, keep)
    out = _Out(x.ttv_dims, x.ttv_rks)
    opts = L.RoundOpts(float(tol), int(rmax), 0 if direction == "left" else 1)
    ctx.check(lib.ttc_tt_rounding(ctx.h, C.byref(xs), C.byref(opts), C.byref(out.s)))
    return out.tt()


def tt_rounding_(x: TTvector, tol=1e-12, rmax=2 ** 14, direction="left") -> None:
    """tt_rounding! (src/tt_rounding.jl:158-167): replaces the cores and ranks of x in place."""
    y = tt_rounding(x, tol=tol, rmax=rmax, direction=direction)
    x.ttv_vec, x.ttv_rks, x.ttv_ot = y.ttv_vec, y.ttv_rks, y.ttv_ot


def orthogonalize(x: TTvector, i: int = 1) -> TTvector:
    """src/tt_rounding.jl:65-97 (1-based root i)."""
    ctx = get_context()
    keep = _Keep()
    xs = _ttv(x, keep)
    out = _Out(x.ttv_dims, x.ttv_rks)
    ctx.check(lib.ttc_orthogonalize(ctx.h, C.byref(xs), int(i), C.byref(out.s)))
    return out.tt()


def norm(x: TTvector) -> float:
    """src/tt_rounding.jl:107-114"""
    ctx = get_context()
    keep = _Keep()
    xs = _ttv(x, keep)
    v = C.c_double()
    ctx.check(lib.ttc_norm(ctx.h, C.byref(xs), C.byref(v)))
    return v.value


def tt_recursive_sketch(A: TTvector, rks, H: Optional[TToperator] = None, orthogonal=True, reverse=True, seed=1234,
                        block_rks=None, precision="fp64", sketch_blocks=None):
    """src/sketches.jl:175-305 (TT) and :317-461 (operator), reverse=true only.
    Returns (W, sketch_rks); W[k] is (r_k, s_k) or, with H, (r_k, R_k, s_k)."""
    if not reverse:
        raise ArgumentError("only the reverse sketch (reverse=true) is on the rounding path")
    N = A.N
    if isinstance(rks, (int, np.integer)):
        rks = [int(rks)] * (N + 1)
        rks[N] = 1
    rks = [int(r) for r in rks]
    s = _sketch_ranks(A.ttv_dims, rks, block_rks)
    ctx = get_context()
    keep = _Keep()
    xs = _ttv(A, keep)
    so = _sketch_opts(orthogonal, seed, block_rks, precision, sketch_blocks, keep)
    R = H.tto_rks if H is not None else [1] * (N + 1)
    W = [np.empty(A.ttv_rks[k] * R[k] * s[k], dtype=np.float64) for k in range(N + 1)]
    srk = np.zeros(N + 1, dtype=np.int64)
    if H is None:
        st = lib.ttc_recursive_sketch(ctx.h, C.byref(xs), _i64(rks, keep), C.byref(so), _ptrs(W, keep),
                                      srk.ctypes.data_as(L.P_i64))
    else:
        hs = _tto(H, keep)
        st = lib.ttc_recursive_sketch_op(ctx.h, C.byref(hs), C.byref(xs), _i64(rks, keep), C.byref(so), _ptrs(W, keep),
                                         srk.ctypes.data_as(L.P_i64))
    ctx.check(st)
    if H is None:
        out = [W[k].reshape((A.ttv_rks[k], s[k]), order="F") for k in range(N + 1)]
    else:
        out = [W[k].reshape((A.ttv_rks[k], R[k], s[k]), order="F") for k in range(N + 1)]
    return out, [int(v) for v in srk]


def _rand_out_caps(dims, s):
    N = len(dims)
    r = [1] * (N + 1)
    for k in range(N - 1):
        r[k + 1] = min(dims[k] * r[k], s[k + 1])
    return r


def ttrand_rounding(y: TTvector, rks=None, orthogonal=True, seed=1234, block_rks=None, precision="fp64",
                    sketch_blocks=None) -> TTvector:
    """src/tt_randtools.jl:112-167 (rks vector, int rmax, or the default heuristic)."""
    rks = _rks_arg(rks, y.N, lambda: default_rank_heuristic(y))
    s = _sketch_ranks(y.ttv_dims, rks, block_rks)
    ctx = get_context()
    keep = _Keep()
    xs = _ttv(y, keep)
    so = _sketch_opts(orthogonal, seed, block_rks, precision, sketch_blocks, keep)
    out = _Out(y.ttv_dims, _rand_out_caps(y.ttv_dims, s))
    ctx.check(lib.ttc_ttrand_rounding(ctx.h, C.byref(xs), _i64(rks, keep), C.byref(so), C.byref(out.s)))
    return out.tt()


def ttrand_rounding_lincomb(alpha: Sequence[float], ys: Sequence[TTvector], rks=None, orthogonal=True, seed=1234,
                            block_rks=None, precision="fp64", sketch_blocks=None) -> TTvector:
    """src/tt_randtools.jl:223-283: rounding of sum_j alpha_j ys[j]."""
    if len(alpha) != len(ys):
        raise DimensionMismatch("ttrand_rounding: length(alpha) != length(y)")
    rks = _rks_arg(rks, ys[0].N, lambda: default_rank_heuristic(list(ys)))
    s = _sketch_ranks(ys[0].ttv_dims, rks, block_rks)
    ctx = get_context()
    keep = _Keep()
    arr = (L.TTV * len(ys))(*[_ttv(t, keep) for t in ys])
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    so = _sketch_opts(orthogonal, seed, block_rks, precision, sketch_blocks, keep)
    out = _Out(ys[0].ttv_dims, _rand_out_caps(ys[0].ttv_dims, s))
    ctx.check(lib.ttc_ttrand_rounding_lincomb(ctx.h, len(ys), al.ctypes.data_as(L.P_f64), arr, _i64(rks, keep),
                                              C.byref(so), C.byref(out.s)))
    return out.tt()


def ttrand_rounding_op(alpha: Sequence[float], A: TToperator, ys: Sequence[TTvector], rks=None, orthogonal=True,
                       seed=1234, block_rks=None, precision="fp64", sketch_blocks=None) -> TTvector:
    """src/tt_randtools.jl:285-361: rounding of alpha_1 A ys[0] + sum_{j>0} alpha_j ys[j]."""
    if len(alpha) != len(ys):
        raise DimensionMismatch("ttrand_rounding: length(alpha) != length(y)")
    rks = _rks_arg(rks, ys[0].N, lambda: default_rank_heuristic(list(ys)))
    s = _sketch_ranks(ys[0].ttv_dims, rks, block_rks)
    ctx = get_context()
    keep = _Keep()
    arr = (L.TTV * len(ys))(*[_ttv(t, keep) for t in ys])
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    hs = _tto(A, keep)
    so = _sketch_opts(orthogonal, seed, block_rks, precision, sketch_blocks, keep)
    out = _Out(ys[0].ttv_dims, _rand_out_caps(ys[0].ttv_dims, s))
    ctx.check(lib.ttc_ttrand_rounding_op(ctx.h, len(ys), al.ctypes.data_as(L.P_f64), C.byref(hs), arr,
                                         _i64(rks, keep), C.byref(so), C.byref(out.s)))
    return out.tt()


def ttrand_rounding_residual(A: TToperator, y: TTvector, b: TTvector, rks=None, orthogonal=True, seed=1234,
                             block_rks=None, precision="fp64", sketch_blocks=None) -> TTvector:
    """src/tt_randtools.jl:169-214: rounding of A y - b."""
    rks = _rks_arg(rks, y.N, lambda: default_rank_heuristic(y))
    s = _sketch_ranks(y.ttv_dims, rks, block_rks)
    ctx = get_context()
    keep = _Keep()
    hs = _tto(A, keep)
    xs, bs = _ttv(y, keep), _ttv(b, keep)
    so = _sketch_opts(orthogonal, seed, block_rks, precision, sketch_blocks, keep)
    out = _Out(y.ttv_dims, _rand_out_caps(y.ttv_dims, s))
    ctx.check(lib.ttc_ttrand_rounding_residual(ctx.h, C.byref(hs), C.byref(xs), C.byref(bs), _i64(rks, keep),
                                               C.byref(so), C.byref(out.s)))
    return out.tt()


def ttrand_rounding_hadamard(ys: Sequence[TTvector], rks, orthogonal=True, seed=1234, block_rks=None,
                             sketch_blocks=None) -> TTvector:
    """ttrand_rounding(y::NTuple, rks; ...) (src/tt_randtools.jl:364-473): randomized rounding of
    the Hadamard product ys[0] .* ys[1] .* ... without forming it for the last factor.  rks: a
    vector or an int rmax (the reference's default heuristic has no method for tuples)."""
    N = ys[0].N
    if rks is None:
        raise ArgumentError("ttrand_rounding of a Hadamard product needs rks (a vector or an int rmax)")
    rks = _rks_arg(rks, N, None)
    s = _sketch_ranks(ys[0].ttv_dims, rks, block_rks)
    ctx = get_context()
    keep = _Keep()
    arr = (L.TTV * len(ys))(*[_ttv(t, keep) for t in ys])
    so = _sketch_opts(orthogonal, seed, block_rks, "fp64", sketch_blocks, keep)
    out = _Out(ys[0].ttv_dims, _rand_out_caps(ys[0].ttv_dims, s))
    ctx.check(lib.ttc_ttrand_rounding_hadamard(ctx.h, len(ys), arr, _i64(rks, keep), C.byref(so), C.byref(out.s)))
    return out.tt()


def _fwd_sketch_ranks(dims, rks, block_rks, oversampling=1.5):
    """Sketch ranks b .* p of the forward sketch (src/sketches.jl:243-258) with block-count oversampling."""
    N = len(dims)
    b = [1] + [block_rks if block_rks else N] * N
    for k in range(N):
        b[k + 1] = min(b[k + 1], dims[k] * b[k])
    p = [int(math.ceil(r / bb)) for r, bb in zip(rks, b)]
    for i in range(N - 1, 0, -1):
        p[i] = max(p[i], p[i + 1])
    p[0] = 1
    if oversampling != 1:
        p = [p[0]] + [int(math.ceil(oversampling * v)) for v in p[1:]]
    return [bb * pp for bb, pp in zip(b, p)]


def stta_lincomb(alpha: Sequence[float], ys: Sequence[TTvector], rks=None, seed_left=1234, seed_right=5678,
                 orthogonal=True, block_rks=None) -> TTvector:
    """stta(alpha, y, rks; seed_left, seed_right, orthogonal, block_rks), src/tt_randtools.jl:592-641:
    streaming TT approximation of sum_j alpha_j ys[j] from two-sided sketches."""
    if len(alpha) != len(ys):
        raise DimensionMismatch("stta: length(alpha) != length(y)")
    N = ys[0].N
    rks = _rks_arg(rks, N, lambda: default_rank_heuristic(list(ys)))
    sl = _fwd_sketch_ranks(ys[0].ttv_dims, rks, block_rks)
    sr = _sketch_ranks(ys[0].ttv_dims, rks, block_rks)
    caps = [1] + [min(a, b) for a, b in zip(sl[1:N], sr[1:N])] + [1]
    ctx = get_context()
    keep = _Keep()
    arr = (L.TTV * len(ys))(*[_ttv(t, keep) for t in ys])
    al = np.ascontiguousarray(alpha, dtype=np.float64)
    out = _Out(ys[0].ttv_dims, caps)
    ctx.check(lib.ttc_stta(ctx.h, len(ys), al.ctypes.data_as(L.P_f64), arr, _i64(rks, keep),
                           int(seed_left) & 0xFFFFFFFFFFFFFFFF, int(seed_right) & 0xFFFFFFFFFFFFFFFF,
                           1 if orthogonal else 0, int(block_rks or 0), C.byref(out.s)))
    return out.tt()


def stta(y: TTvector, rks=None, seed_left=1234, seed_right=5678, orthogonal=True, block_rks=None) -> TTvector:
    """stta(y, rks; seed_left, seed_right, orthogonal, block_rks), src/tt_randtools.jl:551-590 (rks
    vector, int rmax, or the default heuristic)."""
    rks = _rks_arg(rks, y.N, lambda: default_rank_heuristic(y))
    return stta_lincomb([1.0], [y], rks, seed_left, seed_right, orthogonal, block_rks)


def mpo_apply(A: TToperator, v: TTvector) -> TTvector:
    """*(A::TToperator, v::TTvector), src/tt_operations.jl:170-194."""
    if tuple(A.tto_dims) != tuple(v.ttv_dims):
        raise DimensionMismatch("Incompatible dimensions")
    ctx = get_context()
    keep = _Keep()
    hs, xs = _tto(A, keep), _ttv(v, keep)
    out = _Out(v.ttv_dims, [a * b for a, b in zip(A.tto_rks, v.ttv_rks)])
    ctx.check(lib.ttc_mpo_apply(ctx.h, C.byref(hs), C.byref(xs), C.byref(out.s)))
    return out.tt()


def dot(A: TTvector, B: TTvector) -> float:
    """src/tt_operations.jl:302-323"""
    if tuple(A.ttv_dims) != tuple(B.ttv_dims):
        raise DimensionMismatch("TT dimensions are not compatible")
    ctx = get_context()
    keep = _Keep()
    a, b = _ttv(A, keep), _ttv(B, keep)
    v = C.c_double()
    ctx.check(lib.ttc_dot(ctx.h, C.byref(a), C.byref(b), C.byref(v)))
    return v.value


def partial_contraction(A: TTvector, B: TTvector, reverse=True) -> List[np.ndarray]:
    """src/sketches.jl:1047-1070"""
    if tuple(A.ttv_dims) != tuple(B.ttv_dims):
        raise DimensionMismatch("TT dimensions are not compatible")
    ctx = get_context()
    keep = _Keep()
    a, b = _ttv(A, keep), _ttv(B, keep)
    W = [np.empty(A.ttv_rks[k] * B.ttv_rks[k], dtype=np.float64) for k in range(A.N + 1)]
    ctx.check(lib.ttc_partial_contraction(ctx.h, C.byref(a), C.byref(b), 1 if reverse else 0, _ptrs(W, keep)))
    return [W[k].reshape((A.ttv_rks[k], B.ttv_rks[k]), order="F") for k in range(A.N + 1)]


def dot_operator(psi: TTvector, H: TToperator, phi: TTvector) -> float:
    """src/tt_operations.jl:390-421: <psi|H|phi>."""
    ctx = get_context()
    keep = _Keep()
    a, h, b = _ttv(psi, keep), _tto(H, keep), _ttv(phi, keep)
    v = C.c_double()
    ctx.check(lib.ttc_dot_operator(ctx.h, C.byref(a), C.byref(h), C.byref(b), C.byref(v)))
    return v.value


def tt_add(x: TTvector, y: TTvector) -> TTvector:
    """+(x::TTvector, y::TTvector), src/tt_operations.jl:81-112."""
    if tuple(x.ttv_dims) != tuple(y.ttv_dims):
        raise DimensionMismatch("Incompatible dimensions")
    ctx = get_context()
    keep = _Keep()
    a, b = _ttv(x, keep), _ttv(y, keep)
    caps = [p + q for p, q in zip(x.ttv_rks, y.ttv_rks)]
    caps[0] = caps[-1] = 1
    out = _Out(x.ttv_dims, caps)
    ctx.check(lib.ttc_tt_add(ctx.h, C.byref(a), C.byref(b), C.byref(out.s)))
    return out.tt()


def tt_scale(a: float, x: TTvector) -> TTvector:
    """*(a::Number, A::TTvector), src/tt_operations.jl:428-441."""
    ctx = get_context()
    keep = _Keep()
    xs = _ttv(x, keep)
    out = _Out(x.ttv_dims, x.ttv_rks)
    ctx.check(lib.ttc_tt_scale(ctx.h, float(a), C.byref(xs), C.byref(out.s)))
    return out.tt()


def rayleigh_grad(H: TToperator, x: TTvector, ckpt_every: int = 4, precision: str = "fp64"):
    """Value and gradient of <x|H|x>/<x|x> with respect to every core of x (H symmetric), with
    the contractions in FP64 or in FP32 with FP32 accumulation (precision="fp32")."""
    prec = {"fp64": 0, "fp32": 3}.get(precision)
    if prec is None:
        raise ArgumentError(f"precision must be 'fp64' or 'fp32', not {precision!r}")
    ctx = get_context()
    keep = _Keep()
    hs, xs = _tto(H, keep), _ttv(x, keep)
    G = [np.empty(c.size, dtype=np.float64) for c in x.ttv_vec]
    v = C.c_double()
    ctx.check(lib.ttc_rayleigh_grad_prec(ctx.h, C.byref(hs), C.byref(xs), int(ckpt_every), prec, C.byref(v),
                                         _ptrs(G, keep)))
    return v.value, [G[k].reshape(x.ttv_vec[k].shape, order="F") for k in range(x.N)]


# -------------------------------------------------------------------- device batches
class DeviceBatch:
    """A batch of TTvectors resident in HBM (same N and dims; per-TT rank capacities).
    Replaces the Vector{TTvector} a Krylov caller rounds term by term."""

    def __init__(self, dims, caps: Sequence[Sequence[int]], ctx: Optional[Context] = None):
        self.ctx = ctx or get_context()
        self.dims = tuple(int(n) for n in dims)
        self.N = len(self.dims)
        self.count = len(caps)
        self.caps = [list(c) for c in caps]
        keep = _Keep()
        h = L.vp()
        cap_flat = [int(v) for c in caps for v in c]
        self.ctx.check(lib.ttc_batch_create(self.ctx.h, self.count, self.N, _i64(self.dims, keep), _i64(cap_flat, keep),
                                            C.byref(h)))
        self.h = h

    @classmethod
    def from_tts(cls, tts: Sequence[TTvector], caps=None, ctx=None) -> "DeviceBatch":
        caps = caps or [t.ttv_rks for t in tts]
        b = cls(tts[0].ttv_dims, caps, ctx)
        b.upload(tts)
        return b

    def upload(self, tts: Sequence[TTvector]):
        keep = _Keep()
        arr = (L.TTV * len(tts))(*[_ttv(t, keep) for t in tts])
        self.ctx.check(lib.ttc_batch_upload_all(self.h, arr))

    def ranks(self, i: int) -> List[int]:
        r = np.zeros(self.N + 1, dtype=np.int64)
        self.ctx.check(lib.ttc_batch_ranks(self.h, int(i), r.ctypes.data_as(L.P_i64)))
        return [int(v) for v in r]

    def download(self, reuse: bool = False) -> List[TTvector]:
        """The batch's TTs as host TTvectors.  With reuse=True the host buffers of the previous
        reusing download are written again (no allocation; the TTvectors it returned then see
        the new values), as a loop that rounds and downloads the same basis repeatedly wants;
        those buffers are page-locked, so the download kernel writes them directly."""
        if reuse:
            outs = getattr(self, "_outs", None)
            if outs is None:
                outs = self._outs = [_Out(self.dims, c, pinned=True) for c in self.caps]
        else:
            outs = [_Out(self.dims, c) for c in self.caps]
        arr = (L.TTVOut * len(outs))(*[o.s for o in outs])
        self.ctx.check(lib.ttc_batch_download_all(self.h, arr))
        # the library wrote ranks, ot and cores through the pointers each _Out holds
        return [o.tt() for o in outs]

    def nbytes(self) -> int:
        return int(lib.ttc_batch_bytes(self.h))

    def round_det(self, out: "DeviceBatch", tol=1e-12, rmax=2 ** 14, sync=True):
        opts = L.RoundOpts(float(tol), int(rmax), 0)
        f = lib.ttc_batch_round_det if sync else lib.ttc_batch_round_det_async
        self.ctx.check(f(self.ctx.h, self.h, C.byref(opts), out.h))

    def round_rand(self, out: "DeviceBatch", rks, orthogonal=True, seed=1234, block_rks=None, precision="fp64",
                   after_tol: Optional[float] = None, rmax=2 ** 14, sync=True, sketch_blocks=None):
        keep = _Keep()
        so = _sketch_opts(orthogonal, seed, block_rks, precision, sketch_blocks, keep)
        after = L.RoundOpts(float(after_tol), int(rmax), 0) if after_tol is not None else None
        f = lib.ttc_batch_round_rand if sync else lib.ttc_batch_round_rand_async
        self.ctx.check(f(self.ctx.h, self.h, _i64(rks, keep), C.byref(so), C.byref(after) if after else None, out.h))

    def close(self):
        if getattr(self, "h", None):
            lib.ttc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from .json_io import json_to_mpo, json_to_mps, load_json, mpo_to_json, mps_to_json, save_json  # noqa: E402,F401
