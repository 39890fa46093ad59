"""ctypes binding of libttcuda.so (the C ABI declared in include/ttcuda.h).

The library is loaded from this directory.  There is no fallback: if the shared
library is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libttcuda.so")

i32, i64, u64, f64, vp, sz = C.c_int32, C.c_int64, C.c_uint64, C.c_double, C.c_void_p, C.c_size_t
P_i64 = C.POINTER(i64)
P_f64 = C.POINTER(f64)
PP_f64 = C.POINTER(P_f64)


class TTV(C.Structure):
    _fields_ = [("N", i32), ("dims", P_i64), ("rks", P_i64), ("ot", P_i64), ("cores", PP_f64)]


class TTVOut(C.Structure):
    _fields_ = [("N", i32), ("rks_cap", P_i64), ("rks", P_i64), ("ot", P_i64), ("cores", PP_f64)]


class TTO(C.Structure):
    _fields_ = [("N", i32), ("dims", P_i64), ("rks", P_i64), ("cores", PP_f64)]


class RoundOpts(C.Structure):
    _fields_ = [("tol", f64), ("rmax", i64), ("direction", i32)]


class SketchOpts(C.Structure):
    _fields_ = [("orthogonal", i32), ("seed", u64), ("block_rks", i64), ("precision", i32), ("sketch_blocks", PP_f64)]


class Stats(C.Structure):
    _fields_ = [("total_ms", f64), ("sketch_ms", f64), ("orth_ms", f64), ("svd_ms", f64), ("h2d_ms", f64),
                ("d2h_ms", f64), ("kernel_launches", i64), ("kind_ms", f64 * 8), ("kind_launches", i64 * 8),
                ("kind_flops", f64 * 8), ("jacobi_problems", i64), ("jacobi_sweeps_sum", i64),
                ("jacobi_sweeps_max", i64), ("plans_built", i64), ("svd_retries", i64)]


KERNEL_KINDS = ["gemm_f64", "householder_qr", "jacobi_svd", "gemm_bf16_tcgen05", "mpo_apply", "other"]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libttcuda.so not built ({LIB_PATH}); run tensor-train-julia_b200/build.py")
    return C.CDLL(LIB_PATH)


lib = _load()

_SIGS = {
    "ttc_version": (C.c_char_p, []),
    "ttc_create": (i32, [C.POINTER(vp), C.c_int]),
    "ttc_destroy": (i32, [vp]),
    "ttc_set_stream": (i32, [vp, vp]),
    "ttc_last_error": (C.c_char_p, [vp]),
    "ttc_get_stats": (i32, [vp, C.POINTER(Stats)]),
    "ttc_set_profiling": (i32, [vp, C.c_int]),
    "ttc_synchronize": (i32, [vp]),
    "ttc_batch_create": (i32, [vp, i32, i32, P_i64, P_i64, C.POINTER(vp)]),
    "ttc_batch_destroy": (i32, [vp]),
    "ttc_batch_upload": (i32, [vp, i32, C.POINTER(TTV)]),
    "ttc_batch_download": (i32, [vp, i32, C.POINTER(TTVOut)]),
    "ttc_batch_upload_all": (i32, [vp, C.POINTER(TTV)]),
    "ttc_batch_download_all": (i32, [vp, C.POINTER(TTVOut)]),
    "ttc_batch_ranks": (i32, [vp, i32, P_i64]),
    "ttc_batch_bytes": (sz, [vp]),
    "ttc_batch_round_det": (i32, [vp, vp, C.POINTER(RoundOpts), vp]),
    "ttc_batch_round_det_async": (i32, [vp, vp, C.POINTER(RoundOpts), vp]),
    "ttc_batch_round_rand": (i32, [vp, vp, P_i64, C.POINTER(SketchOpts), C.POINTER(RoundOpts), vp]),
    "ttc_batch_round_rand_async": (i32, [vp, vp, P_i64, C.POINTER(SketchOpts), C.POINTER(RoundOpts), vp]),
    "ttc_tt_rounding": (i32, [vp, C.POINTER(TTV), C.POINTER(RoundOpts), C.POINTER(TTVOut)]),
    "ttc_orthogonalize": (i32, [vp, C.POINTER(TTV), i32, C.POINTER(TTVOut)]),
    "ttc_norm": (i32, [vp, C.POINTER(TTV), P_f64]),
    "ttc_recursive_sketch": (i32, [vp, C.POINTER(TTV), P_i64, C.POINTER(SketchOpts), PP_f64, P_i64]),
    "ttc_recursive_sketch_op": (i32, [vp, C.POINTER(TTO), C.POINTER(TTV), P_i64, C.POINTER(SketchOpts), PP_f64, P_i64]),
    "ttc_ttrand_rounding": (i32, [vp, C.POINTER(TTV), P_i64, C.POINTER(SketchOpts), C.POINTER(TTVOut)]),
    "ttc_ttrand_rounding_lincomb": (i32, [vp, i32, P_f64, C.POINTER(TTV), P_i64, C.POINTER(SketchOpts), C.POINTER(TTVOut)]),
    "ttc_ttrand_rounding_hadamard": (i32, [vp, i32, C.POINTER(TTV), P_i64, C.POINTER(SketchOpts), C.POINTER(TTVOut)]),
    "ttc_stta": (i32, [vp, i32, P_f64, C.POINTER(TTV), P_i64, C.c_uint64, C.c_uint64, i32, C.c_int64,
                       C.POINTER(TTVOut)]),
    "ttc_ttrand_rounding_op": (i32, [vp, i32, P_f64, C.POINTER(TTO), C.POINTER(TTV), P_i64, C.POINTER(SketchOpts),
                                     C.POINTER(TTVOut)]),
    "ttc_ttrand_rounding_residual": (i32, [vp, C.POINTER(TTO), C.POINTER(TTV), C.POINTER(TTV), P_i64,
                                           C.POINTER(SketchOpts), C.POINTER(TTVOut)]),
    "ttc_mpo_apply": (i32, [vp, C.POINTER(TTO), C.POINTER(TTV), C.POINTER(TTVOut)]),
    "ttc_dot": (i32, [vp, C.POINTER(TTV), C.POINTER(TTV), P_f64]),
    "ttc_partial_contraction": (i32, [vp, C.POINTER(TTV), C.POINTER(TTV), i32, PP_f64]),
    "ttc_dot_operator": (i32, [vp, C.POINTER(TTV), C.POINTER(TTO), C.POINTER(TTV), P_f64]),
    "ttc_tt_add": (i32, [vp, C.POINTER(TTV), C.POINTER(TTV), C.POINTER(TTVOut)]),
    "ttc_tt_scale": (i32, [vp, f64, C.POINTER(TTV), C.POINTER(TTVOut)]),
    "ttc_rayleigh_grad": (i32, [vp, C.POINTER(TTO), C.POINTER(TTV), i32, P_f64, PP_f64]),
    "ttc_rayleigh_grad_prec": (i32, [vp, C.POINTER(TTO), C.POINTER(TTV), i32, i32, P_f64, PP_f64]),
    "ttc_qr_noalloc": (i32, [i32, i32, vp, i64, vp, i64, vp, i64, vp, vp]),
    "ttc_host_alloc": (i32, [sz, C.POINTER(vp)]),
    "ttc_host_free": (i32, [vp]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

STATUS = {0: "TTC_OK", 1: "TTC_EARG", 2: "TTC_EDIM", 3: "TTC_ENOCONV", 4: "TTC_ENOTPD", 5: "TTC_ECUDA",
          6: "TTC_ENOMEM", 7: "TTC_EINTERNAL", 8: "TTC_ENONFINITE"}
