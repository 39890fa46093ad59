"""Benchmark of the batched TT rounding path (libttcuda on B200).

Workload (the headline configuration): 64 TTvectors, d = 32 sites, n = 2; interior ranks drawn
uniformly in [16, 256] per TT and bond (seeded, clamped by r_and_d_to_rks); bond-k singular
values decay like 10^(-i/32) (left-orthonormal random cores, the bond decay absorbed into the
next core).  Data are synthetic (seeded numpy), generated on the host.

One step rounds the whole batch to tol = 1e-8 in two variants:
  * mixed : ttrand_rounding with a Gaussian sketch whose contractions run in BF16 on the
            tcgen05 tensor cores (FP32 accumulation), sketch ranks = default_rank_heuristic
            (r + ceil(max r / 2)), FP64 range finder / projection, then the FP64 truncated-SVD
            sweep tt_rounding(tol) (no range finder of this workload compresses, so the library
            plans no sketch: see `range_finder_levels_compressing`);   -> `value`
  * rank_limited: the same batch rounded to rank 64 (ttrand_rounding(y, 64) + SVD sweep against
            tt_rounding(rmax = 64)), where every interior range finder compresses;
  * fp64  : deterministic tt_rounding(tol) (FP64 QR sweep + truncated-SVD sweep) -> `fp64`.
`value` is whole-job roundings/s with the inputs resident in HBM (device events around K
replays of the captured plan); `e2e` is the same metric through the C ABI with host buffers
(upload, round, download every step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tensor-train-julia_b200"))

D, NPHYS, BATCH, RMIN, RMAX, TOL = 32, 2, 64, 16, 256, 1e-8
METRIC = "TT roundings/s at d=32,r=256: mixed vs FP64 GPU at 1e-8 rel err; % roofline"
# DRAM bytes (read + write) per launch of the step's two large kernels, from ncu section captures
# (dram__bytes_read.sum + dram__bytes_write.sum) of smaller cases of the same kernels, scaled to a
# 64-TT launch by the problems it holds (the factors stay in L2 within a launch, so a launch reads
# its inputs once and traffic grows with the problem count):
#  * householder_qr_kernel: 7.57 MB for a 32-TT orthogonalisation-sweep launch at bond 12
#    (unfoldings up to 512 x 256) -> 15.1 MB for 64 TTs;
#  * jacobi_svd (the Gram-block kernel): 33.75 MB for 64 preconditioned 256 x 256 factors
#    (bench.py --jacobi-bench), the largest launch of the SVD sweep.
DOMINANT_DRAM_BYTES_PER_LAUNCH_64TT = {
    "householder_qr": (15.1e6, "ncu capture of a 32-TT orthogonalisation-sweep QR launch (bond 12), x2 for 64 TTs"),
    "jacobi_svd": (33.75e6, "ncu capture of a 64-problem 256 x 256 launch (bench.py --jacobi-bench), the largest"),
}


# ------------------------------------------------------------------------- workload
def r_and_d(rks, dims, rmax):
    d = len(dims)
    new = [1] * len(rks)
    for i in range(d):
        new[i] = min(rks[i], int(np.prod(dims[:i])) if i else 1, int(np.prod(dims[i:])), rmax)
    return new


def make_tt(dims, ranks, seed, decay_per=32.0):
    """Left-orthonormal random cores; the decay 10^(-i/decay_per) of bond k is absorbed into core k+1."""
    g = np.random.default_rng(seed)
    N = len(dims)
    vec, prev = [], np.ones(1)
    for k in range(N):
        n, a, b = dims[k], ranks[k], ranks[k + 1]
        if k < N - 1:
            # orthonormal columns; a bond wider than n*a (i.i.d. rank draws) gets zero columns,
            # so its numerical rank is n*a
            q, _ = np.linalg.qr(g.standard_normal((n * a, b)))
            q = q[:, :b] if q.shape[1] >= b else np.pad(q, ((0, 0), (0, b - q.shape[1])))
            core = np.transpose(q.reshape(a, n, b, order="F"), (1, 0, 2)).copy()
        else:
            core = g.standard_normal((n, a, b))
            core /= np.linalg.norm(core)
        vec.append(np.asfortranarray(core * prev[None, :, None]))
        # unit RMS keeps the TT norm O(1) over 32 bonds (the zero test of the rounding is absolute)
        prev = 10.0 ** (-np.arange(b) / decay_per)
        prev /= np.sqrt(np.mean(prev ** 2))
    return vec


def batch_ranks(seed, batch=BATCH):
    """Rank lists of the batch's TTs: interior ranks i.i.d. U[RMIN, RMAX] per TT and bond, clamped."""
    g = np.random.default_rng(seed)
    dims = (NPHYS,) * D
    out = []
    for _ in range(batch):
        r = [1] + [int(v) for v in g.integers(RMIN, RMAX + 1, size=D - 1)] + [1]
        out.append(r_and_d(r, dims, max(r)))
    return dims, out


def workload(seed, batch=BATCH, indices=None):
    """The batch's TTs (all, or those at `indices`): TT i has its own generator seed, so any subset
    is generated without the others."""
    dims, ranks = batch_ranks(seed, batch)
    idx = range(batch) if indices is None else indices
    return dims, [(dims, ranks[i], make_tt(dims, ranks[i], seed * 100003 + i)) for i in idx]


def heuristic(rank_lists):
    """default_rank_heuristic of a list of TTs (src/tt_randtools.jl:40-50)."""
    rks = list(rank_lists[0])
    for r in rank_lists[1:]:
        rks = [max(a, b) for a, b in zip(rks, r)]
    over = int(math.ceil(0.5 * max(rks)))
    for k in range(1, len(rks) - 1):
        rks[k] += over
    return rks


def compressing_levels(dims, rank_lists, s):
    """(TT, bond) pairs whose range finder compresses: the sketch rank s_{k+1} is below both
    dimensions of y_k's unfolding (n_k e_k x r_{k+1}, e the sweep's effective ranks).  Only these
    read the sketch when the SVD sweep follows; with none, the library skips the sketch."""
    count = 0
    for r in rank_lists:
        e = 1
        for k in range(len(dims) - 1):
            q = min(dims[k] * e, r[k + 1], s[k + 1])
            count += q == s[k + 1]
            e = q
    return count


# ------------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, path):
        self.path, self.proc = path, None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, device_index):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l.strip()]
            rows = [r for r in rows if len(r) >= 9 and r[0].strip() == str(device_index)]
            if not rows:
                return out
            sm = [float(r[1]) for r in rows]
            out["sm_mhz"] = float(np.median(sm))
            out["sm_max_mhz"] = float(rows[0][2])
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = set()
            for r in rows:
                for nm, v in zip(names, r[5:9]):
                    if "Active" in v and "Not" not in v:
                        reasons.add(nm)
            out["reasons"] = sorted(reasons)
        except Exception:
            pass
        return out


# ------------------------------------------------------------------ CPU baselines
def cpu_reference_rate(dims, tts, rks, sample, start=0):
    """The FP64 CPU restatement of the reference path (ttrand_rounding + tt_rounding, LAPACK via
    numpy/scipy on all host cores) on `sample` TTs of the batch from index `start` (cyclically);
    returns (roundings/s, seconds, rounded TTs)."""
    sys.path.insert(0, ROOT)
    from oracle import tt_oracle as o
    outs = []
    t0 = time.perf_counter()
    for i in range(sample):
        dims_i, r, vec = tts[(start + i) % len(tts)]
        x = o.TTvector(len(dims_i), [c.copy() for c in vec], tuple(dims_i), list(r), [0] * len(dims_i))
        y = o.ttrand_rounding(x, rks, orthogonal=True, seed=1234, block_rks=len(dims_i))
        outs.append(o.tt_rounding(y, tol=TOL))
    dt = time.perf_counter() - t0
    return sample / dt, dt, outs


def oracle_comparison(oracle_outs, gpu_outs):
    """Largest ||y_gpu - y_oracle|| / ||y_oracle|| over the TTs both sides rounded (FP64 norm of the
    difference TT, computed by the oracle) and whether all truncation ranks are identical."""
    from oracle import tt_oracle as o
    diffs, same = [], True
    for yo, yg in zip(oracle_outs, gpu_outs):
        g = o.TTvector(yg.N, [np.asarray(c) for c in yg.ttv_vec], tuple(yg.ttv_dims), list(yg.ttv_rks), [0] * yg.N)
        same = same and list(yo.ttv_rks) == list(g.ttv_rks)
        diffs.append(o.rel_error(yo, g))
    return max(diffs), same


# ---------------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return
    dims, tts = workload(seed=7)
    rks = heuristic([r for _, r, _ in tts])
    sample = max(1, int(os.environ.get("TTC_REF_SAMPLE", "3")))
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_reference_rate(dims, tts, rks, 1)
    t_all = time.perf_counter()
    for step in range(args.steps):
        # the sample moves through the batch (step i rounds TTs sample*i ...), so that the rate is
        # not that of the same few rank draws every step
        cpu_reference_rate(dims, tts, rks, sample, start=step * sample)
    total = time.perf_counter() - t_all
    v = float(sample * args.steps / total)
    cores = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "roundings/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batched rounding: 64 TTs, d=32, n=2, ranks U[16,256], sigma 10^(-i/32), tol 1e-8",
                   "variant": "FP64 ttrand_rounding + tt_rounding (reference algorithm, CPU restatement)",
                   "sample": f"{sample} TT(s) of the batch per step, the next {sample} each step (cyclic)"},
        "cpu_baseline": {"value": v, "unit": "roundings/s", "cores": cores, "kind": "port",
                         "sample": f"{sample} TT(s) per step, moving through the 64-TT batch "
                                   "(CPU restatement of the Julia path; Julia is absent)"},
        "e2e": {"value": v, "unit": "roundings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- the other configurations
def rand_cores(dims, ranks, g, normalise=False):
    """N(0,1) cores of the given (clamped) ranks, Julia layout (n, r_{k-1}, r_k); with `normalise`
    each core is scaled by 1/sqrt(n r_k) like rand_tt(...; normalise=true)."""
    out = []
    for k, n in enumerate(dims):
        c = g.standard_normal((n, ranks[k], ranks[k + 1]))
        if normalise:
            c /= math.sqrt(n * ranks[k + 1])
        out.append(np.asfortranarray(c))
    return out


def device_ms(ctx, fn, reps, stream):
    """Device time of `reps` calls of fn (events on `stream`, the library's stream), after one
    warm-up call."""
    import torch
    fn()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = stream
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    ctx.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def other_configs(ttcuda, ctx, hbm_peak, stream):
    """Configs 1, 2 and 4 of the benchmark set, each through the library's public API on host
    tensors (end to end, transfers included) and, where one kernel bounds it, with that kernel's
    device time from the per-kernel profile."""
    import ttcuda.models as tm
    out = {}
    # config 1: tt_rounding(X; tol=1e-8, rmax=64), X = sum_{j=1..8} 2^-j X_j, X_j rank 8, n=2, d=20
    g = np.random.default_rng(101)
    dims = (2,) * 20
    r8 = r_and_d([1] + [8] * 19 + [1], dims, 8)
    X = None
    for j in range(1, 9):
        t = ttcuda.tt_scale(2.0 ** -j, ttcuda.TTvector(20, rand_cores(dims, r8, g), dims, r8))
        X = t if X is None else ttcuda.tt_add(X, t)
    ms1 = device_ms(ctx, lambda: ttcuda.tt_rounding(X, tol=1e-8, rmax=64), 20, stream)
    xb = ttcuda.DeviceBatch.from_tts([X], ctx=ctx)
    yb = ttcuda.DeviceBatch(dims, [X.ttv_rks], ctx=ctx)
    ms1d = device_ms(ctx, lambda: xb.round_det(yb, tol=1e-8, rmax=64, sync=False), 50, stream)
    Y = yb.download()[0]
    out["config1"] = {"workload": "tt_rounding(X; tol=1e-8, rmax=64), X = sum of 8 rank-8 N(0,1) TTs scaled 2^-j, "
                                  "n=2, d=20 (input ranks up to 64)",
                      "value": 1e3 / ms1, "unit": "roundings/s", "ms_per_rounding": ms1,
                      "path": "ttc_tt_rounding on host tensors (upload, round, download)",
                      "device_resident_ms": ms1d, "output_ranks_max": max(Y.ttv_rks)}
    # config 2: 1D Hubbard MPO (16 sites, t=1, U=4) applied to a rank-128 TT; apply, and
    # operator-aware randomized rounding with a rank-138 Gaussian sketch
    h, V = tm.hubbard_1D(16, t=1.0, U=4.0)
    H = tm.hV_to_mpo(h, V, (2,) * 32)
    dims2 = (2,) * 32
    r128 = r_and_d([1] + [128] * 31 + [1], dims2, 128)
    y = ttcuda.TTvector(32, rand_cores(dims2, r128, np.random.default_rng(40), normalise=True), dims2, r128)
    ctx.set_profiling(True)
    Hy = ttcuda.mpo_apply(H, y)
    prof = ctx.kernel_profile()["mpo_apply"]
    ctx.set_profiling(False)
    ms_apply = device_ms(ctx, lambda: ttcuda.mpo_apply(H, y), 5, stream)
    out_bytes = sum(8 * 2 * Hy.ttv_rks[k] * Hy.ttv_rks[k + 1] for k in range(32))
    in_bytes = sum(8 * c.size for c in y.ttv_vec) + sum(8 * c.size for c in H.tto_vec)
    kern_ms = prof[0] / max(1, prof[1]) * prof[1]      # device time of all apply launches of one call
    gbs = (out_bytes + in_bytes) / (kern_ms / 1e3) / 1e9 if kern_ms > 0 else None
    rks = [1] + [138] * 31 + [1]
    ms_op = device_ms(ctx, lambda: ttcuda.ttrand_rounding_op([1.0], H, [y], rks, orthogonal=False, seed=5,
                                                             block_rks=138), 3, stream)
    ms_op_tf = device_ms(ctx, lambda: ttcuda.ttrand_rounding_op([1.0], H, [y], rks, orthogonal=False, seed=5,
                                                                block_rks=138, precision="tf32"), 3, stream)
    z64 = ttcuda.ttrand_rounding_op([1.0], H, [y], rks, orthogonal=False, seed=5, block_rks=138)
    ztf = ttcuda.ttrand_rounding_op([1.0], H, [y], rks, orthogonal=False, seed=5, block_rks=138, precision="tf32")
    dz = ttcuda.tt_add(z64, ttcuda.tt_scale(-1.0, ztf))
    rel_tf = ttcuda.norm(dz) / ttcuda.norm(z64)

    def err_vs_Hy(z):     # ||H y - z|| / ||H y|| from inner products (the error is far above their cancellation)
        hh = ttcuda.dot(Hy, Hy)
        return math.sqrt(max(0.0, hh - 2.0 * ttcuda.dot(Hy, z) + ttcuda.dot(z, z)) / hh)
    err64, errtf = err_vs_Hy(z64), err_vs_Hy(ztf)
    out["config2"] = {"workload": "1D Hubbard MPO (hV_to_mpo on the GPU, 16 sites, t=1, U=4, MPO ranks up to "
                                  f"{max(H.tto_rks)}) x rank-128 N(0,1) TT; sketch rank 138 (block_rks=138)",
                      "apply": {"value": 1e3 / ms_apply, "unit": "contractions/s", "ms": ms_apply,
                                "path": "ttc_mpo_apply on host tensors (output ranks up to "
                                        f"{max(Hy.ttv_rks)}, {out_bytes / 1e6:.0f} MB written back)",
                                "roofline": {"kernel": "apply_kernel", "bound": "hbm", "achieved": gbs,
                                             "peak": hbm_peak, "unit": "GB/s",
                                             "frac": (gbs / hbm_peak) if (gbs and hbm_peak) else None,
                                             "bytes_per_call": out_bytes + in_bytes,
                                             "launch_ms": kern_ms, "launches": prof[1]}},
                      "operator_rounding_fp64": {"value": 1e3 / ms_op, "unit": "roundings/s", "ms": ms_op,
                                                 "path": "ttc_ttrand_rounding_op (H y never formed), FP64"},
                      "operator_rounding_tf32": {"value": 1e3 / ms_op_tf, "unit": "roundings/s", "ms": ms_op_tf,
                                                 "path": "the same with the operator sketch on the tcgen05 tensor "
                                                         "cores (TF32 operands, FP32 accumulation), FP64 range finder",
                                                 "rel_diff_vs_fp64": rel_tf,
                                                 "rel_err_vs_Hy": errtf, "rel_err_vs_Hy_fp64": err64,
                                                 "ranks_identical_fp64": ztf.ttv_rks == z64.ttv_rks}}
    # config 4: gradient of <x|H|x>/<x|x>, 4x4 open Hubbard (U=8) in snake ordering, x rank 256
    h4, V4 = tm.hubbard_2D(4, 4, t=1.0, U=8.0, w_pbc=False, L_pbc=False)
    sg = tm.snake_order(4, 4)
    H4 = tm.hV_to_mpo(h4[np.ix_(sg, sg)], V4[np.ix_(sg, sg, sg, sg)], (2,) * 32)
    r256 = r_and_d([1] + [256] * 31 + [1], dims2, 256)
    x4 = ttcuda.TTvector(32, rand_cores(dims2, r256, np.random.default_rng(41), normalise=True), dims2, r256)
    ctx.set_profiling(True)
    ttcuda.rayleigh_grad(H4, x4, ckpt_every=4)
    prof4 = ctx.kernel_profile()["gemm_f64"]
    ctx.set_profiling(False)
    ms_g = device_ms(ctx, lambda: ttcuda.rayleigh_grad(H4, x4, ckpt_every=4), 3, stream)
    ms_g32 = device_ms(ctx, lambda: ttcuda.rayleigh_grad(H4, x4, ckpt_every=4, precision="fp32"), 3, stream)
    R64, G64 = ttcuda.rayleigh_grad(H4, x4, ckpt_every=4)
    R32, G32 = ttcuda.rayleigh_grad(H4, x4, ckpt_every=4, precision="fp32")
    gd = math.sqrt(sum(float(np.sum((a - b) ** 2)) for a, b in zip(G32, G64)))
    gn = math.sqrt(sum(float(np.sum(b ** 2)) for b in G64))
    out["config4"] = {"workload": "gradient of <x|H|x>/<x|x> w.r.t. every core, 4x4 open Hubbard MPO (t=1, U=8, "
                                  f"snake ordering, MPO ranks up to {max(H4.tto_rks)}), x rank 256, environments "
                                  "checkpointed every 4 sites, FP64",
                      "value": 1e3 / ms_g, "unit": "gradients/s", "ms": ms_g,
                      "path": "ttc_rayleigh_grad on host tensors",
                      "gemm_f64": {"ms": prof4[0], "launches": prof4[1], "gflop": prof4[2] / 1e9,
                                   "tflops": (prof4[2] / (prof4[0] / 1e3) / 1e12) if prof4[0] > 0 else None},
                      "fp32": {"value": 1e3 / ms_g32, "unit": "gradients/s", "ms": ms_g32,
                               "variant": "FP32 cores and environments, FP32 accumulation",
                               "rel_diff_gradient_vs_fp64": gd / gn, "rel_diff_value_vs_fp64": abs(R32 - R64) / abs(R64)}}
    # config 5 shapes: 48 sites, x of rank 512, operator-aware rounding to rank 512 (block_rks = 512)
    # with the sketch contractions in BF16 on the tensor cores, FP32 accumulation, FP64 range
    # finder and QR.  The 48-spin-orbital molecular MPO has rank ~2L^2+3L+2 = 1226 (L = 24 spatial
    # orbitals); its roundings need Householder QRs of ~4900 rows, beyond the QR kernel's 1536, so a
    # stand-in MPO of the same sites with ranks min(4^k, 4^(d-k), 192) and N(0,1)/sqrt(4 R_k) cores
    # takes its place here.
    d5, R5, r5, s5 = 48, 192, 512, 512      # block_rks = 512: every bond's sketch rank is 512
    g5 = np.random.default_rng(55)
    Rk = [min(4 ** min(k, d5 - k), R5) for k in range(d5 + 1)]
    H5 = ttcuda.TToperator(d5, [np.asfortranarray(g5.standard_normal((2, 2, Rk[k], Rk[k + 1])) / math.sqrt(4 * Rk[k + 1]))
                                for k in range(d5)], (2,) * d5, Rk)
    dims5 = (2,) * d5
    rx = r_and_d([1] + [r5] * (d5 - 1) + [1], dims5, r5)
    x5 = ttcuda.TTvector(d5, rand_cores(dims5, rx, g5, normalise=True), dims5, rx)
    rks5 = [1] + [s5] * (d5 - 1) + [1]
    run5 = lambda prec: ttcuda.ttrand_rounding_op([1.0], H5, [x5], rks5, orthogonal=False, seed=5, block_rks=s5,  # noqa: E731
                                                  precision=prec)
    ms5b = device_ms(ctx, lambda: run5("bf16"), 2, stream)
    ms5d = device_ms(ctx, lambda: run5("fp64"), 1, stream)
    z5b, z5d = run5("bf16"), run5("fp64")
    # ||a - b|| / ||a|| from inner products: the difference TT has rank 1024, whose norm would need a
    # 2048-row QR; the BF16/FP64 difference is far above the expansion's cancellation level
    aa, ab, bb = ttcuda.dot(z5d, z5d), ttcuda.dot(z5d, z5b), ttcuda.dot(z5b, z5b)
    rel5 = math.sqrt(max(0.0, aa - 2.0 * ab + bb) / aa)
    # a randomized rounding is an orthogonal projection of H x (left-orthonormal cores), so <z, H x>
    # = ||z||^2 is the energy it captures; in this heavy compression (H x has rank up to 98304)
    # two sketches give different projections, and the captured energies compare their quality
    cap_b = ttcuda.dot_operator(z5b, H5, x5) / math.sqrt(bb)
    cap_d = ttcuda.dot_operator(z5d, H5, x5) / math.sqrt(aa)
    ctx.set_profiling(True)
    run5("bf16")
    prof5 = ctx.kernel_profile()
    ctx.set_profiling(False)
    tc = prof5["gemm_bf16_tcgen05"]
    gf5 = prof5["gemm_f64"]
    out["config5_shapes"] = {
        "workload": f"operator-aware ttrand_rounding([1.0], H, [x], rks): d=48, n=2, x rank {r5} (N(0,1), "
                    f"normalised), sketch rank {s5} (block_rks = {s5}, Gaussian), H a stand-in MPO of ranks "
                    f"min(4^k, 4^(d-k), {R5}) (the 48-spin-orbital molecular MPO, rank ~1226, exceeds the QR "
                    "kernel's 1536-row limit in its own rounding)",
        "value": 1e3 / ms5b, "unit": "roundings/s", "ms": ms5b,
        "variant": "BF16 operator sketch (tcgen05), FP32 accumulation; FP64 range finder, QR and projections",
        "fp64": {"value": 1e3 / ms5d, "unit": "roundings/s", "ms": ms5d},
        "rel_diff_vs_fp64": rel5, "ranks_identical_fp64": z5b.ttv_rks == z5d.ttv_rks,
        "captured_norm_bf16": cap_b, "captured_norm_fp64": cap_d,
        "captured_norm_ratio_bf16_over_fp64": cap_b / cap_d,
        "tcgen05_sketch": {"ms": tc[0], "launches": tc[1], "tflop": tc[2] / 1e12,
                           "tflops": (tc[2] / (tc[0] / 1e3) / 1e12) if tc[0] > 0 else None},
        "gemm_f64": {"ms": gf5[0], "launches": gf5[1], "tflop": gf5[2] / 1e12,
                     "tflops": (gf5[2] / (gf5[0] / 1e3) / 1e12) if gf5[0] > 0 else None},
        "profile_ms": {k: round(v[0], 3) for k, v in prof5.items() if v[1]}}
    out["callers"] = callers(ttcuda, ctx, stream, H, dims2)
    return out


def callers(ttcuda, ctx, stream, H, dims2):
    """The rounding path's callers on config-2/config-3 sizes: sketched Rayleigh-Ritz on the
    16-site Hubbard MPO, STTA of a rank-128 TT, and the randomized rounding of a Hadamard product
    (structured, against multiplying the product out and rounding it), each through the public
    API on host tensors."""
    import ttcuda.solvers as ts
    out = {}
    g = np.random.default_rng(60)
    # sketched Rayleigh-Ritz: 10 Krylov vectors, rmax 32, from a rank-16 start, on the MPO scaled by
    # 1/20 (the solver's tol = res_sketch^2 / 2 is a relative tolerance, so the operator's scale
    # must keep the sketched residual below 1)
    Hs = ttcuda.TToperator(32, [H.tto_vec[0] * 0.05] + list(H.tto_vec[1:]), H.tto_dims, H.tto_rks)
    r16 = r_and_d([1] + [16] * 31 + [1], dims2, 16)
    b0 = ttcuda.TTvector(32, rand_cores(dims2, r16, g, normalise=True), dims2, r16)
    ctx.synchronize()
    t0 = time.perf_counter()
    e, psi, hist = ts.sketched_rayleigh_ritz(Hs, b0, 10, 32)
    ctx.synchronize()
    t_rr = time.perf_counter() - t0
    out["sketched_rayleigh_ritz"] = {
        "workload": "sketched_rayleigh_ritz(H/20, b0, d=10, rmax=32): H the 16-site Hubbard MPO (t=1, U=4), b0 rank 16",
        "value": 10 / t_rr, "unit": "Krylov steps/s (wall clock, host linear algebra and transfers included)",
        "s": t_rr, "e_sketch": e, "e_true": hist[-1]["e_true"], "res_sketch": hist[-1]["res_sketch"],
        "e_true_history": [h["e_true"] for h in hist]}
    # STTA of a rank-128 TT (d=32, n=2, bond singular values 10^(-i/32)) to rank 64, against the
    # deterministic rounding to rank 64
    r128 = r_and_d([1] + [128] * 31 + [1], dims2, 128)
    x = ttcuda.TTvector(32, make_tt(dims2, r128, 61), dims2, r128)
    ms_st = device_ms(ctx, lambda: ttcuda.stta(x, 64, block_rks=8), 3, stream)
    ms_tr = device_ms(ctx, lambda: ttcuda.tt_rounding(x, rmax=64), 3, stream)
    zs, zt = ttcuda.stta(x, 64, block_rks=8), ttcuda.tt_rounding(x, rmax=64)

    def rel(a, b):
        return ttcuda.norm(ttcuda.tt_add(a, ttcuda.tt_scale(-1.0, b))) / ttcuda.norm(b)
    out["stta"] = {"workload": "stta(x, 64; block_rks=8), x rank 128, d=32, n=2, bond singular values 10^(-i/32)",
                   "value": 1e3 / ms_st, "unit": "approximations/s", "ms": ms_st,
                   "path": "ttc_stta on host tensors", "rel_err": rel(zs, x),
                   "tt_rounding_rmax64": {"ms": ms_tr, "rel_err": rel(zt, x)}}
    # Hadamard product of two rank-32 TTs (product rank 1024), rounded with sketch rank 64
    r32 = r_and_d([1] + [32] * 31 + [1], dims2, 32)
    x1 = ttcuda.TTvector(32, rand_cores(dims2, r32, g, normalise=True), dims2, r32)
    x2 = ttcuda.TTvector(32, rand_cores(dims2, r32, g, normalise=True), dims2, r32)
    ms_h = device_ms(ctx, lambda: ttcuda.ttrand_rounding_hadamard([x1, x2], 64), 3, stream)
    zh = ttcuda.ttrand_rounding_hadamard([x1, x2], 64)
    # the product multiplied out on the host (slice-wise Kronecker cores) and rounded on the GPU
    vec = []
    for k in range(32):
        a, b = x1.ttv_vec[k], x2.ttv_vec[k]
        vec.append(np.asfortranarray(np.stack([np.kron(a[i], b[i]) for i in range(2)])))
    rp = [p * q for p, q in zip(x1.ttv_rks, x2.ttv_rks)]
    P = ttcuda.TTvector(32, vec, dims2, rp)
    ms_p = device_ms(ctx, lambda: ttcuda.ttrand_rounding(P, 64), 3, stream)
    zp = ttcuda.ttrand_rounding(P, 64)
    out["hadamard_rounding"] = {
        "workload": "ttrand_rounding((x1, x2), 64): x1, x2 rank 32, d=32, n=2 (product rank 1024)",
        "value": 1e3 / ms_h, "unit": "roundings/s", "ms": ms_h, "path": "ttc_ttrand_rounding_hadamard on host tensors",
        "formed_product": {"ms": ms_p, "path": "ttc_ttrand_rounding of the product multiplied out on the host (rank-1024 cores, 512 MB uploaded per call)"},
        "rel_diff_vs_formed": rel(zh, zp)}
    return out


# ------------------------------------------------------------------- kernel benchmarks
def kernel_bench(reps):
    """The tcgen05 sketch GEMM in isolation on the operator-sketch shapes of config 5 (x rank 512,
    MPO rank 192 stand-in, sketch rank 512, n = 2: G1 M=1024 N=98304 K=512, G2 M=262144 N=384
    K=384, G3 M=98304 N=512 K=1024) and on a square 8192^3, device-resident operands, CUDA events
    on the library's stream; prints one JSON line."""
    import ctypes as C
    import torch  # noqa: F401  (initialises the device the way the main bench does)
    import ttcuda
    from ttcuda._lib import lib
    lib.ttc_test_tc_gemm_bench.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.c_double)]
    lib.ttc_test_tc_gemm_bench.restype = C.c_int
    ctx = ttcuda.Context(0)
    peak, src = 1590.0, "fallback (MEASURED_PEAKS.json absent)"
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
        src = "MEASURED_PEAKS.json bf16_tflops (measured burst)"
    except Exception:
        pass
    shapes = {"G1": (1024, 98304, 512), "G2": (262144, 384, 384), "G3": (98304, 512, 1024), "square": (8192, 8192, 8192)}
    out = {}
    for tf32 in (0, 1):
        for name, (m, n, k) in shapes.items():
            ms = C.c_double()
            ctx.check(lib.ttc_test_tc_gemm_bench(ctx.h, m, n, k, tf32, reps, C.byref(ms)))
            tf = 2.0 * m * n * k / (ms.value / 1e3) / 1e12
            out[("tf32:" if tf32 else "bf16:") + name] = {"m": m, "n": n, "k": k, "ms": ms.value, "tflops": tf,
                                                          "frac_of_bf16_peak": tf / peak}
    print(json.dumps({"kernel_bench": "gemm_bf16_tc_kernel", "peak_tflops": peak, "peak_source": src,
                      "results": out}), flush=True)


def jacobi_bench(reps, count=64, n=256):
    """The batched one-sided Jacobi SVD alone on `count` QR-LQ preconditioned n x n factors whose
    singular values decay as 10^(-i/32) (the SVD-sweep problems of the headline workload at full
    rank), CUDA events around `reps` launches (each after a copy of the inputs); prints one JSON
    line with the sweep counts and the work rate (6 m n^2 flops per sweep: the dot products and
    rotations of all n (n - 1) / 2 column pairs)."""
    import ctypes as C
    import torch  # noqa: F401
    import ttcuda
    from ttcuda._lib import lib
    lib.ttc_test_jacobi_bench.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int,
                                          C.POINTER(C.c_double), C.POINTER(C.c_int)]
    lib.ttc_test_jacobi_bench.restype = C.c_int
    ctx = ttcuda.Context(0)
    g = np.random.default_rng(7)
    mats = []
    sig = 10.0 ** (-np.arange(n) / 32.0)
    for _ in range(count):
        u, _ = np.linalg.qr(g.standard_normal((n, n)))
        v, _ = np.linalg.qr(g.standard_normal((n, n)))
        a = (u * sig) @ v.T
        _, r1 = np.linalg.qr(a.T)                 # M^T = Q R1, then R1^T = Q2 R2: Jacobi on R2^T
        _, r2 = np.linalg.qr(r1.T)
        mats.append(np.asfortranarray(r2.T))
    X = np.concatenate([m.ravel(order="F") for m in mats])
    ms = C.c_double()
    sw = np.zeros(count, dtype=np.int32)
    ctx.check(lib.ttc_test_jacobi_bench(ctx.h, count, n, n, X.ctypes.data_as(C.POINTER(C.c_double)), reps,
                                        C.byref(ms), sw.ctypes.data_as(C.POINTER(C.c_int))))
    work = float(np.abs(sw).sum()) * 6.0 * n * n * n     # per sweep: n^2 / 2 pairs of 12 m flops
    print(json.dumps({"jacobi_bench": "jacobi_svd_kernel", "count": count, "m": n, "n": n, "ms": ms.value,
                      "sweeps_mean": float(np.abs(sw).mean()), "sweeps_max": int(np.abs(sw).max()),
                      "work_tflops": work / (ms.value / 1e3) / 1e12}), flush=True)


# ---------------------------------------------------------------------------- ours
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--jacobi-bench", action="store_true",
                    help="time the batched Jacobi SVD alone on 64 preconditioned 256 x 256 factors")
    ap.add_argument("--no-other-configs", action="store_true", help="skip the config 1, 2, 4 and 5 lines")
    ap.add_argument("--kernel-bench", action="store_true",
                    help="time the tcgen05 sketch GEMM alone on the config-5 shapes and exit")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.kernel_bench:
        kernel_bench(max(3, args.steps))
        return
    if args.jacobi_bench:
        jacobi_bench(max(1, args.steps))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    import ttcuda
    from ttcuda import shard

    ctx = ttcuda.Context(local)
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream.cuda_stream)
    ttcuda._CTX = ctx

    # one job of batch x world TTs, partitioned over the ranks by estimated work (sum of r_k^3)
    job = args.batch * world
    _, job_ranks = batch_ranks(7, job)
    mine = shard.shard_by_work([shard.tt_work(r) for r in job_ranks], world)[rank]
    dims, tts = workload(seed=7, batch=job, indices=mine)
    ranks = [r for _, r, _ in tts]
    tt_objs = [ttcuda.TTvector(len(d_), v, d_, r, [0] * len(d_)) for d_, r, v in tts]
    rks = heuristic(job_ranks)              # the whole job's default_rank_heuristic
    block = D                        # ttrand_rounding's default block_rks = N
    s = ttcuda._sketch_ranks(dims, rks, block)
    rho = ttcuda._rand_out_caps(dims, s)
    n_compress = compressing_levels(dims, ranks, s)
    xb = ttcuda.DeviceBatch.from_tts(tt_objs, ctx=ctx)
    y_mixed = ttcuda.DeviceBatch(dims, [rho] * len(tts), ctx=ctx)
    y_fp64 = ttcuda.DeviceBatch(dims, ranks, ctx=ctx)
    y_tf32 = ttcuda.DeviceBatch(dims, [rho] * len(tts), ctx=ctx)

    def step_mixed(sync=False):
        xb.round_rand(y_mixed, rks, orthogonal=True, seed=1234, block_rks=block, precision="bf16",
                      after_tol=TOL, sync=sync)

    def step_fp64(sync=False):
        xb.round_det(y_fp64, tol=TOL, sync=sync)

    def step_tf32(sync=False):     # the same randomized rounding with TF32 sketch contractions
        xb.round_rand(y_tf32, rks, orthogonal=True, seed=1234, block_rks=block, precision="tf32",
                      after_tol=TOL, sync=sync)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(fn, K):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            fn()
        e1.record(stream)
        barrier()
        return shard.max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")

    # warm-up (builds and captures the plans)
    for _ in range(max(3, args.warmup)):
        step_mixed(sync=True)
        step_fp64(sync=True)
        step_tf32(sync=True)
    ctx.synchronize()

    # L2: the resident inputs (sum of core bytes) exceed the 126 MB L2
    in_bytes = sum(8 * sum(d_[k] * r[k] * r[k + 1] for k in range(D)) for d_, r, _ in tts)

    import tempfile
    clock_path = os.path.join(tempfile.gettempdir(), f"ttc_bench_clocks_rank{rank}_{os.getpid()}.csv")
    with ClockSampler(clock_path) as cs:
        ms_mixed = timed(step_mixed, args.steps)
        ms_fp64 = timed(step_fp64, args.steps)
        ms_tf32 = timed(step_tf32, args.steps)
    launches_t = ctx.stats()["kernel_launches"]     # launches of one TF32 step (the last plan run)
    ctx.synchronize()
    clocks = cs.summary(local)

    value = shard.job_rate(job, args.steps, ms_mixed)
    fp64_value = shard.job_rate(job, args.steps, ms_fp64)
    tf32_value = shard.job_rate(job, args.steps, ms_tf32)

    # accuracy on the GPU: ||x - round(x)|| / ||x|| through the library (difference TT, norm)
    def rel_err(x, y):
        d_ = ttcuda.tt_add(x, ttcuda.tt_scale(-1.0, ttcuda.TTvector(y.N, y.ttv_vec, y.ttv_dims, y.ttv_rks, [0] * y.N)))
        return ttcuda.norm(d_) / ttcuda.norm(x)

    out_m = y_mixed.download()
    out_f = y_fp64.download()
    nerr = min(4, len(tts))
    err_mixed = max(rel_err(tt_objs[i], out_m[i]) for i in range(nerr))
    err_fp64 = max(rel_err(tt_objs[i], out_f[i]) for i in range(nerr))
    err_mf = max(rel_err(out_f[i], out_m[i]) for i in range(nerr))
    ranks_equal = all(out_m[i].ttv_rks == out_f[i].ttv_rks for i in range(len(tts)))
    out_t = y_tf32.download()
    err_tf = max(rel_err(out_f[i], out_t[i]) for i in range(nerr))
    ranks_equal_tf = all(out_t[i].ttv_rks == out_f[i].ttv_rks for i in range(len(tts)))

    # the same batch rounded to rank 64 (ttrand_rounding(y, 64) + SVD sweep, against tt_rounding with
    # rmax = 64): here the sketch compresses every interior bond, the case randomized rounding is for
    rmax_c = 64
    rks_c = [1] + [rmax_c] * (D - 1) + [1]
    s_c = ttcuda._sketch_ranks(dims, rks_c, block)
    y_cm = ttcuda.DeviceBatch(dims, [ttcuda._rand_out_caps(dims, s_c)] * len(tts), ctx=ctx)
    y_cf = ttcuda.DeviceBatch(dims, ranks, ctx=ctx)

    def step_c_mixed(sync=False):
        xb.round_rand(y_cm, rks_c, orthogonal=True, seed=1234, block_rks=block, precision="bf16",
                      after_tol=TOL, rmax=rmax_c, sync=sync)

    def step_c_fp64(sync=False):
        xb.round_det(y_cf, tol=TOL, rmax=rmax_c, sync=sync)

    for _ in range(max(3, args.warmup)):
        step_c_mixed(sync=True)
        step_c_fp64(sync=True)
    ms_cm = timed(step_c_mixed, args.steps)
    ms_cf = timed(step_c_fp64, args.steps)
    out_cm, out_cf = y_cm.download(), y_cf.download()
    compress_line = {
        "variant": f"rank {rmax_c}: BF16-sketch ttrand_rounding(y, {rmax_c}) + FP64 SVD sweep (tol {TOL:g}, rmax "
                   f"{rmax_c}) against deterministic tt_rounding(tol {TOL:g}, rmax {rmax_c})",
        "mixed": {"value": shard.job_rate(job, args.steps, ms_cm), "ms_per_step": ms_cm / args.steps,
                  "rel_err_max": max(rel_err(tt_objs[i], out_cm[i]) for i in range(nerr))},
        "fp64": {"value": shard.job_rate(job, args.steps, ms_cf), "ms_per_step": ms_cf / args.steps,
                 "rel_err_max": max(rel_err(tt_objs[i], out_cf[i]) for i in range(nerr))},
        "mixed_over_fp64": ms_cf / ms_cm,
        "range_finder_levels_compressing": compressing_levels(dims, ranks, s_c),
        "unit": "roundings/s", "checked_tts": nerr,
    }

    # per-kernel profile of one extra step of each variant (event pair around every launch)
    ctx.set_profiling(True)

    def sweeps(st):
        n_ = max(1, st["jacobi_problems"])
        return {"problems": st["jacobi_problems"], "mean": round(st["jacobi_sweeps_sum"] / n_, 2),
                "max": st["jacobi_sweeps_max"]}

    # NVTX ranges name the profiled steps for ncu (--nvtx --nvtx-include "ttc_mixed_step/")
    torch.cuda.nvtx.range_push("ttc_mixed_step")
    step_mixed(sync=True)
    torch.cuda.nvtx.range_pop()
    prof_m = ctx.kernel_profile()
    st = ctx.stats()
    launches_m, sw_m = st["kernel_launches"], sweeps(st)
    torch.cuda.nvtx.range_push("ttc_fp64_step")
    step_fp64(sync=True)
    torch.cuda.nvtx.range_pop()
    prof_f = ctx.kernel_profile()
    st = ctx.stats()
    launches_f, sw_f = st["kernel_launches"], sweeps(st)
    ctx.set_profiling(False)

    # FP64 and TF32 peaks of this GPU (torch.matmul, best of 10): the roofline denominators of
    # the FP64 kernels and of the TF32 sketch
    def matmul_peak(nmat, dtype):
        a = torch.randn(nmat, nmat, dtype=dtype, device=f"cuda:{local}")
        bmat = torch.randn(nmat, nmat, dtype=dtype, device=f"cuda:{local}")
        torch.matmul(a, bmat)
        best = 1e9
        for _ in range(10):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, bmat)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return 2 * nmat ** 3 / (best / 1e3) / 1e12

    fp64_peak_tflops = matmul_peak(4096, torch.float64)
    allow = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    tf32_peak_tflops = matmul_peak(8192, torch.float32)
    torch.backends.cuda.matmul.allow_tf32 = allow

    # dominant kernel of the mixed step: device time per launch (event pair around each launch)
    # and its algorithmic FLOPs per launch (the library's fixed conventions, from the launch shapes)
    dom, (dom_ms, dom_n, dom_flops) = max(prof_m.items(), key=lambda kv: kv[1][0])
    dom_avg_ms = dom_ms / max(1, dom_n)
    achieved = (dom_flops / max(1, dom_n)) / (dom_avg_ms / 1e3) / 1e12 if dom_flops else None
    flops_mixed = sum(v[2] for v in prof_m.values())
    flops_fp64 = sum(v[2] for v in prof_f.values())

    others = None
    if rank == 0 and not args.no_other_configs:
        hbm, hbm_src = 6650.0, "fallback (MEASURED_PEAKS.json absent)"
        try:
            hbm = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
            hbm_src = "MEASURED_PEAKS.json hbm_gbs (measured)"
        except Exception:
            pass
        others = other_configs(ttcuda, ctx, hbm, stream)
        others["config2"]["apply"]["roofline"]["peak_source"] = hbm_src

    # end-to-end through the C ABI with host buffers (upload, round, download) every step; device
    # events on the library's stream bracket the whole loop, host-side gaps included.  The
    # inputs sit in page-locked host memory (copied there before the timed region), the results
    # come back into the reused page-locked buffers of download(reuse=True)
    tt_pinned = [ttcuda.pinned_tt(t) for t in tt_objs]
    y_mixed.download(reuse=True)
    h2d = in_bytes
    d2h = 0
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        xb.upload(tt_pinned)
        step_mixed(sync=True)
        outs = y_mixed.download(reuse=True)
        d2h = sum(8 * sum(o_.ttv_dims[k] * o_.ttv_rks[k] * o_.ttv_rks[k + 1] for k in range(D)) for o_ in outs)
    e1.record(stream)
    barrier()
    e2e_ms = shard.max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")
    e2e_value = shard.job_rate(job, args.steps, e2e_ms)

    cpu = None
    oracle_cmp = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, secs, ref_outs = cpu_reference_rate(dims, tts, rks, 3)
        cpu = {"value": rate, "unit": "roundings/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"first 3 TTs of the batch ({secs:.1f} s): FP64 ttrand_rounding + tt_rounding, "
                         "numpy/LAPACK on all host threads"}
        # the same 3 TTs rounded by the GPU (mixed and FP64 variants) against the oracle's results
        d_m, same_m = oracle_comparison(ref_outs, out_m[:3])
        d_f, same_f = oracle_comparison(ref_outs, out_f[:3])
        oracle_cmp = {"rel_diff_vs_oracle": d_m, "ranks_identical_oracle": same_m,
                      "fp64_rel_diff_vs_oracle": d_f, "fp64_ranks_identical_oracle": same_f, "oracle_checked_tts": 3,
                      "oracle": "FP64 restatement, same Philox sketch blocks (seed 1234)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "roundings/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_mixed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 sketch + f64", "data": "synthetic",
            "config": {"workload": f"batched rounding: {job} TTs ({args.batch} per GPU, partitioned by sum of r^3), "
                                   "d=32, n=2, ranks U[16,256] (seeded), sigma 10^(-i/32), tol 1e-8",
                       "variant": "mixed: BF16-sketch (tcgen05) ttrand_rounding + FP64 SVD sweep",
                       "sketch_ranks": "default_rank_heuristic of the batch (r + ceil(max r/2)); block_rks = N, "
                                       "orthogonal blocks, seed 1234 (ttrand_rounding defaults)",
                       "range_finder_levels_compressing": n_compress,
                       "range_finder_levels": len(tts) * (D - 1),
                       "range_finder_note": "a level compresses when its sketch rank is below both dimensions of "
                                            "y_k's unfolding; with none, every range finder is a plain QR of y_k "
                                            "and the library skips the sketch (the SVD sweep needs only range(Q)), "
                                            "so the mixed and FP64 steps do the same FP64 work",
                       "l2": f"inputs {in_bytes / 1e6:.0f} MB resident > 126 MB L2"},
            "fp64": {"value": fp64_value, "unit": "roundings/s", "ms_per_step": ms_fp64 / args.steps,
                     "variant": "deterministic tt_rounding (FP64 Householder QR sweep + Jacobi SVD sweep)"},
            "tf32": {"value": tf32_value, "unit": "roundings/s", "ms_per_step": ms_tf32 / args.steps,
                     "variant": "TF32-sketch (tcgen05 kind::tf32) ttrand_rounding + FP64 SVD sweep",
                     "rel_diff_vs_fp64": err_tf, "ranks_identical_fp64": ranks_equal_tf},
            "peaks": {"fp64_tflops": fp64_peak_tflops, "tf32_tflops": tf32_peak_tflops,
                      "source": "torch.matmul 4096^3 FP64 and 8192^3 FP32 with TF32 allowed, best of 10, "
                                "this run"},
            "mixed_over_fp64": value / fp64_value,
            "rank_limited": compress_line,
            "accuracy": {"rel_err_mixed_max": err_mixed, "rel_err_fp64_max": err_fp64,
                         "rel_diff_mixed_vs_fp64": err_mf, "ranks_identical": ranks_equal,
                         "checked_tts": nerr},
            "gflops_per_s": {"mixed_algorithmic": flops_mixed * world * args.steps
                             / (ms_mixed / 1e3) / 1e9,
                             "fp64_algorithmic": flops_fp64 * world * args.steps / (ms_fp64 / 1e3) / 1e9},
            "roofline": {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": fp64_peak_tflops,
                         "unit": "TFLOP/s", "frac": (achieved / fp64_peak_tflops) if achieved else None,
                         "traffic": (DOMINANT_DRAM_BYTES_PER_LAUNCH_64TT[dom][0]
                                     if dom in DOMINANT_DRAM_BYTES_PER_LAUNCH_64TT and len(tts) == 64 else None),
                         "traffic_note": (DOMINANT_DRAM_BYTES_PER_LAUNCH_64TT[dom][1] + "; far below the launch's "
                                          "algorithmic bytes: latency-bound, the factors stay in L2"
                                          if dom in DOMINANT_DRAM_BYTES_PER_LAUNCH_64TT else None),
                         "peak_source": "FP64 torch.matmul (cuBLAS DGEMM) 4096^3, best of 10, measured in this run "
                                        "(MEASURED_PEAKS.json has no FP64 entry)",
                         "avg_launch_ms": dom_avg_ms, "launches_per_step": dom_n,
                         "profile_ms_per_step": {k: round(v[0], 3) for k, v in prof_m.items() if v[1]},
                         "profile_gflop_per_step": {k: round(v[2] / 1e9, 3) for k, v in prof_m.items() if v[1]}},
            "kernel_profile_fp64_ms": {k: round(v[0], 3) for k, v in prof_f.items() if v[1]},
            "jacobi_sweeps": {"mixed": sw_m, "fp64": sw_f},
            "e2e": {"value": e2e_value, "unit": "roundings/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "path": "DeviceBatch.upload (cores in page-locked host memory, DMA) -> round_rand -> "
                            "download(reuse=True) into page-locked host buffers"},
            "gpu_launches": int((launches_m + launches_f + launches_t) * args.steps),
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if oracle_cmp:
            line["accuracy"].update(oracle_cmp)
        if others:
            line["configs"] = others
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
