"""Multi-GPU batch sharding (bench.py --gpus N), run as two gloo ranks on CPU.

Every rank derives the whole job's rank lists from one seed, partitions the job by estimated
work (sum over bonds of r_k^3, greedy), generates and rounds only its own TTs (here with the FP64
oracle standing in for the device), and the results are gathered on the host.  The gathered
ranks and errors must equal those of one rank rounding the whole job, every TT must be rounded
exactly once, and the job time is the maximum over ranks.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JOB = 6
DIMS = (2,) * 10


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _job_ranks(seed=3):
    g = np.random.default_rng(seed)
    out = []
    from oracle import tt_oracle as o
    for _ in range(JOB):
        r = [1] + [int(v) for v in g.integers(2, 13, size=len(DIMS) - 1)] + [1]
        out.append(o.r_and_d_to_rks(r, DIMS, rmax=max(r)))
    return out


def _round_one(i, ranks):
    """The oracle's tt_rounding of job TT i (its own seed): (ranks, relative error)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_helpers import decaying_tt
    from oracle import tt_oracle as o
    x = decaying_tt(DIMS, ranks, seed=1000 + i, decay_per=2.0)
    y = o.tt_rounding(x, tol=1e-4)
    return list(y.ttv_rks), o.rel_error(x, y)


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tensor-train-julia_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import pickle
    import time

    import torch.distributed as dist

    from ttcuda import shard

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        job_ranks = _job_ranks()
        shards = shard.shard_by_work([shard.tt_work(r) for r in job_ranks], world)
        t0 = time.perf_counter()
        mine = {i: _round_one(i, job_ranks[i]) for i in shards[rank]}
        ms = 1e3 * (time.perf_counter() - t0)
        job_ms = shard.max_over_ranks(ms, dist, "cpu")
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump({"shards": shards, "gathered": gathered, "ms": ms, "job_ms": job_ms}, f)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_shard_by_work_balances_uneven_batches():
    sys.path.insert(0, os.path.join(ROOT, "tensor-train-julia_b200"))
    from ttcuda import shard
    works = [1000.0, 10.0, 10.0, 10.0, 990.0, 5.0]
    s = shard.shard_by_work(works, 2)
    assert sorted(i for part in s for i in part) == list(range(6))
    loads = [sum(works[i] for i in part) for part in s]
    assert max(loads) - min(loads) <= max(works)
    assert s == [[0, 2, 5], [1, 3, 4]]                  # 1000+10+5 vs 990+10+10
    # (a count split of this list, [0,1,2] and [3,4,5], would carry 1020 against 1005)
    assert shard.tt_work([1, 4, 2, 1]) == 1 + 64 + 8 + 1


def test_two_gloo_ranks_round_their_work_shards(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    import pickle
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    r0 = pickle.load(open(tmp_path / "rank0.pkl", "rb"))
    r1 = pickle.load(open(tmp_path / "rank1.pkl", "rb"))
    # both ranks computed the same partition, covering the job once
    assert r0["shards"] == r1["shards"]
    assert sorted(i for part in r0["shards"] for i in part) == list(range(JOB))
    # max over ranks: both report the slower rank's time
    assert r0["job_ms"] == r1["job_ms"] == pytest.approx(max(r0["ms"], r1["ms"]))
    merged = {}
    for part in r0["gathered"]:
        merged.update(part)
    assert r0["gathered"] == r1["gathered"]
    sys.path.insert(0, ROOT)
    job_ranks = _job_ranks()
    for i in range(JOB):                                # one rank rounding the whole job
        ranks, err = _round_one(i, job_ranks[i])
        assert merged[i][0] == ranks
        assert merged[i][1] == pytest.approx(err, rel=1e-12, abs=1e-15)
