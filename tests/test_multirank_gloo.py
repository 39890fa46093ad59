"""Host logic of the multi-GPU batch sharding (bench.py --gpus N), run as two gloo ranks on CPU.

Each rank generates its own synthetic batch from its rank seed, rounds it with no data-path
collective, and the job time is the maximum over ranks; these checks cover that logic without
a GPU.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tensor-train-julia_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    import bench
    from ttcuda import shard

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dims, tts = bench.workload(seed=shard.rank_seed(7, rank), batch=2)
        checksum = float(sum(float(np.sum(c)) for _, _, vec in tts for c in vec[:3]))
        ms = 10.0 * (rank + 1)                      # stand-in device time of this rank
        job_ms = shard.max_over_ranks(ms, dist, "cpu")
        rate = shard.whole_job_rate(len(tts), world, 3, job_ms)
        idx = list(shard.shard_indices(5, rank, world))
        import torch
        sums = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(sums, torch.tensor([checksum], dtype=torch.float64))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([job_ms, rate, len(idx), idx[0] if idx else -1] + [float(t.item()) for t in sums]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_batch_and_reduce_max(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    # max over ranks: both ranks report the slower rank's time and the same whole-job rate
    assert r0[0] == r1[0] == 20.0
    assert r0[1] == r1[1] == pytest.approx(2 * 2 * 3 / 0.020)
    # 5 TTs over 2 ranks: 3 + 2, contiguous
    assert (r0[2], r0[3], r1[2], r1[3]) == (3, 0, 2, 3)
    # each rank owns a different, reproducible batch
    assert r0[4] == r1[4] and r0[5] == r1[5] and r0[4] != r0[5]
