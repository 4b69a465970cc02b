"""Multi-rank host path on CPU: two gloo ranks split a batch, solve their
slices with the oracle, and must reproduce the single-process result; the
timing reduction must return the maximum over ranks.

This is the N > 1 path of bench.py and of user code (one process per GPU,
batch split, no collective on the data path), exercised without GPUs.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from oracle import oracle
    from qpax_b200 import workloads as wl
    from qpax_b200.shard import barrier, max_over_ranks, shard_bounds

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        data = wl.dense(13, 6, 2, 12, 11)  # 13 instances: the two slices differ in size
        lo, hi = shard_bounds(13, rank, world)
        x, s, z, y, conv, iters = oracle.solve_qp(*[a[lo:hi] for a in data], solver_tol=1e-8, nthreads=1)
        barrier()
        t = max_over_ranks(10.0 * (rank + 1))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), lo=lo, hi=hi, x=x, conv=conv, iters=iters, t=t)
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_the_batch():
    from qpax_b200.shard import shard_bounds

    for batch in (0, 1, 7, 4096):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(batch, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == batch
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(4, 2, 2)


def test_two_gloo_ranks_split_the_batch(tmp_path):
    from oracle import oracle
    from qpax_b200 import workloads as wl

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    assert [int(p["lo"]) for p in parts] == [0, 6] and [int(p["hi"]) for p in parts] == [6, 13]
    assert all(float(p["t"]) == 20.0 for p in parts)  # max over ranks, seen by every rank
    full = oracle.solve_qp(*wl.dense(13, 6, 2, 12, 11), solver_tol=1e-8, nthreads=1)
    x = np.concatenate([p["x"] for p in parts])
    np.testing.assert_array_equal(x, full[0])
    np.testing.assert_array_equal(np.concatenate([p["conv"] for p in parts]), full[4])
    np.testing.assert_array_equal(np.concatenate([p["iters"] for p in parts]), full[5])
