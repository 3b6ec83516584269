"""The multi-GPU path on CPU: two ranks over torch.distributed (gloo).

bench.py runs one shard of particles per rank with no data-path collective
(particles are independent; every rank holds its own copy of the mesh and
records) and takes the job's time as the maximum over ranks.  Here two
processes check, with the gloo backend, that the shards' key ranges
(bench.shard_pid_base) tile the global range, that the draws of each shard
(the oracle's counter RNG, the same function the kernels compute) equal the
draws of one run over all particles, and that bench.max_over_ranks returns
the slowest rank's time on every rank.
"""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P_PER_RANK = 5000


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    import bench
    from oracle import oracle as O
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        base = bench.shard_pid_base(rank, P_PER_RANK)
        draws = O.lib()   # the oracle's draws for this shard's keys
        g = np.empty((P_PER_RANK, 2))
        draws.orc_normals(P_PER_RANK, 20240917, 3, 77, base, 0, O._p(g))
        slowest = bench.max_over_ranks(10.0 + rank, dist, "cpu")
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), base=base, draws=g, slowest=slowest)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_keys_and_max_time(tmp_path):
    import multiprocessing as mp
    from oracle import oracle as O
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    assert [int(r["base"]) for r in res] == [r * P_PER_RANK for r in range(world)]
    assert all(float(r["slowest"]) == 10.0 + world - 1 for r in res)
    whole = np.empty((world * P_PER_RANK, 2))
    O.lib().orc_normals(world * P_PER_RANK, 20240917, 3, 77, 0, 0, O._p(whole))
    assert np.array_equal(np.concatenate([r["draws"] for r in res]), whole)


def test_single_process_helpers():
    import bench
    assert bench.shard_pid_base(0, 123) == 0 and bench.shard_pid_base(3, 123) == 369
    assert bench.max_over_ranks(4.5, None, "cpu") == 4.5
