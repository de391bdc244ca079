"""Replica timing of bench.py across ranks (gloo, world size 2, CPU): the slowest rank's time
sets the whole-job rate, which sums the ranks' work ("replicas only": no data-path
collective)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 if rank == 0 else 25.0          # rank 1 is the slow one
        q.put((rank, bench.reduce_max(ms), bench.replica_rate(1e9, ms, world)))
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, rate in out:
        assert mx == 25.0
        assert rate == pytest.approx(2 * 1e9 / 25.0 / 1e6)
