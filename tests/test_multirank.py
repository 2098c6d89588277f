"""World-size-2 gloo test of the bench's multi-GPU bookkeeping (CPU only).

The multi-GPU mode is "replicas only": each rank advances its own copy of
the model with no data-path exchange; the job's time is the slowest rank's
timed region and the throughput counts all replicas' work.
"""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    local = [0.75, 1.25][rank]  # seconds each replica took
    t = bench.max_over_ranks(local, dist, "cpu")
    units = bench.replica_units(1000, 3, 10, world)
    q.put((rank, t, units / t, bench.dist_env()))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, value, env in out:
        assert t == pytest.approx(1.25)
        assert value == pytest.approx(1000 * 125 * 3 * 10 * 2 / 1.25)
        assert env[0] == rank and env[1] == 2
