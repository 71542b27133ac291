"""Multi-GPU runs of bench.py are replicas: every rank advances its own
lattice (a single lattice's sweep does not shard without a halo exchange) and
the job time is the slowest rank's.  The rank-level host logic is checked
here with two gloo processes on the CPU."""
import datetime
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    t = bench.max_over_ranks_dist(1.5 + rank, world, "cpu")
    q.put((rank, t, bench.replica_seed(rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_time_is_max_over_ranks_and_seeds_differ():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert [r for r, _, _ in res] == [0, 1]
    assert all(t == 2.5 for _, t, _ in res)
    assert res[0][2] != res[1][2]
    assert all(p.exitcode == 0 for p in procs)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks_dist(3.0, 1, "cpu") == 3.0
