"""The multi-process path (replicas, one process per GPU) on CPU with gloo,
world size 2: the job's time is the maximum over ranks, its throughput all
ranks' units over that time; a rank that leaves before the collective makes
the other rank's collective end with an error (short process-group timeout),
not hang."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _init(rank, world, port, timeout_s=30):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _aggregate(rank, world, port, q):
    dist = _init(rank, world, port)
    from unifiedparticleframeworkcuda_b200 import replicas
    r, w, lr = replicas.world()
    units = 1000.0 * (rank + 1)        # rank 0: 1000 units, rank 1: 2000
    ms = 10.0 + 5.0 * rank             # rank 0: 10 ms, rank 1: 15 ms
    replicas.barrier()
    thr, job_ms = replicas.job_throughput(units, ms)
    mx = replicas.max_over_ranks(ms, -ms)
    q.put((r, w, lr, thr, job_ms, mx))
    dist.destroy_process_group()


def _leaver(rank, world, port, q):
    dist = _init(rank, world, port, timeout_s=3)
    from unifiedparticleframeworkcuda_b200 import replicas
    replicas.barrier()
    if rank == 1:
        q.put((rank, "left"))
        return  # leaves between steps, before the next collective
    try:
        replicas.max_over_ranks(1.0)
        q.put((rank, "no error"))
    except Exception as e:  # the collective ends with an error instead of waiting forever
        q.put((rank, "error: %s" % type(e).__name__))


def _run(fn, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_replica_aggregation_gloo_world_2():
    out = sorted(_run(_aggregate))
    for r, (rank, w, lr, thr, job_ms, mx) in enumerate(out):
        assert rank == r and w == 2 and lr == r
        assert job_ms == 15.0                       # the slowest rank's time
        assert thr == pytest.approx(3000.0 / 0.015)  # all ranks' units over it
        assert mx == [15.0, -10.0]


def test_rank_leaving_ends_the_collective_with_an_error():
    out = dict(_run(_leaver))
    assert out[1] == "left"
    assert out[0].startswith("error")
