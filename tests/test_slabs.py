"""Bookkeeping of the slab decomposition (unifiedparticleframeworkcuda_b200/
slabs.py) on the CPU: migration of particles that crossed a face, the halo
(ghosts) each slab receives, the exchange of fixed rows and the maximum over
slabs. Two gloo ranks (one slab each, DistTransport) and one process with
three slabs (LocalTransport). The same functions run on the device tensors
of a GPU run."""
import math
import os
import socket

import numpy as np
import pytest
import torch

from unifiedparticleframeworkcuda_b200 import slabs

WIDTH = 0.05


def _state(ids, rng):
    n = len(ids)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0, 1, (n, 3))
    return {"pos": torch.from_numpy(pos), "vel": torch.from_numpy(rng.normal(size=(n, 4)).astype(np.float32)),
            "lag": torch.from_numpy(rng.normal(size=(n, 4)).astype(np.float32)),
            "type": torch.full((n,), 2, dtype=torch.int32), "id": torch.from_numpy(np.asarray(ids, np.int32))}


def _check(all_pos, bounds, owned, ghosts, sent):
    """Ownership and halo invariants against the global picture."""
    ids = np.concatenate([o["id"].numpy() for o in owned])
    assert np.array_equal(np.sort(ids), np.arange(len(all_pos)))  # every particle owned exactly once
    for k, ((lo, hi), o) in enumerate(zip(bounds, owned)):
        x = o["pos"][:, 0].numpy()
        assert np.all((x >= lo) & (x < hi))
        np.testing.assert_array_equal(o["pos"].numpy(), all_pos[o["id"].numpy()])  # payload intact
        g = ghosts[k]
        gid = slabs.untag(torch, g["id"]).numpy() if g is not None else np.zeros(0, np.int64)
        fr = slabs.is_from_right(torch, g["id"]).numpy() if g is not None else np.zeros(0, bool)
        assert g is None or np.all(g["id"].numpy() < 0)  # ghost bit
        gx = all_pos[:, 0]
        want_left = np.flatnonzero((gx >= bounds[k - 1][0]) & (gx < lo) & (gx >= lo - WIDTH)) if k > 0 else []
        want_right = np.flatnonzero((gx >= hi) & (gx < hi + WIDTH) & (gx < bounds[k + 1][1])) \
            if k + 1 < len(bounds) else []
        assert np.array_equal(gid[~fr], np.sort(want_left))
        assert np.array_equal(gid[fr], np.sort(want_right))
        if g is not None:
            np.testing.assert_array_equal(g["pos"].numpy(), all_pos[gid])
        # what this slab sent: its own particles near each face, ascending
        sl, sr = sent[k]
        ox = all_pos[:, 0]
        mine = (ox >= lo) & (ox < hi)
        assert np.array_equal(sl.numpy(), np.flatnonzero(mine & (ox < lo + WIDTH))) if k > 0 or True else True
        assert np.array_equal(sr.numpy(), np.flatnonzero(mine & (ox >= hi - WIDTH)))


def test_local_transport_three_slabs():
    rng = np.random.default_rng(1)
    n = 3000
    bounds = slabs.slab_bounds(0.0, 1.0, 3)
    start = _state(np.arange(n), rng)
    x0 = start["pos"][:, 0].numpy()
    states = [slabs.select(start, torch.from_numpy((x0 >= lo) & (x0 < hi))) for lo, hi in bounds]
    # a step moves particles, some across faces; the previous ghosts are dropped
    for st in states:
        st["pos"][:, 0] += torch.from_numpy(rng.uniform(-0.04, 0.04, st["pos"].shape[0]).astype(np.float32))
    ghost = slabs.select(_state(np.arange(50), rng), torch.ones(50, dtype=torch.bool))
    ghost["id"] = slabs.tag_ghosts(torch, ghost["id"], False)
    states[1] = slabs.concat(torch, [states[1], ghost])
    all_pos = np.zeros((n, 4), np.float32)
    for st in states:
        own = st["id"] >= 0
        all_pos[st["id"][own].numpy()] = st["pos"][own].numpy()
    owned, ghosts, sent = slabs.migrate_and_halo(torch, slabs.LocalTransport(), states, bounds, WIDTH)
    assert math.isinf(bounds[0][0]) and math.isinf(bounds[-1][1])
    _check(all_pos, bounds, owned, ghosts, sent)
    t = [torch.tensor([v], dtype=torch.int32) for v in (5, 9, 2)]
    slabs.LocalTransport().allreduce_max_(torch, t)
    assert [int(v) for v in t] == [9, 9, 9]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        rng = np.random.default_rng(7)  # the same global picture on both ranks
        n = 2000
        bounds = slabs.slab_bounds(0.0, 1.0, world)
        start = _state(np.arange(n), rng)
        moved = start["pos"].clone()
        moved[:, 0] += torch.from_numpy(rng.uniform(-0.03, 0.03, n).astype(np.float32))
        x0 = start["pos"][:, 0].numpy()
        lo, hi = bounds[rank]
        mine = torch.from_numpy((x0 >= lo) & (x0 < hi))
        st = slabs.select(dict(start, pos=moved), mine)
        tr = slabs.DistTransport(rank, world)
        owned, ghosts, sent = slabs.migrate_and_halo(torch, tr, [st], [bounds[rank]], WIDTH)
        # gather every rank's result to check the global picture on rank 0
        obj = [None] * world
        dist.all_gather_object(obj, (owned[0], ghosts[0], sent[0]))
        # fixed rows: each rank sends its rank number to both sides
        # to the left 3 rows, to the right 2: a rank receives 2 from its left
        # neighbour and 3 from its right one
        rows = (torch.full((3, 4), float(rank)), torch.full((2, 4), float(rank) + 0.5))
        shapes = [((2, 4) if rank > 0 else (0, 4), (3, 4) if rank + 1 < world else (0, 4))]
        got = tr.exchange_rows(torch, [rows], shapes)[0]
        m = torch.tensor([rank * 10 + 3], dtype=torch.int32)
        tr.allreduce_max_(torch, [m])
        dist.destroy_process_group()
        all_pos = moved.numpy()
        if rank == 0:
            _check(all_pos, bounds, [o[0] for o in obj], [o[1] for o in obj], [o[2] for o in obj])
        if rank > 0:
            assert torch.all(got[0] == rank - 1 + 0.5)  # the left neighbour's right rows
        if rank + 1 < world:
            assert torch.all(got[1] == rank + 1)
        assert int(m) == (world - 1) * 10 + 3
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent
        import traceback
        q.put((rank, traceback.format_exc()))


def test_gloo_two_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert out == {0: "ok", 1: "ok"}, out
