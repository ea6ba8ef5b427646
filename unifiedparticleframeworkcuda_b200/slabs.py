"""One PCISPH scene split into slabs along x, one slab per GPU.

The reference runs one scene on one device (src/cpu/main.cpp:42-53); its
loop test reads the maximum predicted density back every iteration
(GetMaxPredictedDensityCUDA, src/gpu/particles.cu:2139-2154). Here the scene's
x range is cut into slabs [lo, hi); slab k owns the dynamic particles whose x
lies in its range and holds, besides them:

  * ghosts: copies of the neighbouring slabs' particles within `width` (the
    support radius and a margin) of its faces, refreshed every step;
  * the boundary particles within two `width`s of its range (static, set
    once), so that those within one width have complete Akinci volumes.

Each slab is an ordinary upf_system. A step runs the library's phases on
every slab, with exchanges between neighbouring slabs:

  * at the step's start, migration (owned particles that left the range go to
    the neighbour) and then the halo (the new ghosts);
  * after the external forces and after every pressure-force pass, the
    ghosts' predicted positions;
  * after every density pass, the ghosts' correction pressure and p / rho0^2
    (what the pressure-force pass gathers), and the maximum predicted density
    for the loop test, a maximum over all slabs.

Every owned particle then sees all of its neighbours with their owners'
values, in the Morton order of the particles present, which is the unsplit
scene's order: a slab run equals the unsplit run. A ghost's own density,
forces and integration come from an incomplete neighbourhood and are thrown
away (overwritten by the exchanges, or dropped at the next step); its partial
density is never above its full one (every term is non-negative), so the
maximum over all slabs is the unsplit maximum. Two particles with equal
Morton keys may be ordered differently (the unsplit run keeps their previous
order, a slab the order they arrived in).

Transports: LocalTransport passes buffers between slabs of one process
(several slabs on one GPU, the way the split is checked on a single device);
DistTransport uses torch.distributed point-to-point calls with the
neighbouring ranks and an all-reduce (NCCL between GPUs; gloo on CPU for the
bookkeeping). Particles keep their global input index as id; bit 31 marks a
ghost and bit 30 a ghost from the right neighbour, so a scene holds at most
2^30 particles.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

GHOST = 1 << 31
FROM_RIGHT = 1 << 30
ID_MASK = FROM_RIGHT - 1
FIELDS = ("pos", "vel", "lag", "type", "id")


# ---------------------------------------------------------------- device views
class _DeviceView:
    """A device array of the library seen by torch without a copy (CUDA array
    interface)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_tensor(torch, ptr, shape, dtype, device):
    if any(d == 0 for d in shape):
        return torch.empty(shape, dtype=dtype, device=device)
    typestr = {torch.float32: "<f4", torch.int32: "<i4"}[dtype]
    return torch.as_tensor(_DeviceView(ptr, shape, typestr), device=device)


# ---------------------------------------------------------------- bookkeeping
def slab_bounds(x_min: float, x_max: float, nslabs: int):
    """Equal slabs of [x_min, x_max); the outer faces open to infinity, so
    that every particle has an owner."""
    edges = [x_min + (x_max - x_min) * k / nslabs for k in range(nslabs + 1)]
    edges[0], edges[-1] = -math.inf, math.inf
    return [(edges[k], edges[k + 1]) for k in range(nslabs)]


def select(state: dict, mask):
    return {k: v[mask] for k, v in state.items()}


def by_id(torch, state: dict):
    order = torch.argsort(state["id"])
    return {k: v[order] for k, v in state.items()}


def concat(torch, parts):
    parts = [p for p in parts if p is not None]
    return {k: torch.cat([p[k] for p in parts]) for k in FIELDS}


def tag_ghosts(torch, ids, from_right: bool):
    """Ghost ids: bit 31 set (negative as int32), bit 30 when the ghost comes
    from the receiver's right neighbour."""
    t = ids.to(torch.int64) | GHOST | (FROM_RIGHT if from_right else 0)
    return (t - (1 << 32)).to(torch.int32)


def untag(torch, ids):
    return (ids.to(torch.int64) & ID_MASK).to(torch.int32)


def is_from_right(torch, ids):
    return (ids.to(torch.int64) & FROM_RIGHT) != 0


def migrate_and_halo(torch, transport, states, bounds, width):
    """Step-start bookkeeping of the local slabs: drop the ghosts, send the
    owned particles that left their slab to the neighbour, then send each
    neighbour, as its ghosts, the owned particles within `width` of the face
    they share (ordered by global id).

    states[k]: dict of pos (n,4) float32, vel, lag (n,4), type (n,) int32 and
    id (n,) int32 of local slab k, owned particles and ghosts; bounds[k] =
    (lo, hi). Returns per slab (owned, ghosts, (ids sent left, ids sent
    right)); the sent ids are ascending, as the ghosts arrive."""
    owned, sends = [], []
    for st, (lo, hi) in zip(states, bounds):
        mine = select(st, st["id"] >= 0)
        x = mine["pos"][:, 0]
        left, right = x < lo, x >= hi
        owned.append(select(mine, ~(left | right)))
        sends.append((select(mine, left), select(mine, right)))
    recv = transport.exchange(torch, sends)
    halos, sent_ids = [], []
    for k, ((from_left, from_right), (lo, hi)) in enumerate(zip(recv, bounds)):
        o = concat(torch, [owned[k], from_left, from_right])
        owned[k] = o
        x = o["pos"][:, 0]
        to_left = by_id(torch, select(o, x < lo + width))
        to_right = by_id(torch, select(o, x >= hi - width))
        sent_ids.append((to_left["id"].clone(), to_right["id"].clone()))
        # the left neighbour receives to_left from its right, and vice versa
        to_left["id"] = tag_ghosts(torch, to_left["id"], True)
        to_right["id"] = tag_ghosts(torch, to_right["id"], False)
        halos.append((to_left, to_right))
    recv = transport.exchange(torch, halos)
    ghosts = [concat(torch, [fl, fr]) if (fl is not None or fr is not None) else None for fl, fr in recv]
    return owned, ghosts, sent_ids


class LocalTransport:
    """Several slabs of one process: buffers pass by reference, the maximum
    is taken over the list."""

    def exchange(self, torch, sends):
        """sends[k] = (to_left, to_right) of local slab k (dicts of tensors);
        returns [(from_left, from_right)] per slab (None at the outer faces)."""
        n = len(sends)
        return [(sends[k - 1][1] if k > 0 else None, sends[k + 1][0] if k + 1 < n else None) for k in range(n)]

    def exchange_rows(self, torch, sends, recv_shapes):
        return self.exchange(torch, sends)

    def allreduce_max_(self, torch, tensors):
        m = torch.stack([t.view(torch.int32) for t in tensors]).max(0).values
        for t in tensors:
            t.view(torch.int32).copy_(m)


class DistTransport:
    """One slab per rank of a torch.distributed group: payload sizes first,
    then the payload, with ranks rank - 1 and rank + 1; the maximum by an
    all-reduce (positive float bits order as int32)."""

    SHAPES = {"pos": (4,), "vel": (4,), "lag": (4,), "type": (), "id": ()}

    def __init__(self, rank: int, world: int, group=None):
        self.rank, self.world, self.group = rank, world, group

    def _peers(self, to_left, to_right):
        return [(p, s) for p, s in ((self.rank - 1, to_left), (self.rank + 1, to_right)) if 0 <= p < self.world]

    @staticmethod
    def _run(ops):
        import torch.distributed as dist
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def exchange(self, torch, sends):
        import torch.distributed as dist
        (to_left, to_right), = sends
        dev = (to_left or to_right)["id"].device
        peers = self._peers(to_left, to_right)
        ops, sizes = [], {}
        for peer, payload in peers:
            n = torch.tensor([payload["id"].shape[0]], dtype=torch.int64, device=dev)
            sizes[peer] = torch.empty(1, dtype=torch.int64, device=dev)
            ops += [dist.P2POp(dist.isend, n, peer, self.group), dist.P2POp(dist.irecv, sizes[peer], peer, self.group)]
        self._run(ops)
        ops, out = [], {}
        for peer, payload in peers:
            m = int(sizes[peer].item())
            out[peer] = {k: torch.empty((m,) + self.SHAPES[k], dtype=payload[k].dtype, device=dev) for k in FIELDS}
            for k in FIELDS:
                if payload[k].shape[0]:
                    ops.append(dist.P2POp(dist.isend, payload[k].contiguous(), peer, self.group))
                if m:
                    ops.append(dist.P2POp(dist.irecv, out[peer][k], peer, self.group))
        self._run(ops)
        return [(out.get(self.rank - 1), out.get(self.rank + 1))]

    def exchange_rows(self, torch, sends, recv_shapes):
        """Fixed-size rows whose counts both sides know (the halo of this
        step): sends = [(to_left, to_right)], recv_shapes = [(left, right)]."""
        import torch.distributed as dist
        (to_left, to_right), = sends
        (shape_l, shape_r), = recv_shapes
        ops, out = [], {}
        for peer, payload, shape in ((self.rank - 1, to_left, shape_l), (self.rank + 1, to_right, shape_r)):
            if not (0 <= peer < self.world):
                continue
            out[peer] = torch.empty(shape, dtype=payload.dtype, device=payload.device)
            if payload.numel():
                ops.append(dist.P2POp(dist.isend, payload, peer, self.group))
            if out[peer].numel():
                ops.append(dist.P2POp(dist.irecv, out[peer], peer, self.group))
        self._run(ops)
        return [(out.get(self.rank - 1), out.get(self.rank + 1))]

    def allreduce_max_(self, torch, tensors):
        import torch.distributed as dist
        (t,) = tensors
        dist.all_reduce(t.view(torch.int32), op=dist.ReduceOp.MAX, group=self.group)


# ---------------------------------------------------------------- the scene
class SlabScene:
    """A PCISPH scene (liquid and static boundary particles) split into
    `nslabs` slabs along x; this process runs the slabs `local` (all of them
    with a LocalTransport, its own rank's with a DistTransport)."""

    def __init__(self, scene, nslabs: int, transport, local=None, device: int = 0, x_range=None,
                 width_factor: float = 1.001, capacity_factor: float = 1.6):
        import torch

        import unifiedparticleframeworkcuda_b200 as upf

        self.torch, self.upf = torch, upf
        p = upf.derive_params(scene.params)
        if p.method != upf.METHOD_PCISPH:
            raise ValueError("slabs: PCISPH scenes only")
        if scene.n >= (1 << 30):
            raise ValueError("slabs: at most 2^30 particles")
        typ = np.asarray(scene.type, np.int32)
        if np.any((typ != upf.FROZEN) & (typ != upf.LIQUID)):
            raise ValueError("slabs: liquid and boundary particles only")
        self.params = p
        self.width = float(p.support_radius) * width_factor
        pos = np.ascontiguousarray(scene.pos, np.float32)
        vel = np.ascontiguousarray(scene.vel, np.float32)
        dyn = typ != upf.FROZEN
        if x_range is None:
            x_range = (float(pos[dyn, 0].min()), float(pos[dyn, 0].max()))
        self.bounds_all = slab_bounds(x_range[0], x_range[1], nslabs)
        self.local = list(range(nslabs)) if local is None else list(local)
        self.bounds = [self.bounds_all[k] for k in self.local]
        self.transport = transport
        self.dev = torch.device("cuda", device)
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        self.systems = []
        x = pos[:, 0]
        for lo, hi in self.bounds:
            own = dyn & (x >= lo) & (x < hi)
            # boundary particles within two widths: those within one width
            # (the neighbours of owned particles and ghosts) then have their
            # complete boundary neighbourhood for the Akinci volume
            bnd = (~dyn) & (x >= lo - 2 * self.width) & (x < hi + 2 * self.width)
            near = dyn & (x >= lo - self.width) & (x < hi + self.width)
            # room for the owned particles growing by migration, and the ghosts
            cap = int(capacity_factor * near.sum()) + int(bnd.sum()) + 1024
            s = upf.ParticleSystem(p, capacity=min(cap, scene.n + 1024), device=device, derive=False)
            s.set_stream(stream)
            sel = np.flatnonzero(own | bnd)
            s.set_particles(pos[sel], vel[sel], typ[sel])
            o = np.flatnonzero(own)
            st = {"pos": torch.from_numpy(pos[o]).to(self.dev), "vel": torch.from_numpy(vel[o]).to(self.dev),
                  "lag": torch.tensor([0.0, 0.0, float(p.rest_density), 0.0], device=self.dev).repeat(len(o), 1),
                  "type": torch.from_numpy(typ[o]).to(self.dev), "id": torch.from_numpy(o.astype(np.int32)).to(self.dev)}
            self._set_dynamic(s, st)
            self.systems.append(s)
        torch.cuda.current_stream(self.dev).synchronize()
        self.iterations = []

    # ---- library access
    def _state(self, s):
        d = self.upf.UpfDeviceState()
        self.upf.check(self.upf.lib().upf_get_device_state(s.handle, C.byref(d)), "upf_get_device_state")
        return d

    def _dynamic(self, s):
        torch = self.torch
        d = self._state(s)
        n = d.n
        t = lambda ptr, shape, dt: device_tensor(torch, ptr, shape, dt, self.dev)  # noqa: E731
        return {"pos": t(d.pos4, (n, 4), torch.float32), "vel": t(d.vel4, (n, 4), torch.float32),
                "lag": t(d.lag4, (n, 4), torch.float32), "type": t(d.type, (n,), torch.int32),
                "id": t(d.id, (n,), torch.int32)}

    def _set_dynamic(self, s, st):
        c = {k: v.contiguous() for k, v in st.items()}
        n = int(c["id"].shape[0])
        ptr = lambda t, ct: C.cast(t.data_ptr(), C.POINTER(ct))  # noqa: E731
        self.upf.check(self.upf.lib().upf_set_dynamic_device(
            s.handle, ptr(c["pos"], C.c_float), ptr(c["vel"], C.c_float), ptr(c["lag"], C.c_float),
            ptr(c["type"], C.c_int32), ptr(c["id"], C.c_uint32), n), "upf_set_dynamic_device")
        s.n_dynamic = n
        return c  # the sources of the stream-ordered copies

    def _rows(self, src, row_bytes, idx, dst, scatter, stream):
        L = self.upf.lib()
        f = L.upf_scatter_rows if scatter else L.upf_gather_rows
        self.upf.check(f(C.c_void_p(src), row_bytes, C.c_void_p(idx.data_ptr()), idx.numel(), C.c_void_p(dst),
                         C.c_void_p(stream)), "upf_scatter_rows" if scatter else "upf_gather_rows")

    def _maps(self, s, sent_ids):
        """After the sort: the rows of the ghosts from each side and of the
        owned particles sent to each side, both in ascending global id."""
        torch = self.torch
        d = self._state(s)
        sid = device_tensor(torch, d.sorted_id, (d.n,), torch.int32, self.dev)
        rows = torch.arange(d.n, device=self.dev, dtype=torch.int32)
        ghost = sid < 0
        gid = untag(torch, sid)
        fr = is_from_right(torch, sid)
        out = {"state": d}
        for name, m in (("ghost_left", ghost & ~fr), ("ghost_right", ghost & fr)):
            out[name] = rows[m][torch.argsort(gid[m])].contiguous()
        own_ids, own_rows = gid[~ghost], rows[~ghost]
        order = torch.argsort(own_ids)
        own_ids, own_rows = own_ids[order], own_rows[order]
        for name, ids in (("halo_left", sent_ids[0]), ("halo_right", sent_ids[1])):
            out[name] = own_rows[torch.searchsorted(own_ids, ids)].contiguous() if ids.numel() else \
                torch.empty(0, dtype=torch.int32, device=self.dev)
        return out

    def _exchange_field(self, field, row_bytes, maps):
        """The owners' values of `field` (a upf_device_state array) at their
        halo rows into the neighbours' ghost rows."""
        torch = self.torch
        words = row_bytes // 4
        sends, shapes = [], []
        for m in maps:
            d = m["state"]
            bufs = []
            for side in ("halo_left", "halo_right"):
                idx = m[side]
                buf = torch.empty((idx.numel(), words), dtype=torch.float32, device=self.dev)
                if idx.numel():
                    self._rows(getattr(d, field), row_bytes, idx, buf.data_ptr(), False, d.stream)
                bufs.append(buf)
            sends.append(tuple(bufs))
            shapes.append(((m["ghost_left"].numel(), words), (m["ghost_right"].numel(), words)))
        recv = self.transport.exchange_rows(torch, sends, shapes)
        for m, (from_left, from_right) in zip(maps, recv):
            d = m["state"]
            for buf, side in ((from_left, "ghost_left"), (from_right, "ghost_right")):
                idx = m[side]
                if idx.numel() == 0:
                    continue
                if buf is None or buf.shape[0] != idx.numel():
                    raise RuntimeError("halo sizes disagree on %s: %s values for %d ghosts"
                                       % (side, None if buf is None else buf.shape[0], idx.numel()))
                self._rows(buf.data_ptr(), row_bytes, idx, getattr(d, field), True, d.stream)

    # ---- one step
    def step(self):
        """One PCISPH step of the whole scene; returns its iteration count."""
        torch, upf = self.torch, self.upf
        L = upf.lib()
        states = [self._dynamic(s) for s in self.systems]
        owned, ghosts, sent_ids = migrate_and_halo(torch, self.transport, states, self.bounds, self.width)
        sources = [self._set_dynamic(s, concat(torch, [o, g])) for s, o, g in zip(self.systems, owned, ghosts)]
        maps = []
        for s, ids in zip(self.systems, sent_ids):
            s.phase("sort")
            s.phase("neighbors")
            maps.append(self._maps(s, ids))
        for s in self.systems:
            s.phase("forces")
        self._exchange_field("predicted_pos4", 16, maps)
        for s in self.systems:
            upf.check(L.upf_phase_loop_begin(s.handle), "upf_phase_loop_begin")
        it = 0
        while True:
            for s in self.systems:
                upf.check(L.upf_phase_density(s.handle), "upf_phase_density")
            self._exchange_field("pressure", 4, maps)
            self._exchange_field("pq4", 16, maps)
            self.transport.allreduce_max_(torch, [device_tensor(torch, m["state"].loop_max_density_bits, (1,),
                                                                torch.int32, self.dev) for m in maps])
            for s in self.systems:
                upf.check(L.upf_phase_pressure_force(s.handle), "upf_phase_pressure_force")
            self._exchange_field("predicted_pos4", 16, maps)
            conts = []
            for s in self.systems:
                c = C.c_int32()
                upf.check(L.upf_phase_loop_control(s.handle, C.byref(c)), "upf_phase_loop_control")
                conts.append(c.value)
            it += 1
            if len(set(conts)) != 1:
                raise RuntimeError("local slabs disagree on the loop test: %s" % conts)
            if not conts[0]:
                break
        for s in self.systems:
            s.phase("integrate")
        torch.cuda.current_stream(self.dev).synchronize()
        del sources
        self.iterations.append(it)
        return it

    # ---- readback
    def particles(self):
        """Owned dynamic particles of the local slabs (numpy, by global id)."""
        parts = []
        for s in self.systems:
            st = self._dynamic(s)
            own = st["id"] >= 0
            parts.append({k: v[own].cpu().numpy() for k, v in st.items()})
        out = {k: np.concatenate([p[k] for p in parts]) for k in FIELDS}
        order = np.argsort(out["id"])
        return {k: v[order] for k, v in out.items()}

    def close(self):
        for s in self.systems:
            s.close()
        self.systems = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
