"""Edge cases of the step against the CPU oracle, with the bars of the
small-scene parity tests: Morton keys, sort order and neighbour lists
bit-exact; one step with an equal iteration count and every field within
1e-5 relative of its scale.

  * coincident particles: copies at the same positions share a Morton key
    (the order among equal keys is the stable one) and form pairs at zero
    distance;
  * particles outside the Morton grid: their keys are clamped to the grid's
    edge, as the reference's table lookup is;
  * ragged sizes: one fluid particle, and 2, 31 and 33 (partial warps);
  * no fluid at all: boundary particles only; the step runs and nothing
    changes.
"""
import numpy as np
import pytest

from test_gpu_parity import RTOL, _compare_step
from unifiedparticleframeworkcuda_b200 import FROZEN, LIQUID, scenes

pytestmark = pytest.mark.gpu


def _with(sc, pos, vel, typ):
    return scenes.Scene(sc.name, sc.params, np.ascontiguousarray(pos, np.float32),
                        np.ascontiguousarray(vel, np.float32), np.ascontiguousarray(typ, np.int32))


def _check(upf, oracle, sc):
    p = upf.derive_params(sc.params)
    with upf.ParticleSystem(p, capacity=sc.n, derive=False) as sysm:
        sysm.set_particles(sc.pos, sc.vel, sc.type)
        o = oracle.OracleSim(p, sc.pos, sc.vel, sc.type)
        try:
            sysm.phase("sort")
            sysm.phase("neighbors")
            keys, ids = sysm.sorted_keys()
            st = o.state()
            dyn = st["type"] != FROZEN
            assert np.array_equal(ids, st["id"][dyn]), "sort order differs"
            assert np.array_equal(keys, st["key"][dyn]), "Morton keys differ"
            counts, lists = sysm.neighbors()
            off, nb = o.neighbors()
            row = {int(i): k for k, i in enumerate(st["id"])}
            for r, pid in enumerate(ids):
                k = row[int(pid)]
                assert np.array_equal(lists[r, :counts[r]], nb[off[k]:off[k + 1]]), "list of particle %d" % pid
            sysm.step(1)
            stats = sysm.stats()
            info = o.step()
            assert stats.iterations == info.iterations
            res = _compare_step(sysm, o, "pcisph")
            bad = {k: v for k, v in res.items() if not v[0]}
            assert not bad, "fields beyond %g relative: %s" % (RTOL, bad)
            return keys, counts
        finally:
            o.close()


def test_coincident_particles(upf_lib, oracle_lib):
    sc = scenes.small_pcisph()
    liq = np.flatnonzero(sc.type == LIQUID)
    pick = np.random.default_rng(3).choice(liq, 40, replace=False)
    pos = np.concatenate([sc.pos, sc.pos[pick]])
    vel = np.concatenate([sc.vel, np.zeros_like(sc.pos[pick])])
    typ = np.concatenate([sc.type, sc.type[pick]])
    keys, counts = _check(upf_lib, oracle_lib, _with(sc, pos, vel, typ))
    assert np.count_nonzero(np.diff(keys.astype(np.int64)) == 0) >= 40  # equal keys present


def test_particles_outside_the_key_grid(upf_lib, oracle_lib):
    sc = scenes.small_pcisph()
    p = sc.params
    org = np.array(p.zindex_origin[:], np.float32)
    ext = np.array(p.zindex_extent[:], np.float32)
    liq = np.flatnonzero(sc.type == LIQUID)
    pos = sc.pos.copy()
    rng = np.random.default_rng(4)
    low = rng.choice(liq, 10, replace=False)
    high = rng.choice(np.setdiff1d(liq, low), 10, replace=False)
    # below the grid's origin on one axis each, and beyond its far end
    for k, i in enumerate(low):
        pos[i, k % 3] = org[k % 3] - 0.01 * (1 + k)
    for k, i in enumerate(high):
        pos[i, k % 3] = org[k % 3] + ext[k % 3] * 1.05 + 0.01 * k
    keys, _ = _check(upf_lib, oracle_lib, _with(sc, pos, sc.vel, sc.type))
    assert keys.max() > 0


@pytest.mark.parametrize("n_fluid", [1, 2, 31, 33])
def test_ragged_fluid_counts(upf_lib, oracle_lib, n_fluid):
    sc = scenes.small_pcisph()
    liq = np.flatnonzero(sc.type == LIQUID)
    keep = np.concatenate([liq[:n_fluid], np.flatnonzero(sc.type == FROZEN)])
    _check(upf_lib, oracle_lib, _with(sc, sc.pos[keep], sc.vel[keep], sc.type[keep]))


def test_boundary_only_scene(upf_lib):
    sc = scenes.small_pcisph()
    b = sc.type == FROZEN
    p = upf_lib.derive_params(sc.params)
    with upf_lib.ParticleSystem(p, capacity=int(b.sum()), derive=False) as sysm:
        sysm.set_particles(sc.pos[b], sc.vel[b], sc.type[b])
        sysm.step(3)
        g = sysm.particles()
        assert g["id"].shape[0] == 0
        assert sysm.stats().iterations >= 0


def test_phase_entry_points_repeat_and_compose(upf_lib):
    """The sort phase can be called again, and a step after the sort and
    list phases equals a step alone bit for bit: a repeated sort finds the
    state in order and changes nothing, as re-sorting sorted arrays does in
    the reference."""
    sc = scenes.small_pcisph()
    p = upf_lib.derive_params(sc.params)
    out = []
    for phases in ((), ("sort",), ("sort", "sort", "neighbors", "sort")):
        with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
            s.set_particles(sc.pos, sc.vel, sc.type)
            for ph in phases:
                s.phase(ph)
            s.step(2)
            g = s.particles()
            o = np.argsort(g["id"], kind="stable")
            out.append({k: v[o] for k, v in g.items()})
    for got in out[1:]:
        for f in ("id", "pos", "vel", "density", "pressure"):
            assert np.array_equal(got[f], out[0][f]), f


def test_phases_in_order_make_one_step(upf_lib):
    """sort, neighbors, forces, predict_correct and integrate, called in
    order, advance the state exactly as one graph-launched step does."""
    sc = scenes.small_pcisph()
    p = upf_lib.derive_params(sc.params)
    out = []
    for by_phase in (False, True):
        with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
            s.set_particles(sc.pos, sc.vel, sc.type)
            iters = []
            for _ in range(2):
                if by_phase:
                    for ph in ("sort", "neighbors", "forces", "predict_correct", "integrate"):
                        s.phase(ph)
                else:
                    s.step(1)
                iters.append(s.stats().iterations)
            g = s.particles()
            o = np.argsort(g["id"], kind="stable")
            out.append(({k: v[o] for k, v in g.items()}, iters))
    (a, ia), (b, ib) = out
    assert ia == ib
    for f in ("id", "pos", "vel", "density", "pressure"):
        assert np.array_equal(a[f], b[f]), f
