"""The benchmark workloads at full size against the CPU oracle.

  * pcisph_dam_break_1M (128 x 128 x 64 = 1,048,576 fluid + 279,308
    boundary particles): Morton keys, sort order, cell ranges and every
    neighbour list bit-exact; one step with an equal iteration count and
    every field within 1e-5 relative of its scale (the small-scene bars);
  * rigid_fluid_granular_coupling_524k (524,288 fluid, 131,072 grains, 16
    bodies): one step with an equal iteration count; particle fields, forces
    and body states within 1e-5 relative of their scales;
  * batched_scenes_256: scenes of the full batch equal the same scenes run
    alone, bit for bit, and the largest agrees with the oracle;
  * wcsph_dam_break_32k: one step at the specified dt within 1e-5 of the
    oracle, 20 steps at the timed dt on kinetic energy and momentum;
  * adjoint_pcisph at 65,536 particles over 20 steps: loss and gradients
    against the FP64 oracle adjoint.

The oracle runs its OpenMP restatement on all host cores: a few seconds per
step at these sizes."""
import numpy as np
import pytest

from test_gpu_coupling import compare_bodies, compare_forces, compare_particles
from test_gpu_parity import RTOL, _compare_step
from unifiedparticleframeworkcuda_b200 import FROZEN, scenes

pytestmark = pytest.mark.gpu


def _make(upf, oracle, sc, bodies=False):
    p = upf.derive_params(sc.params)
    sysm = upf.ParticleSystem(p, capacity=sc.n, derive=False)
    sysm.set_particles(sc.pos, sc.vel, sc.type)
    o = oracle.OracleSim(p, sc.pos, sc.vel, sc.type)
    if bodies:
        sysm.set_rigid_bodies(sc.body, sc.num_bodies)
        o.set_rigid_bodies(sc.body, sc.num_bodies)
    return p, sysm, o


def test_full_size_keys_cells_and_lists_bit_exact(upf_lib, oracle_lib):
    sc = scenes.pcisph_dam()
    assert int(np.count_nonzero(sc.type != FROZEN)) == 1 << 20
    p, sysm, o = _make(upf_lib, oracle_lib, sc)
    sysm.phase("sort")
    keys, ids = sysm.sorted_keys()
    st = o.state()
    dyn = st["type"] != FROZEN
    assert np.array_equal(ids, st["id"][dyn]), "sort order differs"
    assert np.array_equal(keys, st["key"][dyn]), "Morton keys differ"
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)

    start, end = sysm.cell_ranges()
    bs3 = int(p.search_cell) ** 3
    k = st["key"][dyn].astype(np.int64)
    occupied = np.unique(k // bs3)
    assert np.array_equal(start[occupied], np.searchsorted(k, occupied * bs3, side="left"))
    assert np.array_equal(end[occupied], np.searchsorted(k, (occupied + 1) * bs3, side="left"))
    empty = np.ones(start.shape[0], bool)
    empty[occupied] = False
    assert not start[empty].any() and not end[empty].any()

    sysm.phase("neighbors")
    counts, lists = sysm.neighbors()
    off, nb = o.neighbors()
    # the oracle's row of each sorted particle
    row = np.full(int(st["id"].max()) + 1, -1, np.int64)
    row[st["id"]] = np.arange(st["id"].shape[0])
    r = row[ids]
    assert (r >= 0).all()
    counts = counts.astype(np.int64)
    want_counts = (off[r + 1] - off[r]).astype(np.int64)
    bad = np.flatnonzero(counts != want_counts)
    assert bad.size == 0, "neighbour counts differ at %d particles, first id %d" % (bad.size, ids[bad[0]])
    total = int(counts.sum())
    assert total > 20 * counts.shape[0]  # 28.6 entries per fluid particle on average
    got = lists[np.arange(lists.shape[1])[None, :] < counts[:, None]].astype(np.int64)
    first = np.cumsum(counts) - counts
    want = np.asarray(nb, np.int64)[np.arange(total) + np.repeat(off[r] - first, counts)]
    diff = np.flatnonzero(got != want)
    assert diff.size == 0, "neighbour entries differ: %d of %d, first in the list of id %d" % (
        diff.size, total, ids[np.searchsorted(first, diff[0], side="right") - 1])
    sysm.close()
    o.close()


def test_full_size_pcisph_step(upf_lib, oracle_lib):
    sc = scenes.pcisph_dam()
    p, sysm, o = _make(upf_lib, oracle_lib, sc)
    sysm.step(1)
    stats = sysm.stats()
    info = o.step()
    assert stats.iterations == info.iterations
    assert abs(stats.max_predicted_density - info.max_predicted_density) <= RTOL * info.max_predicted_density
    res = _compare_step(sysm, o, "pcisph")
    bad = {k: v for k, v in res.items() if not v[0]}
    assert not bad, "fields beyond %g relative: %s" % (RTOL, bad)
    sysm.close()
    o.close()


def test_full_size_staged_modes_equal_the_default_shape(upf_lib):
    """pcisph_dam_break_1M, three steps from rest (every iteration of the
    loop, 150 launches of each pass): the staged-neighbourhood passes (mode 2,
    both batch sizes) give results identical to the default shapes, which the
    step test above holds to the oracle."""
    from unifiedparticleframeworkcuda_b200 import UpfLaunchConfig
    sc = scenes.pcisph_dam()
    p = upf_lib.derive_params(sc.params)
    out = []
    for rows in (0, 4, 8):
        with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
            s.set_particles(sc.pos, sc.vel, sc.type)
            if rows:
                c = s.launch_config()
                c.density_mode, c.density_threads, c.density_rows = 2, 256, rows
                c.pforce_mode, c.pforce_threads, c.pforce_rows = 2, 256, rows
                s.set_launch_config(c)
            s.step(3)
            g = s.particles()
            o = np.argsort(g["id"], kind="stable")
            out.append(({k: g[k][o] for k in ("pos", "vel", "density", "pressure")}, s.stats().iterations))
    ref, it = out[0]
    for got, it2 in out[1:]:
        assert it2 == it
        for f in ref:
            assert np.array_equal(got[f], ref[f]), f


def test_full_size_coupling_step(upf_lib, oracle_lib):
    sc = scenes.coupling_scene()
    assert sc.num_bodies == 16
    p, sysm, o = _make(upf_lib, oracle_lib, sc, bodies=True)
    sysm.step(1)
    stats = sysm.stats()
    info = o.step()
    assert stats.iterations == info.iterations
    res = {}
    res.update(compare_particles(sysm, o))
    res.update(compare_forces(sysm, o))
    res.update(compare_bodies(sysm, o))
    bad = {k: v for k, v in res.items() if not v[0]}
    assert not bad, "beyond %g relative: %s" % (RTOL, bad)
    sysm.close()
    o.close()


def test_full_size_batch_scenes_equal_single_runs(upf_lib, oracle_lib):
    """batched_scenes_256: all 256 scenes (counts log-uniform in [2048,
    65536], about 4.7 M particles) step together; the smallest, the largest
    and four seeded picks equal the same scenes run alone bit for bit, and
    the largest agrees with the oracle after one step."""
    from test_gpu_batch import run_single

    scs = scenes.batch_scenes(256, seed=2024)
    sizes = np.array([sc.n for sc in scs])
    assert sizes.sum() > 4_000_000
    picks = sorted({int(sizes.argmin()), int(sizes.argmax())}
                   | set(np.random.default_rng(5).choice(len(scs), 4, replace=False).tolist()))
    steps = 2
    with upf_lib.ParticleBatch.from_scenes(scs) as b:
        iters = []
        for _ in range(steps):
            b.step(1)
            iters.append([st.iterations for st in b.stats()])
        stats = b.stats()
        got = {k: b.particles(k) for k in picks}
    for k in picks:
        want, want_iters, want_st = run_single(upf_lib, scs[k], steps)
        g = {f: v[np.argsort(got[k]["id"], kind="stable")] for f, v in got[k].items()}
        assert [it[k] for it in iters] == want_iters, "scene %d iterations" % k
        for f in ("id", "pos", "vel", "density", "pressure"):
            assert np.array_equal(g[f], want[f]), "scene %d field %s" % (k, f)
        assert stats[k].max_predicted_density == want_st.max_predicted_density

    big = scs[int(sizes.argmax())]
    p, sysm, o = _make(upf_lib, oracle_lib, big)
    sysm.step(1)
    info = o.step()
    assert sysm.stats().iterations == info.iterations
    res = _compare_step(sysm, o, "pcisph")
    bad = {k: v for k, v in res.items() if not v[0]}
    assert not bad, "fields beyond %g relative: %s" % (RTOL, bad)
    sysm.close()
    o.close()


def test_full_size_wcsph_dam(upf_lib, oracle_lib):
    """wcsph_dam_break_32k (32,768 fluid + 15,002 boundary particles): one
    step at the specified dt = 1e-3 within 1e-5 of the oracle; then 20 steps
    at the timed dt = 5e-4 (the specified step diverges within 12 steps in
    both), compared on kinetic energy and momentum within 1e-3."""
    sc = scenes.wcsph_dam(32)
    assert sc.n_fluid == 32_768
    p, sysm, o = _make(upf_lib, oracle_lib, sc)
    sysm.step(1)
    sysm.synchronize()
    o.step()
    res = _compare_step(sysm, o, "wcsph")
    bad = {k: v for k, v in res.items() if not v[0]}
    assert not bad, "fields beyond %g relative: %s" % (RTOL, bad)
    sysm.close()
    o.close()

    sc.params.dt = 5e-4
    p, sysm, o = _make(upf_lib, oracle_lib, sc)
    for s in range(20):
        sysm.step(1)
        g = sysm.stats()
        c = o.step()
        assert abs(g.kinetic_energy - c.kinetic_energy) <= 1e-3 * c.kinetic_energy, s
        mg = np.array(g.momentum[:])
        mc = np.array(c.momentum[:])
        assert np.abs(mg - mc).max() <= 1e-3 * np.abs(mc).max(), s
    sysm.close()
    o.close()


def test_full_size_adjoint_particle_count(upf_lib, oracle_lib):
    """adjoint_pcisph at its full particle count (32 x 32 x 64 = 65,536) over
    20 steps, checkpoints every 5: the loss within 1e-4 and the gradients
    (initial velocities, L2; viscosity) within 1e-3 of the FP64 oracle
    adjoint. The trajectory length itself is covered by the small test of
    checkpoint intervals, which shows that gradients do not depend on them."""
    sc = scenes.adjoint_scene(32, 32, 64)
    assert sc.n == 65_536
    p = upf_lib.derive_params(sc.params)
    tgt = sc.pos[:, :3].astype(np.float64).mean(0) + np.array([0.1, 0.0, 0.0])
    with upf_lib.Adjoint(p, sc.pos, sc.vel, 20, checkpoint_interval=5, loop_iterations=3, target=tgt,
                         com_weight=1.0, density_weight=1e-6, derive=False) as a:
        loss = a.forward()
        gv, gm = a.backward()
    x = sc.pos[:, :3].astype(np.float64)
    v = sc.vel[:, :3].astype(np.float64)
    L64, gv64, gm64 = oracle_lib.adjoint_run(p, x, v, viscosity=p.viscosity, steps=20, iterations=3, target=tgt,
                                             com_weight=1.0, density_weight=1e-6)
    assert abs(loss - L64) <= 1e-4 * abs(L64)
    assert np.linalg.norm(gv - gv64) <= 1e-3 * np.linalg.norm(gv64)
    assert abs(gm - gm64) <= 1e-3 * abs(gm64)
