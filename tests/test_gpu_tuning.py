"""Launch shapes and the autotuner: every shape of every tunable pass must
give the same results bit for bit (shapes change timing only), the tuner
must leave the simulation state as it found it, and invalid shapes are
rejected."""
import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import UpfError, UpfLaunchConfig, scenes

pytestmark = pytest.mark.gpu

# (mode, threads, rows) with the TMA ring (mode 0), direct loads (mode 1) and
# staged neighbourhoods (mode 2, single scenes)
LOOP_PAIRS = [(0, 128, 4), (0, 128, 8), (0, 128, 16), (0, 256, 2), (0, 256, 4), (0, 256, 8), (0, 512, 2),
              (0, 512, 4), (0, 1024, 2), (1, 128, 4), (1, 128, 8), (1, 256, 4), (1, 256, 8), (1, 512, 4),
              (1, 512, 8), (2, 256, 4), (2, 256, 8)]
# the pressure-force pass also streams a 32-bit value per list entry: its
# larger TMA rings do not fit in static shared memory and are not built
PFORCE_PAIRS = [p for p in LOOP_PAIRS if p[0] != 0 or p[1:] in ((128, 4), (128, 8), (256, 2), (256, 4), (512, 2))]
STAGED = [p for p in LOOP_PAIRS if p[0] == 2]


def shape(nl, ext, dens, pf):
    """dens, pf: (threads, rows) for the TMA ring or (mode, threads, rows)."""
    dens = dens if len(dens) == 3 else (0,) + tuple(dens)
    pf = pf if len(pf) == 3 else (0,) + tuple(pf)
    c = UpfLaunchConfig()
    c.nlist_threads, c.external_threads = nl, ext
    c.density_mode, c.density_threads, c.density_rows = dens
    c.pforce_mode, c.pforce_threads, c.pforce_rows = pf
    return c


def run(upf, sc, cfg, steps=3, tune=False):
    p = upf.derive_params(sc.params)
    s = upf.ParticleSystem(p, capacity=sc.n, derive=False)
    s.set_particles(sc.pos, sc.vel, sc.type)
    if cfg is not None:
        s.set_launch_config(cfg)
    chosen = None
    s.step(1)
    if tune:
        chosen = s.autotune(repeats=2)
    s.step(steps - 1)
    g = s.particles()
    st = s.stats()
    s.close()
    o = np.argsort(g["id"], kind="stable")
    return {k: v[o] for k, v in g.items()}, st, chosen


def test_every_shape_gives_identical_results(upf_lib):
    sc = scenes.small_pcisph()
    ref, ref_st, _ = run(upf_lib, sc, None)
    nls = [64, 128, 256]
    exts = [128, 256]
    for k, dens in enumerate(LOOP_PAIRS):
        pf = PFORCE_PAIRS[(k + 2) % len(PFORCE_PAIRS)]
        cfg = shape(nls[k % 3], exts[k % 2], dens, pf)
        cfg.nlist_mode = k % 2
        got, st, _ = run(upf_lib, sc, cfg)
        assert st.iterations == ref_st.iterations
        for f in ("pos", "vel", "density", "pressure"):
            assert np.array_equal(got[f], ref[f]), (cfg.as_dict(), f)


@pytest.mark.parametrize("cap", [2048, 600, 300, 0])
def test_staged_passes_with_and_without_room_for_the_union(upf_lib, cap):
    """Staged neighbourhoods (mode 2) in both passes, with the union capacity
    lowered so that some chunks (600: a few, 300: most, 0: all) do not fit and
    read the plain lists: identical results to the default shape either way.
    The scene includes rigid bodies and grains, whose lists are not staged."""
    for name in ("small_pcisph", "small_coupling"):
        sc = getattr(scenes, name)()
        p = upf_lib.derive_params(sc.params)
        out = []
        for cfg in (None, shape(128, 256, STAGED[0], STAGED[0]), shape(128, 256, STAGED[1], STAGED[1]),
                    shape(128, 256, STAGED[0], (1, 256, 4)), shape(128, 256, (0, 256, 4), STAGED[1])):
            with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
                s.set_particles(sc.pos, sc.vel, sc.type)
                if getattr(sc, "num_bodies", 0):
                    s.set_rigid_bodies(sc.body, sc.num_bodies)
                if cfg is not None:
                    s.set_launch_config(cfg)
                    upf_lib.check(upf_lib.lib().upf_test_stage_union_cap(s._h, cap), "upf_test_stage_union_cap")
                s.step(3)
                g = s.particles()
                o = np.argsort(g["id"], kind="stable")
                out.append(({k: v[o] for k, v in g.items()}, s.stats().iterations))
        ref, ref_it = out[0]
        for got, it in out[1:]:
            assert it == ref_it, name
            for f in ("pos", "vel", "density", "pressure"):
                assert np.array_equal(got[f], ref[f]), (name, cap, f)


def test_staged_mode_chosen_between_phases(upf_lib):
    """Lists built under a plain shape, then the staged mode set before the
    loop (phase by phase): the loop passes stage the lists themselves, and
    the step equals one taken wholly under the default shape."""
    sc = scenes.small_pcisph()
    p = upf_lib.derive_params(sc.params)
    with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        s.step(1)
        ref = s.particles()
    with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        s.phase("sort")
        s.phase("neighbors")
        s.set_launch_config(shape(128, 256, STAGED[0], STAGED[1]))
        for ph in ("forces", "predict_correct", "integrate"):
            s.phase(ph)
        s.synchronize()
        got = s.particles()
    for f in ("pos", "vel", "density", "pressure"):
        assert np.array_equal(got[f][np.argsort(got["id"])], ref[f][np.argsort(ref["id"])]), f


@pytest.mark.parametrize("scene", ["small_pcisph", "small_coupling"])
def test_every_list_mode_builds_the_same_lists(upf_lib, scene):
    """Neighbour lists (ids, order, counts) of both list-building modes and
    every CTA size equal those of the default shape; the scenes have boundary
    particles, so cells with both sets (merged by key) are covered too."""
    sc = getattr(scenes, scene)()
    p = upf_lib.derive_params(sc.params)

    def lists(nl, mode):
        with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
            s.set_particles(sc.pos, sc.vel, sc.type)
            if getattr(sc, "num_bodies", 0):
                s.set_rigid_bodies(sc.body, sc.num_bodies)
            if nl:
                c = s.launch_config()
                c.nlist_threads, c.nlist_mode = nl, mode
                s.set_launch_config(c)
            s.phase("sort")
            s.phase("neighbors")
            return s.neighbors()

    ref_cnt, ref_lists = lists(0, 0)
    assert ref_cnt.max() > 0
    for nl in (64, 128, 256):
        for mode in (0, 1):
            cnt, lst = lists(nl, mode)
            assert np.array_equal(cnt, ref_cnt), (nl, mode)
            for i in np.flatnonzero(cnt):
                assert np.array_equal(lst[i, :cnt[i]], ref_lists[i, :cnt[i]]), (nl, mode, i)


def test_autotune_keeps_state_and_picks_a_valid_shape(upf_lib):
    sc = scenes.small_pcisph()
    ref, _, _ = run(upf_lib, sc, None)
    got, _, chosen = run(upf_lib, sc, None, tune=True)
    for f in ("pos", "vel", "density", "pressure"):
        assert np.array_equal(got[f], ref[f]), f
    assert (chosen.density_mode, chosen.density_threads, chosen.density_rows) in LOOP_PAIRS
    assert (chosen.pforce_mode, chosen.pforce_threads, chosen.pforce_rows) in PFORCE_PAIRS
    assert chosen.nlist_threads in (64, 128, 256) and chosen.external_threads in (128, 256)
    assert all(m > 0 for m in chosen.measured_ms)


def test_batch_shapes_and_autotune(upf_lib):
    scs = scenes.batch_scenes(num=5, seed=13, counts=(2048, 8192))

    def go(cfg, tune):
        with upf_lib.ParticleBatch.from_scenes(scs) as b:
            if cfg is not None:
                b.set_launch_config(cfg)
            b.step(1)
            chosen = b.autotune(repeats=2) if tune else None
            b.step(2)
            return [b.particles(k) for k in range(len(scs))], chosen

    ref, _ = go(None, False)
    for cfg in (shape(64, 128, (128, 16), (256, 4)), shape(128, 256, (256, 4), (128, 8)),
                shape(256, 256, (1, 256, 8), (1, 128, 4))):
        cfg.nlist_mode = 1
        got, _ = go(cfg, False)
        for a, b in zip(got, ref):
            assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])
    got, chosen = go(None, True)
    for a, b in zip(got, ref):
        assert np.array_equal(a["pos"], b["pos"])
    assert chosen.density_threads <= 256 and chosen.pforce_threads <= 256


def test_invalid_shapes_rejected(upf_lib):
    sc = scenes.small_pcisph()
    p = upf_lib.derive_params(sc.params)
    with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        for bad in (shape(96, 256, (256, 8), (256, 4)), shape(256, 256, (256, 16), (256, 4)),
                    shape(256, 64, (256, 8), (256, 4)), shape(256, 256, (1, 256, 2), (256, 4)),
                    shape(256, 256, (256, 8), (2, 128, 4)), shape(256, 256, (2, 256, 2), (256, 4)),
                    shape(256, 256, (256, 8), (3, 256, 8)), shape(256, 256, (256, 8), (128, 16)),
                    shape(256, 256, (256, 8), (1024, 2))):
            with pytest.raises(UpfError):
                s.set_launch_config(bad)
        bad = shape(256, 256, (256, 8), (256, 4))
        bad.nlist_mode = 2
        with pytest.raises(UpfError):
            s.set_launch_config(bad)
    scs = scenes.batch_scenes(num=2, seed=3, counts=(2048, 4096))
    with upf_lib.ParticleBatch.from_scenes(scs) as b:
        with pytest.raises(UpfError):
            b.set_launch_config(shape(256, 256, (512, 4), (256, 8)))  # a CTA across two scenes
        with pytest.raises(UpfError):
            b.set_launch_config(shape(128, 128, (2, 256, 4), (128, 4)))  # staged: single scenes only
        b.set_launch_config(shape(128, 128, (256, 2), (128, 4)))
