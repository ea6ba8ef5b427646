"""Batched scenes (upf_batch_*): every scene of a batch must come out exactly
as the same scene run alone through upf_system (same sort order, neighbour
lists, per-scene iteration counts and float sums), so the bar is bit-exact
per scene on positions, velocities, predicted densities and pressures, and
equal iteration counts every step. Kinetic energy and momentum are FP64
atomic sums whose order depends on the CTA grid: 1e-9 relative."""
import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import UpfError, scenes

pytestmark = pytest.mark.gpu


def by_id(d):
    o = np.argsort(d["id"], kind="stable")
    return {k: v[o] for k, v in d.items()}


def run_single(upf, sc, steps):
    p = upf.derive_params(sc.params)
    s = upf.ParticleSystem(p, capacity=sc.n, derive=False)
    s.set_particles(sc.pos, sc.vel, sc.type)
    iters = []
    for _ in range(steps):
        s.step(1)
        iters.append(s.stats().iterations)
    st = s.stats()
    out = by_id(s.particles())
    s.close()
    return out, iters, st


def test_batch_equals_single_scene_runs(upf_lib):
    scs = scenes.batch_scenes(num=10, seed=31, counts=(2048, 12000))
    steps = 4
    with upf_lib.ParticleBatch.from_scenes(scs) as b:
        iters = []
        for _ in range(steps):
            b.step(1)
            iters.append([st.iterations for st in b.stats()])
        stats = b.stats()
        for k, sc in enumerate(scs):
            want, want_iters, want_st = run_single(upf_lib, sc, steps)
            got = by_id(b.particles(k))
            assert [it[k] for it in iters] == want_iters, "scene %d iterations" % k
            for f in ("id", "pos", "vel", "density", "pressure"):
                assert np.array_equal(got[f], want[f]), "scene %d field %s" % (k, f)
            assert stats[k].max_predicted_density == want_st.max_predicted_density
            assert abs(stats[k].kinetic_energy - want_st.kinetic_energy) <= 1e-9 * abs(want_st.kinetic_energy)
    # the scenes converge at different iterations: the batch's while-node
    # must stop each one at its own count
    assert len({tuple(it) for it in np.array(iters).T.tolist()}) > 1


def test_batch_checkpoint_restore_replays(upf_lib):
    scs = scenes.batch_scenes(num=6, seed=5, counts=(2048, 8192))
    with upf_lib.ParticleBatch.from_scenes(scs) as b:
        b.step(2)
        b.checkpoint(0)
        b.step(3)
        first = [b.particles(k) for k in range(len(scs))]
        b.restore(0)
        b.step(3)
        for k in range(len(scs)):
            again = b.particles(k)
            for f in ("pos", "vel", "id"):
                assert np.array_equal(first[k][f], again[f])


def test_batch_upload_download_roundtrip(upf_lib):
    import ctypes as C
    scs = scenes.batch_scenes(num=5, seed=9, counts=(2048, 6000))
    with upf_lib.ParticleBatch.from_scenes(scs) as b:
        b.step(1)
        n = int(b.offsets[-1])
        pos = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        L = upf_lib.lib()
        fp = C.POINTER(C.c_float)
        upf_lib.check(L.upf_batch_download_state(b.handle, pos.ctypes.data_as(fp), vel.ctypes.data_as(fp)), "dl")
        for k in range(len(scs)):
            got = b.particles(k)
            o = b.offsets[k]
            assert np.array_equal(pos[o:o + b.counts[k]], got["pos"])
        pos[:, 1] += 0.001
        upf_lib.check(L.upf_batch_upload_state(b.handle, pos.ctypes.data_as(fp), vel.ctypes.data_as(fp)), "ul")
        got = b.particles(0)
        assert np.array_equal(got["pos"][:, 1], pos[:b.counts[0], 1])


def test_batch_argument_checks(upf_lib):
    w = scenes.small_wcsph()
    with pytest.raises(UpfError):
        upf_lib.ParticleBatch([w.params], [w.n])  # WCSPH is not batched
    scs = scenes.batch_scenes(num=2, seed=3, counts=(2048, 4096))
    b = upf_lib.ParticleBatch([s.params for s in scs], [s.n for s in scs])
    with pytest.raises(UpfError):
        b.step(1)  # no particles yet
    with pytest.raises(ValueError):
        b.set_particles(np.zeros((3, 4), np.float32), np.zeros((3, 4), np.float32))
    b.close()


def test_batch_with_tiny_and_ragged_scenes(upf_lib):
    """Scenes of 1, 2, 31, 33 and 257 particles beside a 6,000-particle
    scene: each equals its single-scene run bit for bit. Every scene starts
    its own segment, so scenes smaller than a warp or a CTA share no CTA."""
    counts = [1, 2, 31, 33, 257, 6000]
    scs = [scenes.batch_scene(n, (0.6, 0.8, 0.5), 100 + k, stream=k + 1) for k, n in enumerate(counts)]
    assert [sc.n for sc in scs] == counts
    steps = 3
    with upf_lib.ParticleBatch.from_scenes(scs) as b:
        iters = []
        for _ in range(steps):
            b.step(1)
            iters.append([st.iterations for st in b.stats()])
        got = [by_id(b.particles(k)) for k in range(len(scs))]
    for k, sc in enumerate(scs):
        want, want_iters, _ = run_single(upf_lib, sc, steps)
        assert [it[k] for it in iters] == want_iters, "scene %d iterations" % k
        for f in ("id", "pos", "vel", "density", "pressure"):
            assert np.array_equal(got[k][f], want[f]), "scene %d field %s" % (k, f)
