"""The slab decomposition of one scene (unifiedparticleframeworkcuda_b200/
slabs.py) run as two and three slabs on one GPU (LocalTransport: the halo
and migration exchanges as device copies, the loop test's maximum over the
slabs): every step's iteration count equals the unsplit scene's, and after
several steps every liquid particle's position and velocity agree with the
unsplit run within 1e-5 of the field's scale (the same neighbours in the
same order, so in practice bit for bit)."""
import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import LIQUID, scenes
from unifiedparticleframeworkcuda_b200 import slabs

pytestmark = pytest.mark.gpu

STEPS = 6


def _unsplit(upf, sc):
    p = upf.derive_params(sc.params)
    its = []
    with upf.ParticleSystem(p, capacity=sc.n, derive=False) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        for _ in range(STEPS):
            s.step(1)
            its.append(s.stats().iterations)
        g = s.particles()
    o = np.argsort(g["id"])
    return {k: v[o] for k, v in g.items()}, its


@pytest.mark.parametrize("nslabs", [2, 3])
def test_slabs_on_one_gpu_equal_the_unsplit_scene(upf_lib, nslabs):
    sc = scenes.pcisph_dam(24, 12, 12, box=(0.5, 0.3, 0.3))
    want, want_its = _unsplit(upf_lib, sc)
    with slabs.SlabScene(sc, nslabs, slabs.LocalTransport()) as ss:
        its = [ss.step() for _ in range(STEPS)]
        got = ss.particles()
        owned_counts = [int((ss._dynamic(s)["id"] >= 0).sum()) for s in ss.systems]
    assert its == want_its
    assert all(c > 0 for c in owned_counts)
    assert np.array_equal(got["id"], want["id"].astype(got["id"].dtype))
    liq = want["type"] == LIQUID
    for k in ("pos", "vel"):
        a = got[k][liq, :3].astype(np.float64)
        b = want[k][liq, :3].astype(np.float64)
        scale = max(np.abs(b).max(), 1e-30)
        assert np.abs(a - b).max() <= 1e-5 * scale, (k, np.abs(a - b).max() / scale)
