"""The FP64 CPU adjoint (oracle/adjoint_oracle.cpp) against central finite
differences of its own loss: the gradient with respect to the initial
velocities (random directions) and to the viscosity agrees within 1e-6
relative on a 512-particle blob over 10 steps (eps = 1e-6 in FP64)."""
import numpy as np

from unifiedparticleframeworkcuda_b200 import scenes


def test_oracle_adjoint_matches_central_differences(oracle_lib, upf_lib):
    sc = scenes.adjoint_scene(8, 8, 8)
    p = upf_lib.derive_params(sc.params)
    x = sc.pos[:, :3].astype(np.float64)
    v = sc.vel[:, :3].astype(np.float64)
    tgt = x.mean(0) + np.array([0.1, 0.0, 0.0])
    args = dict(steps=10, iterations=3, target=tgt, com_weight=1.0, density_weight=1e-6)
    L, gv, gm = oracle_lib.adjoint_run(p, x, v, viscosity=p.viscosity, **args)
    assert L > 0 and np.isfinite(gv).all()
    rng = np.random.default_rng(3)
    eps = 1e-6
    for _ in range(3):
        u = rng.normal(size=v.shape)
        lp = oracle_lib.adjoint_run(p, x, v + eps * u, viscosity=p.viscosity, grad=False, **args)
        lm = oracle_lib.adjoint_run(p, x, v - eps * u, viscosity=p.viscosity, grad=False, **args)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - (gv * u).sum()) <= 1e-6 * abs(fd)
    e = eps * p.viscosity
    lp = oracle_lib.adjoint_run(p, x, v, viscosity=p.viscosity + e, grad=False, **args)
    lm = oracle_lib.adjoint_run(p, x, v, viscosity=p.viscosity - e, grad=False, **args)
    fd = (lp - lm) / (2 * e)
    assert abs(fd - gm) <= 1e-6 * abs(fd)
