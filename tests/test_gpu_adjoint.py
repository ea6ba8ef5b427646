"""The device adjoint (upf_adjoint_*) on a 4,096-particle copy of the
differentiation workload, 20 steps, 3 predict-correct iterations per step,
checkpoints every 5 steps, the pressure update's maximum smoothed over
+-1% of rho0 (the default):
  * loss equal to the FP64 oracle's within 1e-4 relative (FP32 trajectory);
  * gradient with respect to the initial velocities within 1e-3 relative (L2)
    of the FP64 oracle adjoint, directional derivatives within 1e-3 of FP64
    central differences, and the viscosity derivative likewise;
  * the checkpoint interval changes nothing: bit-identical velocity gradients
    and final state; the loss and the viscosity derivative are FP64 atomic
    sums (order of the CTAs), equal within 1e-12 relative."""
import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import scenes

pytestmark = pytest.mark.gpu

T, K = 20, 3


def setup(upf):
    sc = scenes.adjoint_scene(16, 16, 16)
    p = upf.derive_params(sc.params)
    tgt = sc.pos[:, :3].astype(np.float64).mean(0) + np.array([0.1, 0.0, 0.0])
    return sc, p, tgt


def test_adjoint_matches_fp64_oracle_and_differences(upf_lib, oracle_lib):
    sc, p, tgt = setup(upf_lib)
    with upf_lib.Adjoint(p, sc.pos, sc.vel, T, checkpoint_interval=5, loop_iterations=K, target=tgt,
                         com_weight=1.0, density_weight=1e-6, derive=False) as a:
        loss = a.forward()
        gv, gm = a.backward()
    x = sc.pos[:, :3].astype(np.float64)
    v = sc.vel[:, :3].astype(np.float64)
    args = dict(steps=T, iterations=K, target=tgt, com_weight=1.0, density_weight=1e-6)
    L64, gv64, gm64 = oracle_lib.adjoint_run(p, x, v, viscosity=p.viscosity, **args)
    assert abs(loss - L64) <= 1e-4 * abs(L64)
    assert np.linalg.norm(gv - gv64) <= 1e-3 * np.linalg.norm(gv64)
    assert abs(gm - gm64) <= 1e-3 * abs(gm64)
    rng = np.random.default_rng(11)
    eps = 1e-6
    for _ in range(2):
        u = rng.normal(size=v.shape)
        lp = oracle_lib.adjoint_run(p, x, v + eps * u, viscosity=p.viscosity, grad=False, **args)
        lm = oracle_lib.adjoint_run(p, x, v - eps * u, viscosity=p.viscosity, grad=False, **args)
        fd = (lp - lm) / (2 * eps)
        assert abs((gv.astype(np.float64) * u).sum() - fd) <= 1e-3 * abs(fd)
    e = eps * p.viscosity
    lp = oracle_lib.adjoint_run(p, x, v, viscosity=p.viscosity + e, grad=False, **args)
    lm = oracle_lib.adjoint_run(p, x, v, viscosity=p.viscosity - e, grad=False, **args)
    assert abs(gm - (lp - lm) / (2 * e)) <= 1e-3 * abs((lp - lm) / (2 * e))


def test_checkpoint_interval_does_not_change_gradients(upf_lib):
    sc, p, tgt = setup(upf_lib)
    out = []
    for c in (1, 7, 20):
        with upf_lib.Adjoint(p, sc.pos, sc.vel, T, checkpoint_interval=c, loop_iterations=K, target=tgt,
                             derive=False) as a:
            loss = a.forward()
            gv, gm = a.backward()
            pos, _ = a.state()
        out.append((loss, gv, gm, pos))
    for o in out[1:]:
        assert abs(o[0] - out[0][0]) <= 1e-12 * abs(out[0][0])
        assert abs(o[2] - out[0][2]) <= 1e-12 * abs(out[0][2])
        assert np.array_equal(o[1], out[0][1]) and np.array_equal(o[3], out[0][3])
