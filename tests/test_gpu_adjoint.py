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
    sums (order of the CTAs), equal within 1e-12 relative;
  * the same bars with the density term alone (the centre-of-mass term's
    gradient is the same vector for every particle and never reaches the
    pair adjoints), and over the configured 200 steps with checkpoints every
    20. In the default loss (centre-of-mass weight 1, density weight 1e-6)
    the FP64 oracle puts 1.6% of |dL/dv0| in the centre-of-mass term over 20
    steps and 15% over 200."""
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


def _check_against_fp64(upf, oracle, p, sc, tgt, steps, interval, com_weight, density_weight, directions=2,
                        along_gradient=False):
    with upf.Adjoint(p, sc.pos, sc.vel, steps, checkpoint_interval=interval, loop_iterations=K, target=tgt,
                     com_weight=com_weight, density_weight=density_weight, derive=False) as a:
        loss = a.forward()
        gv, gm = a.backward()
    x = sc.pos[:, :3].astype(np.float64)
    v = sc.vel[:, :3].astype(np.float64)
    args = dict(steps=steps, iterations=K, target=tgt, com_weight=com_weight, density_weight=density_weight)
    L64, gv64, gm64 = oracle.adjoint_run(p, x, v, viscosity=p.viscosity, **args)
    assert abs(loss - L64) <= 1e-4 * abs(L64)
    assert np.linalg.norm(gv - gv64) <= 1e-3 * np.linalg.norm(gv64)
    assert abs(gm - gm64) <= 1e-3 * abs(gm64)
    rng = np.random.default_rng(17)
    eps = 1e-6
    dirs = [rng.normal(size=v.shape) for _ in range(directions)]
    if along_gradient:
        # a random direction's derivative is a sum with heavy cancellation
        # (about 1% of |g| |u| here), so its relative error says little;
        # along the FP64 gradient it is the gradient's own size
        dirs = [gv64 / np.linalg.norm(gv64)]
    for u in dirs:
        lp = oracle.adjoint_run(p, x, v + eps * u, viscosity=p.viscosity, grad=False, **args)
        lm = oracle.adjoint_run(p, x, v - eps * u, viscosity=p.viscosity, grad=False, **args)
        fd = (lp - lm) / (2 * eps)
        assert abs((gv.astype(np.float64) * u).sum() - fd) <= 1e-3 * abs(fd)
    e = eps * p.viscosity
    lp = oracle.adjoint_run(p, x, v, viscosity=p.viscosity + e, grad=False, **args)
    lm = oracle.adjoint_run(p, x, v, viscosity=p.viscosity - e, grad=False, **args)
    assert abs(gm - (lp - lm) / (2 * e)) <= 1e-3 * abs((lp - lm) / (2 * e))
    return gv64


def test_density_only_loss_exercises_the_pair_adjoints(upf_lib, oracle_lib):
    """With the centre-of-mass term off the loss depends on the initial
    velocities only through the pair terms (pressure, viscosity, density),
    whose adjoints k_ab_pforce / k_ab_density / k_ab_external carry the whole
    gradient; the centre-of-mass term alone would give every particle the
    same gradient."""
    sc, p, tgt = setup(upf_lib)
    gv64 = _check_against_fp64(upf_lib, oracle_lib, p, sc, tgt, T, 5, com_weight=0.0, density_weight=1.0)
    # far from uniform: the spread across particles is of the gradient's size
    assert np.abs(gv64 - gv64.mean(0)).max() >= 0.5 * np.abs(gv64).max()


def test_adjoint_over_the_configured_200_steps(upf_lib, oracle_lib):
    """The configured trajectory length (200 steps, checkpoints every 20) on
    the 4,096-particle copy: device gradients against the FP64 oracle adjoint
    (which equals FP64 central differences to 3e-6 in a random direction) and
    against FP64 central differences along the gradient."""
    sc, p, tgt = setup(upf_lib)
    _check_against_fp64(upf_lib, oracle_lib, p, sc, tgt, 200, 20, com_weight=1.0, density_weight=1e-6,
                        along_gradient=True)


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
