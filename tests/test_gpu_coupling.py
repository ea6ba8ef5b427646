"""Rigid-fluid coupling and granular contact: the CUDA path against the CPU
oracle on a small coupling scene (12^3 liquid, an 8x4x8 granular pile, three
rigid bodies: sphere, cube, torus).

Bars:
  * one step: iteration count equal; positions, velocities and external
    forces of every liquid, granular and rigid particle, and the bodies'
    positions, velocities, angular velocities and quaternions within 1e-5
    relative (|gpu - cpu| <= 1e-5 * max(|cpu|, field scale)). The per-body
    force and torque are FP64 sums in a different order on each side (a tree
    on the GPU, array order on the CPU), so they may differ in the last FP64
    bits, far below the FP32 state's resolution;
  * several steps: per-step iteration counts equal while the trajectories
    agree, body states within 1e-4 relative after 10 steps;
  * a lone body in free fall keeps zero angular velocity and falls with
    v = -g t exactly as the float update computes it.
"""
import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import FROZEN, GRANULAR, LIQUID, RIGID, UpfError, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def close(gpu, cpu, rtol=RTOL):
    gpu = np.asarray(gpu, np.float64)
    cpu = np.asarray(cpu, np.float64)
    if cpu.size == 0:
        return True, 0.0
    scale = max(np.abs(cpu).max(), 1e-30)
    err = np.abs(gpu - cpu)
    bound = rtol * np.maximum(np.abs(cpu), scale)
    return bool(np.all(err <= bound)), float((err / scale).max())


def make(upf, oracle, sc):
    p = upf.derive_params(sc.params)
    sysm = upf.ParticleSystem(p, capacity=sc.n, derive=False)
    sysm.set_particles(sc.pos, sc.vel, sc.type)
    sysm.set_rigid_bodies(sc.body, sc.num_bodies)
    o = oracle.OracleSim(p, sc.pos, sc.vel, sc.type)
    o.set_rigid_bodies(sc.body, sc.num_bodies)
    return p, sysm, o


def compare_particles(sysm, o, rtol=RTOL):
    g = sysm.particles()
    c = o.state()
    dyn = c["type"] != FROZEN
    go = np.argsort(g["id"], kind="stable")
    co = np.argsort(c["id"][dyn], kind="stable")
    gid, gtype = g["id"][go], g["type"][go]
    assert np.array_equal(gid, c["id"][dyn][co])
    assert np.array_equal(gtype, c["type"][dyn][co])
    out = {}
    for t, name in ((LIQUID, "liquid"), (GRANULAR, "granular"), (RIGID, "rigid")):
        m = gtype == t
        for f in ("pos", "vel"):
            out["%s.%s" % (name, f)] = close(g[f][go][m, :3], c[f][dyn][co][m, :3], rtol)
    return out


def compare_forces(sysm, o):
    f = sysm.step_fields()
    cf = o.step_fields()
    c = o.state()
    type_of = dict(zip(c["id"].tolist(), c["type"].tolist()))
    fo = np.argsort(f["id"], kind="stable")
    fid = f["id"][fo]
    co = np.argsort(cf["id"], kind="stable")
    cid = cf["id"][co]
    keep = np.isin(cid, fid)
    assert np.array_equal(cid[keep], fid)
    ftype = np.array([type_of[int(i)] for i in fid])
    out = {}
    for t, name in ((LIQUID, "liquid"), (GRANULAR, "granular"), (RIGID, "rigid")):
        m = ftype == t
        out["force." + name] = close(f["force"][fo][m, :3], cf["force"][co][keep][m, :3])
    return out


def compare_bodies(sysm, o, rtol=RTOL):
    gp, gv, gw, gq = sysm.rigid_bodies()
    cp, cv, cw, cq = o.rigid()
    out = {}
    for name, a, b in (("body.pos", gp, cp), ("body.vel", gv, cv), ("body.omega", gw, cw), ("body.quat", gq, cq)):
        out[name] = close(a, b, rtol)
    return out


def test_coupling_single_step_parity(upf_lib, oracle_lib):
    sc = scenes.small_coupling()
    p, sysm, o = make(upf_lib, oracle_lib, sc)
    assert int(np.count_nonzero(sc.type == GRANULAR)) > 0 and sc.num_bodies == 3
    # the bodies at rest, as assembled (FP64 sums on both sides)
    res = compare_bodies(sysm, o)
    assert all(v[0] for v in res.values()), res
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


def test_coupling_multi_step(upf_lib, oracle_lib):
    sc = scenes.small_coupling()
    p, sysm, o = make(upf_lib, oracle_lib, sc)
    for k in range(10):
        sysm.step(1)
        it = sysm.stats().iterations
        info = o.step()
        assert it == info.iterations, "step %d: iterations %d vs %d" % (k, it, info.iterations)
    res = compare_bodies(sysm, o, rtol=1e-4)
    res.update(compare_particles(sysm, o, rtol=1e-4))
    bad = {k: v for k, v in res.items() if not v[0]}
    assert not bad, "beyond 1e-4 relative after 10 steps: %s" % bad
    # the bodies fall (gravity, no contact yet at this height)
    gp, gv, _, _ = sysm.rigid_bodies()
    assert np.all(gv[:, 1] < 0)
    sysm.close()
    o.close()


def test_bodies_in_contact_against_the_oracle(upf_lib, oracle_lib):
    """The rigid case of tests/golden/reference_step.npz (a sphere half sunk
    into the fluid, a cube beside it within spring range, a torus on the
    floor; surface tension, penalty walls, adhesion), whose reference steps
    the oracle reproduces bit for bit under the literal rigid rules: here
    the device against the oracle under this build's rules. One step: forces
    of every particle and the body states within 1e-5; 20 steps: iteration
    counts equal every step, bodies and particles within 1e-4."""
    import os
    from unifiedparticleframeworkcuda_b200._abi import UpfParams
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_step.npz"))
    name = "rigid_contact"
    p = UpfParams.from_buffer_copy(g[name + "_params"].tobytes())
    pos, vel, typ = g[name + "_pos_in"], g[name + "_vel_in"], g[name + "_type_in"]
    body, nb = g[name + "_body_in"], int(g[name + "_num_bodies"])
    sysm = upf_lib.ParticleSystem(p, capacity=len(typ), derive=False)
    sysm.set_particles(pos, vel, typ)
    sysm.set_rigid_bodies(body, nb)
    o = oracle_lib.OracleSim(p, pos, vel, typ)
    o.set_rigid_bodies(body, nb)
    sysm.step(1)
    info = o.step()
    assert sysm.stats().iterations == info.iterations
    res = compare_forces(sysm, o)
    res.update(compare_bodies(sysm, o))
    res.update(compare_particles(sysm, o))
    bad = {k: v for k, v in res.items() if not v[0]}
    assert not bad, "beyond %g relative after one step: %s" % (RTOL, bad)
    for k in range(1, int(g[name + "_steps"])):
        sysm.step(1)
        it = sysm.stats().iterations
        info = o.step()
        assert it == info.iterations, "step %d: iterations %d vs %d" % (k, it, info.iterations)
    res = compare_bodies(sysm, o, rtol=1e-4)
    res.update(compare_particles(sysm, o, rtol=1e-4))
    bad = {k: v for k, v in res.items() if not v[0]}
    assert not bad, "beyond 1e-4 relative after the case's steps: %s" % bad
    sysm.close()
    o.close()


def test_free_fall_body(upf_lib):
    """One cube far from everything: the momentum update P += (sum f + M g) dt
    with no contact force keeps omega = 0 and v_y = M g t / M in float."""
    p = scenes.default_params()
    p.method = scenes.METHOD_PCISPH
    p.flags = 0
    p.particle_spacing = 0.01
    p.support_radius = 0.02
    p.dt = 5e-4
    p.zindex_extent[:] = (2.048, 2.048, 2.048)
    scenes._set_box(p, np.array([0.02, 0.02, 0.02]), np.array([2.0, 2.0, 2.0]))
    pts = scenes.sample_box(0.05, 200) + np.array([1.0, 1.5, 1.0])
    n = pts.shape[0]
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = pts
    vel = np.zeros_like(pos)
    typ = np.full(n, RIGID, np.int32)
    q = upf_lib.derive_params(p)
    with upf_lib.ParticleSystem(q, capacity=n, derive=False) as s:
        s.set_particles(pos, vel, typ)
        s.set_rigid_bodies(np.zeros(n, np.int32), 1)
        P = np.float32(0)
        M = np.float32(np.float64(q.mass) * n)
        dt = np.float32(q.dt)
        g = np.float64(-np.float32(q.mass) * np.float32(q.gravity)) * n  # FP64 sum of n equal terms
        for k in range(20):
            s.step(1)
            P = np.float32(P + np.float32(g) * dt)
        _, v, w, quat = s.rigid_bodies()
        assert np.all(w == 0) and np.array_equal(quat[0], np.array([1, 0, 0, 0], np.float32))
        assert v[0, 1] == np.float32(P * (np.float32(1) / M))
        assert v[0, 0] == 0 and v[0, 2] == 0


def test_rigid_body_argument_checks(upf_lib):
    sc = scenes.small_coupling()
    p = upf_lib.derive_params(sc.params)
    with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        bad = sc.body.copy()
        bad[np.flatnonzero(sc.type == LIQUID)[0]] = 0  # a liquid particle in a body
        with pytest.raises(UpfError):
            s.set_rigid_bodies(bad, sc.num_bodies)
        with pytest.raises(UpfError):
            s.set_rigid_bodies(sc.body, sc.num_bodies + 1)  # an empty body
        s.set_rigid_bodies(sc.body, sc.num_bodies)
        s.step(1)
        with pytest.raises(UpfError) as e:
            s.set_rigid_bodies(sc.body, sc.num_bodies)  # after a step
        assert "before the first step" in str(e.value)
    w = scenes.small_wcsph()
    pw = upf_lib.derive_params(w.params)
    with upf_lib.ParticleSystem(pw, capacity=w.n, derive=False) as s:
        typ = w.type.copy()
        typ[0] = GRANULAR
        with pytest.raises(UpfError):
            s.set_particles(w.pos, w.vel, typ)  # granular needs PCISPH
