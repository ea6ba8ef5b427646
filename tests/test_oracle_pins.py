"""The oracle restatement pinned against the reference's own CPU code: the
golden fixtures in tests/golden/reference_tables.npz and
tests/golden/reference_rigid.npz (made by tests/golden/make_golden.py from the
reference's zIndex.cpp, WeightingKernel.cpp, UnifiedConstants.cpp,
RigidBody.cpp and Matrix3x3.cpp), and, where the reference tree is available,
the compiled reference directly."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import pyoracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_tables.npz")
GOLDEN_RIGID = os.path.join(os.path.dirname(__file__), "golden", "reference_rigid.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def golden_rigid():
    return np.load(GOLDEN_RIGID)


def test_rigid_body_update_bit_equal_to_reference(oracle_lib, golden_rigid):
    """RigidBody::UpdateMomenta + PerformStep + UpdateRotationMatrix: the
    oracle's float body update reproduces the reference's compiled code bit
    for bit on 256 seeded states (clamped and free momenta)."""
    g = golden_rigid
    for k in range(g["body_in"].shape[0]):
        out = oracle_lib.rigid_body_step(g["body_in"][k], g["body_force"][k], g["body_torque"][k],
                                         g["body_dt"][k], g["body_terminal_speed"][k])
        assert np.array_equal(out.view(np.uint32), g["body_out"][k].view(np.uint32)), "state %d" % k


def test_inertia_inverse_vs_reference(oracle_lib, golden_rigid):
    """Matrix3x3::CalculateInverse: the oracle inverts in FP64 (the reference in
    float); on seeded inertia tensors the two agree to float accuracy scaled
    by the condition number, and the FP64 inverse is the closer to exact."""
    g = golden_rigid
    for m, ref, ok in zip(g["inertia"], g["inertia_inverse"], g["inertia_ok"]):
        assert ok == 1
        ours = oracle_lib.inverse3(m)
        exact = np.linalg.inv(m.astype(np.float64).reshape(3, 3)).ravel()
        cond = np.linalg.cond(m.astype(np.float64).reshape(3, 3))
        scale = np.abs(exact).max()
        assert np.abs(ours - exact).max() <= 1e-6 * scale
        assert np.abs(ref - exact).max() <= 1e-6 * cond * scale
        assert np.abs(ours - exact).max() <= np.abs(ref - exact).max() + 1e-7 * scale


def test_morton_table_matches_reference(oracle_lib, golden):
    assert np.array_equal(oracle_lib.morton_table(), golden["morton_table"])


def test_luts_bit_equal_to_reference(oracle_lib, golden):
    for h, ref in zip(golden["lut_h"], golden["luts"]):
        p = oracle_lib.default_params()
        p.support_radius = float(h)
        got = oracle_lib.luts(p)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), "h=%r" % h


def test_box_query_matches_reference(oracle_lib, golden):
    off = 0
    for box, bs, n in zip(golden["bq_boxes"], golden["bq_block"], golden["bq_count"]):
        f, l = oracle_lib.box_query(int(bs), box[:3], box[3:])
        assert len(f) == n
        assert np.array_equal(f, golden["bq_first"][off:off + n])
        assert np.array_equal(l, golden["bq_last"][off:off + n])
        off += n


def test_block_size_rounding_matches_reference(oracle_lib, golden):
    # ZIndex::SetBlockSize: smallest power of two >= size
    for s, bs in zip(golden["block_size_in"], golden["block_size_out"]):
        p = oracle_lib.default_params()
        p.support_radius = 1.0
        p.zindex_extent[:] = (1024.0, 1024.0, 1024.0)
        p.scales[:] = (float(s), float(s), float(s))
        q = oracle_lib.derive(p)
        assert q.block_size == bs, (s, q.block_size, bs)


def test_default_constants_match_reference(oracle_lib, golden):
    c = golden["default_constants"]
    p = oracle_lib.derive(oracle_lib.default_params())
    got = [p.particle_spacing, p.particle_radius, p.support_radius, p.mass, p.rest_density,
           p.gas_constant, p.gamma, p.viscosity, p.gravity, p.dt, p.density_error_fudge,
           p.max_density_error, p.min_loops, p.max_loops, p.surface_tension_gamma,
           p.surface_adhesion_beta, p.force_distance, p.max_boundary_force, p.spring_coefficient,
           p.spring_coefficient_boundary, p.damping_coefficient, p.terminal_speed, p.granular_kr,
           p.granular_kd, p.granular_kt, p.granular_mu, *p.scales]
    assert np.array_equal(np.float32(got), c[:29])


def test_morton_key_of_position(oracle_lib, golden):
    tab = golden["morton_table"]
    p = oracle_lib.derive(oracle_lib.default_params())
    rng = np.random.default_rng(5)
    for _ in range(200):
        x = rng.uniform(0, 1.4, 3).astype(np.float32)
        c = [int(np.float32(p.scales[a]) * x[a]) for a in range(3)]
        want = int(tab[c[0], 0] | tab[c[1], 1] | tab[c[2], 2])
        assert oracle_lib.lib().orc_morton(C.byref(p), *map(float, x)) == want


@pytest.mark.skipif(not pyoracle.reference_present(), reason="reference tree not present")
def test_fixtures_regenerate_identically(oracle_lib, golden):
    """The committed fixtures are what the compiled reference produces now."""
    R = oracle_lib.ref()
    for h, ref in zip(golden["lut_h"], golden["luts"]):
        out = np.zeros((5, 301), np.float32)
        R.ref_luts(C.c_float(h), out.ctypes.data_as(C.POINTER(C.c_float)))
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


def test_density_error_factor_fp32_vs_fp64(oracle_lib):
    from unifiedparticleframeworkcuda_b200 import scenes
    for sc in (scenes.small_pcisph(), scenes.pcisph_dam(8, 8, 8)):
        p = oracle_lib.derive(sc.params)
        d32 = oracle_lib.lib().orc_density_error_factor(C.byref(p), 0)
        d64 = oracle_lib.lib().orc_density_error_factor(C.byref(p), 1)
        assert d32 > 0 and abs(d32 - d64) <= 1e-5 * abs(d64)


def test_oracle_multi_step_runs(oracle_lib):
    from unifiedparticleframeworkcuda_b200 import scenes
    sc = scenes.small_pcisph()
    p = oracle_lib.derive(sc.params)
    o = oracle_lib.OracleSim(p, sc.pos, sc.vel, sc.type)
    for _ in range(3):
        info = o.step()
        assert p.min_loops <= info.iterations <= p.max_loops
    st = o.state()
    liquid = st["type"] == 2
    assert np.all(np.isfinite(st["pos"][liquid]))
    # clamped into the collision box
    assert np.all(st["pos"][liquid, :3] >= np.float32(p.collision_min) - 1e-7)
    assert np.all(st["pos"][liquid, :3] <= np.float32(p.collision_max) + 1e-7)
    # sorted by key after the step (SortParticles)
    assert np.all(np.diff(st["key"].astype(np.int64)) >= 0)


# ---- the step itself, pinned to the reference's own compiled CPU step ------
# tests/golden/reference_step.npz holds what the reference's own CPU steps
# make of seeded scenes (tests/golden/make_golden.py, step_cases): the PCISPH
# coupling step CpuParticlePhysicsVersatileCouplingPCISPH
# (UnifiedPhysics.cpp:4991-5024) on two dams in a box of frozen boundary
# particles over 5 and 3 steps at the 50-iteration cap and on three rigid
# bodies in contact with the fluid, each other and the floor over 20 steps,
# and the WCSPH step CpuParticlePhysicsPureFluidsSPH over 1 and 5 steps;
# each with the member functions it calls (neighbour search, forces, the
# predict-correct loop, integration, boundary handling, the re-sort, the
# per-body force and torque sums, body update and particle sync), compiled
# unchanged by oracle/Makefile into oracle/_ref/libupfref_physics.so.
GOLDEN_STEP = os.path.join(os.path.dirname(__file__), "golden", "reference_step.npz")
STEP_CASES = ("dam_st_pw", "dam_st_pw_adh", "wcsph_ww_st", "wcsph_ww_st_box", "rigid_contact")
# the reference's literal rules for rigid bodies (see oracle/upf_oracle.h)
RIGID_LITERAL = (pyoracle.LITERAL_OWN_BODY_SPRING | pyoracle.LITERAL_ZERO_INVERSE_INERTIA
                 | pyoracle.LITERAL_FLOAT_RIGID_ASSEMBLY | pyoracle.LITERAL_FLOAT_BODY_SUMS
                 | pyoracle.LITERAL_STALE_RIGID_KEYS | pyoracle.LITERAL_STALE_RIGID_PREDICTED)


def step_case(g, name):
    from unifiedparticleframeworkcuda_b200._abi import UpfParams
    p = UpfParams.from_buffer_copy(g[name + "_params"].tobytes())
    return p, g[name + "_pos_in"], g[name + "_vel_in"], g[name + "_type_in"], int(g[name + "_steps"])


def oracle_run(oracle_lib, g, name, literal=0, steps=None):
    p, pos, vel, typ, n_steps = step_case(g, name)
    o = oracle_lib.OracleSim(p, pos, vel, typ)
    o.set_reference_literal(literal)
    if int(g[name + "_num_bodies"]):
        o.set_rigid_bodies(g[name + "_body_in"], int(g[name + "_num_bodies"]))
    for _ in range(n_steps if steps is None else steps):
        o.step()
    st = o.state()
    bodies = o.rigid() if int(g[name + "_num_bodies"]) else None
    o.close()
    order = np.argsort(st["id"])
    out = {k: st[k][order] for k in ("pos", "vel", "density", "pressure", "type", "id")}
    out["bodies"] = bodies
    return out


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


@pytest.mark.parametrize("name", STEP_CASES)
def test_oracle_steps_bit_equal_to_reference_steps(oracle_lib, name):
    """The oracle's restatement, run from the same particles and parameters,
    against the reference's own steps: every particle's position and velocity
    and every liquid particle's density and pressure are bit-identical after
    each case's steps. The one-step WCSPH case runs with the reference's
    literal boundary handling (every particle clamped to the collision box,
    frozen ones included), the rigid case with the reference's literal
    rigid-body rules (RIGID_LITERAL), and there every body's position,
    velocity, angular velocity and quaternion is bit-identical too."""
    g = np.load(GOLDEN_STEP)
    literal = {"wcsph_ww_st": pyoracle.LITERAL_WCSPH_CLAMP_ALL, "rigid_contact": RIGID_LITERAL}.get(name, 0)
    got = oracle_run(oracle_lib, g, name, literal)
    assert np.array_equal(got["id"], g[name + "_id"]) and np.array_equal(got["type"], g[name + "_type"])
    liq = got["type"] == 2
    for k in ("pos", "vel"):
        assert bits_equal(got[k], g[name + "_" + k]), k
    for k in ("density", "pressure"):
        assert bits_equal(got[k][liq], g[name + "_" + k][liq]), k
    if got["bodies"] is not None:
        pos, vel, omega, quat = got["bodies"]
        ref = g[name + "_bodies"]
        for k, (a, b) in {"pos": (pos, ref[:, 0:3]), "vel": (vel, ref[:, 3:6]), "omega": (omega, ref[:, 6:9]),
                          "quat": (quat, ref[:, 10:14])}.items():
            assert bits_equal(a, b), k


def test_wcsph_boundary_clamp_deviation_moves_only_boundary_particles(oracle_lib):
    """The deliberate deviation in WCSPH boundary handling (only liquid
    particles clamped, so the static boundary stays where it was built),
    measured against the reference's own step: after one step every liquid
    particle is bit-identical; only frozen particles that lie outside the
    collision box differ, by their clamped coordinates."""
    g = np.load(GOLDEN_STEP)
    name = "wcsph_ww_st"
    got = oracle_run(oracle_lib, g, name)
    liq = got["type"] == 2
    for k in ("pos", "vel", "density", "pressure"):
        assert bits_equal(got[k][liq], g[name + "_" + k][liq]), k
    moved = np.any(got["pos"][:, :3] != g[name + "_pos"][:, :3], axis=1)
    assert moved.any() and not moved[liq].any()


def test_boundary_pressure_deviation_measured_against_reference_step(oracle_lib):
    """The deliberate deviation in the Akinci boundary pressure (table indexed
    by distance, flag FLAG_BOUNDARY_PRESSURE) measured against the
    reference's own step, whose lookup by bin index
    (UnifiedPhysics.cpp:4240-4250) makes the term 0 for every pair: the
    fixture runs with the flag clear and the oracle equals it; with the flag
    set the liquid moves differently within three steps (the term reads the
    lagged pressure, which starts at 0) while the frozen boundary stays
    bit-identical."""
    from unifiedparticleframeworkcuda_b200._abi import FLAG_BOUNDARY_PRESSURE
    g = np.load(GOLDEN_STEP)
    name = "dam_st_pw"
    p, pos, vel, typ, _ = step_case(g, name)
    assert not (p.flags & FLAG_BOUNDARY_PRESSURE)
    runs = []
    for flags in (p.flags, p.flags | FLAG_BOUNDARY_PRESSURE):
        p.flags = flags
        o = oracle_lib.OracleSim(p, pos, vel, typ)
        for _ in range(3):
            o.step()
        st = o.state()
        o.close()
        order = np.argsort(st["id"])
        runs.append({k: st[k][order] for k in ("pos", "vel", "type")})
    liq = runs[0]["type"] == 2
    moved = np.any(runs[0]["vel"][:, :3] != runs[1]["vel"][:, :3], axis=1)
    assert moved[liq].sum() > 0.05 * liq.sum()
    for k in ("pos", "vel"):
        assert bits_equal(runs[0][k][~liq], runs[1][k][~liq]), k


@pytest.mark.parametrize("bit", [pyoracle.LITERAL_OWN_BODY_SPRING, pyoracle.LITERAL_FLOAT_RIGID_ASSEMBLY,
                                 pyoracle.LITERAL_FLOAT_BODY_SUMS, pyoracle.LITERAL_STALE_RIGID_KEYS,
                                 pyoracle.LITERAL_STALE_RIGID_PREDICTED, pyoracle.LITERAL_ZERO_INVERSE_INERTIA])
def test_rigid_deviations_measured_against_reference_step(oracle_lib, bit):
    """Each deliberate deviation of the rigid-body rules, measured against
    the reference's own coupling step on the rigid case (20 steps): the
    oracle with every literal rule but one against the fixture.
    * own-body spring-damper, float assembly, float per-body sums: rounding
      only. Liquid and rigid positions stay bit-identical; body velocities
      move by under 1e-4 of the largest body speed.
    * rigid keys taken after the sync: a different sort and summation order
      for the particles near moving bodies, positions within 1e-7 m.
    * rigid predicted positions kept current: the liquid's predicted density
      sees the bodies where they are, so the liquid moves differently; the
      bodies themselves stay bit-identical over these steps.
    * inverse inertia stored: the bodies rotate (the reference's never do)."""
    g = np.load(GOLDEN_STEP)
    name = "rigid_contact"
    got = oracle_run(oracle_lib, g, name, RIGID_LITERAL & ~bit)
    ref = g[name + "_bodies"]
    pos, vel, omega, _ = got["bodies"]
    liq = got["type"] == 2
    rig = got["type"] == 0
    same = {k: bits_equal(got[k], g[name + "_" + k]) for k in ("pos", "vel")}
    assert not (same["pos"] and same["vel"] and bits_equal(vel, ref[:, 3:6]) and bits_equal(pos, ref[:, 0:3]))
    speed = np.abs(ref[:, 3:6]).max()
    if bit in (pyoracle.LITERAL_OWN_BODY_SPRING, pyoracle.LITERAL_FLOAT_RIGID_ASSEMBLY,
               pyoracle.LITERAL_FLOAT_BODY_SUMS):
        assert same["pos"]
        assert bits_equal(got["vel"][liq], g[name + "_vel"][liq])
        assert np.abs(vel - ref[:, 3:6]).max() <= 1e-4 * speed
        assert np.all(omega == 0)
    elif bit == pyoracle.LITERAL_STALE_RIGID_KEYS:
        assert np.abs(got["pos"] - g[name + "_pos"]).max() <= 1e-7
        assert np.abs(got["vel"] - g[name + "_vel"]).max() <= 1e-4 * speed
    elif bit == pyoracle.LITERAL_STALE_RIGID_PREDICTED:
        assert bits_equal(pos, ref[:, 0:3]) and bits_equal(vel, ref[:, 3:6])
        assert bits_equal(got["pos"][rig], g[name + "_pos"][rig])
        assert not bits_equal(got["pos"][liq], g[name + "_pos"][liq])
    else:
        assert np.abs(omega).max() > 1.0
        assert not np.any(np.all(got["pos"][rig] == g[name + "_pos"][rig], axis=1))


@pytest.mark.skipif(not pyoracle.reference_present(), reason="reference tree not present")
def test_reference_resumes_from_the_oracles_lagged_state(oracle_lib):
    """The reference's step resumed mid-trajectory (the state and the lagged
    PCISPH state of another run: the step before last's and the last step's
    correction pressures and the last predicted density, as the CPU
    baselines hand it over) continues the trajectory bit for bit: the oracle
    runs 2 steps of the first dam case, the reference 3 more from its state,
    against the oracle's own 3 more."""
    from oracle import refstep
    if not refstep.available():
        pytest.skip("oracle/_ref/libupfref_physics.so not built")
    g = np.load(GOLDEN_STEP)
    p, pos, vel, typ, _ = step_case(g, "dam_st_pw")
    o = oracle_lib.OracleSim(p, pos, vel, typ)
    for _ in range(2):
        o.step()
    st = o.state()
    lag = o.lagged()
    order = np.argsort(st["id"])
    pos2, vel2 = st["pos"][order], st["vel"][order]
    for _ in range(3):
        o.step()
    want = o.state()
    o.close()
    r = refstep.reference_steps(p, pos2, vel2, typ, 3, lagged=lag)
    wo, ro = np.argsort(want["id"]), np.argsort(r["id"])
    liq = want["type"][wo] == 2
    for k in ("pos", "vel"):
        assert bits_equal(want[k][wo], r[k][ro]), k
    for k in ("density", "pressure"):
        assert bits_equal(want[k][wo][liq], r[k][ro][liq]), k


@pytest.mark.skipif(not pyoracle.reference_present(), reason="reference tree not present")
def test_reference_timing_reports_the_loops_iterations(oracle_lib):
    """The timed reference step (the CPU baselines' leg) counts each step's
    predict-correct iterations from the loop's own per-iteration report: on
    one thread they equal the oracle's counts for the same steps, and the
    last reported error of each step is the oracle's final density error."""
    from oracle import refstep
    if not refstep.available():
        pytest.skip("oracle/_ref/libupfref_physics.so not built")
    g = np.load(GOLDEN_STEP)
    p, pos, vel, typ, _ = step_case(g, "dam_st_pw")
    r = refstep.reference_time(p, pos, vel, typ, None, "pcisph", threads=1, warmup=1, steps=3, max_seconds=1e9)
    o = oracle_lib.OracleSim(p, pos, vel, typ)
    o.step()
    infos = [o.step() for _ in range(3)]
    o.close()
    assert r["seconds"].size == 3 and np.all(r["seconds"] > 0)
    assert r["iterations"].tolist() == [int(i.iterations) for i in infos]
    assert np.allclose(r["error_percent"], [float(i.density_error_percent) for i in infos], rtol=1e-5, atol=1e-4)


@pytest.mark.skipif(not pyoracle.reference_present(), reason="reference tree not present")
def test_step_fixture_regenerates_identically(oracle_lib):
    """The committed step fixture is what the compiled reference steps
    produce now (each case in a fresh process, oracle/refstep.py)."""
    from oracle import refstep
    if not refstep.available():
        pytest.skip("oracle/_ref/libupfref_physics.so not built")
    g = np.load(GOLDEN_STEP)
    for name in STEP_CASES:
        p, pos, vel, typ, steps = step_case(g, name)
        r = refstep.reference_steps(p, pos, vel, typ, steps, bool(g[name + "_weighted_volumes"]),
                                    str(g[name + "_method"]), g[name + "_body_in"], int(g[name + "_num_bodies"]))
        order = np.argsort(r["id"])
        for k in ("pos", "vel", "density", "pressure", "type", "id"):
            assert np.array_equal(r[k][order], g[name + "_" + k]), (name, k)
        assert np.array_equal(r["body"], g[name + "_bodies"]), name
