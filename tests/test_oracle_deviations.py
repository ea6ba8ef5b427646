"""Each deliberate deviation of the oracle from the reference's CPU path,
measured against the reference's literal rule (the oracle's
orc_set_reference_literal switches, one per deviation), on the small
coupling scene (12^3 fluid, an 8x4x8 granular pile, three rigid bodies).
The device path follows the oracle's rule; these tests state what each
deviation changes, so that it is a measured choice rather than an assumed
one. The un-clamped query box of GetNeighbors (UnifiedPhysics.cpp:2246-2252)
has no switch: for particles inside the key grid it gives the same box as
the clamped one, and outside it converts an out-of-range float to an
unsigned short, which is undefined behaviour."""
import numpy as np
import pytest

from oracle import pyoracle
from unifiedparticleframeworkcuda_b200 import GRANULAR, RIGID, derive_params, scenes

STEPS = 10


def _run(mask, steps=STEPS, scene=None):
    sc = scene or scenes.small_coupling()
    p = derive_params(sc.params)
    o = pyoracle.OracleSim(p, sc.pos, sc.vel, sc.type, threads=4, keep_fields=False)
    o.set_reference_literal(mask)
    o.set_rigid_bodies(sc.body, sc.num_bodies)
    for _ in range(steps):
        o.step()
    st = o.state()
    bodies = o.rigid()
    o.close()
    order = np.argsort(st["id"])
    return {k: v[order] for k, v in st.items()}, bodies, sc


def test_zero_inverse_inertia_freezes_rotation(oracle_lib):
    """Literal UnifiedPhysics.cpp:150: the inverse inertia is written into a
    temporary, so every body keeps omega = 0 and its initial orientation;
    with the inverse stored (this build) the bodies rotate under the
    torques of the fluid and of each other."""
    _, (pos0, vel0, om0, q0), _ = _run(0)
    _, (pos1, vel1, om1, q1), _ = _run(pyoracle.LITERAL_ZERO_INVERSE_INERTIA)
    assert np.all(om1 == 0) and np.all(q1[:, 0] == 1) and np.all(q1[:, 1:] == 0)
    assert np.abs(om0).max() > 1e-3
    # the linear motion does not depend on the inertia within the first steps'
    # contacts to more than a small fraction of the speed
    assert np.abs(vel1 - vel0).max() <= 0.5 * max(np.abs(vel0).max(), 1e-3)


def test_own_body_spring_adds_only_internal_forces(oracle_lib):
    """Literal UnifiedPhysics.cpp:5300-5311: the spring-damper also acts
    between particles of one body. Those pair forces cancel in the body's
    force sum (linear motion unchanged to rounding), but their damping part
    acts along v_ij = omega x r_ij, perpendicular to r_ij, and adds a torque
    that brakes each body's spin."""
    _, (pos0, vel0, om0, q0), _ = _run(0)
    _, (pos1, vel1, om1, q1), _ = _run(pyoracle.LITERAL_OWN_BODY_SPRING)
    assert np.abs(vel1 - vel0).max() <= 1e-3 * max(np.abs(vel0).max(), 1e-3)
    assert not np.array_equal(om0, om1)
    assert np.linalg.norm(om1, axis=1).sum() < np.linalg.norm(om0, axis=1).sum()


def test_tangential_only_granular_contact_lets_grains_interpenetrate(oracle_lib):
    """Literal UnifiedPhysics.cpp:3276-3287: grains add only F_t (and bound
    friction by mu * f_n with the signed f_n). Without the normal force the
    pile has no contact stiffness: after the same steps its grains sit
    closer together than with F_n + F_t (this build)."""
    st0, _, sc = _run(0)
    st1, _, _ = _run(pyoracle.LITERAL_GRANULAR_TANGENTIAL_ONLY)
    g = sc.type == GRANULAR
    assert not np.array_equal(st0["pos"][g], st1["pos"][g])

    def min_gap(pos):
        x = pos[g, :3].astype(np.float64)
        d = np.sqrt(((x[:, None, :] - x[None, :, :]) ** 2).sum(-1))
        np.fill_diagonal(d, np.inf)
        return d.min(1).mean()

    assert min_gap(st1["pos"]) < min_gap(st0["pos"])
    # liquid and rigid particles see grains only through their positions:
    # the difference starts at the grains
    r = sc.type == RIGID
    assert np.abs(st1["pos"][g, :3] - st0["pos"][g, :3]).max() >= np.abs(
        st1["pos"][r, :3] - st0["pos"][r, :3]).max()
