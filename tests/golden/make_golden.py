"""Generate the golden fixtures in tests/golden/ from the reference's own CPU
code (src/cpu/zIndex.cpp, src/cpu/WeightingKernel.cpp,
src/sceneConfigure/UnifiedConstants.cpp, src/cpu/RigidBody.cpp,
src/cpu/Matrix3x3.cpp, src/cpu/UnifiedIO.cpp), compiled by oracle/Makefile into
oracle/_ref/libupfref.so. Run in a checkout where the reference source tree
is available:

    make -C oracle ref REF=/path/to/reference
    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py step     # reference_step.npz only

reference_step.npz comes from the reference's CPU steps themselves
(src/cpu/UnifiedPhysics.cpp's step functions, extracted unchanged into
oracle/_ref/libupfref_physics.so). The reference has no tests, fixtures or
known-answer vectors of its own; these files pin the oracle (and through it
the device path) to the reference's tables, constants and steps.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402

# support radii: the reference default (2.00002 * 1/40), the two benchmark
# scenes, and two arbitrary ones
H_VALUES = [np.float32(2.5e-2 * 2.0 * 1.00001), np.float32(0.04), np.float32(0.02), np.float32(0.0123),
            np.float32(0.0375)]


def fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def main():
    if not pyoracle.ref_available():
        raise SystemExit("oracle/_ref/libupfref.so missing: make -C oracle ref")
    if sys.argv[1:] == ["step"]:  # only reference_step.npz
        step = step_vectors()
        np.savez_compressed(os.path.join(HERE, "reference_step.npz"), **step)
        print("wrote", os.path.join(HERE, "reference_step.npz"))
        return
    R = pyoracle.ref()
    out = {}
    tab = np.zeros((1024, 3), np.uint32)
    R.ref_morton_table(tab.ctypes.data_as(C.POINTER(C.c_uint32)))
    out["morton_table"] = tab
    luts = np.zeros((len(H_VALUES), 5, 301), np.float32)
    for k, h in enumerate(H_VALUES):
        R.ref_luts(C.c_float(h), fp(luts[k]))
    out["lut_h"] = np.array(H_VALUES, np.float32)
    out["luts"] = luts
    # analytic kernels at sample distances for h = 0.02
    d = np.linspace(0.0, 0.021, 97).astype(np.float32)
    kv = np.zeros((d.size, 5), np.float32)
    for i, x in enumerate(d):
        R.ref_kernels(C.c_float(x), C.c_float(0.02), fp(kv[i]))
    out["kernel_dist"] = d
    out["kernel_values_h002"] = kv
    # BoxQuery ranges for seeded boxes and block sizes
    rng = np.random.default_rng(20240601)
    boxes, sizes, firsts, lasts, counts = [], [], [], [], []
    for bs in (4, 8, 16, 32, 64):
        for _ in range(40):
            lo = rng.integers(0, 1000, 3)
            ext = rng.integers(0, 3 * bs, 3)
            hi = np.minimum(lo + ext, 1023)
            a = lo.astype(np.uint16)
            b = hi.astype(np.uint16)
            f = np.zeros(4096, np.uint32)
            l = np.zeros(4096, np.uint32)
            n = R.ref_box_query(bs, a.ctypes.data_as(C.POINTER(C.c_uint16)), b.ctypes.data_as(C.POINTER(C.c_uint16)),
                                f.ctypes.data_as(C.POINTER(C.c_uint32)), l.ctypes.data_as(C.POINTER(C.c_uint32)), 4096)
            boxes.append(np.concatenate([a, b]))
            sizes.append(bs)
            counts.append(n)
            firsts.append(f[:n])
            lasts.append(l[:n])
    out["bq_boxes"] = np.array(boxes, np.uint16)
    out["bq_block"] = np.array(sizes, np.uint32)
    out["bq_count"] = np.array(counts, np.uint32)
    out["bq_first"] = np.concatenate(firsts)
    out["bq_last"] = np.concatenate(lasts)
    # ZIndex::SetBlockSize rounding
    sz = np.arange(0, 130, dtype=np.int32)
    out["block_size_in"] = sz
    out["block_size_out"] = np.array([R.ref_block_size(int(s)) for s in sz], np.uint32)
    # UnifiedConstants defaults
    cst = np.zeros(64, np.float32)
    R.ref_default_constants(fp(cst))
    out["default_constants"] = cst[:41]
    np.savez_compressed(os.path.join(HERE, "reference_tables.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_tables.npz"))
    rigid = rigid_vectors(R)
    np.savez_compressed(os.path.join(HERE, "reference_rigid.npz"), **rigid)
    print("wrote", os.path.join(HERE, "reference_rigid.npz"))
    io = io_vectors()
    np.savez_compressed(os.path.join(HERE, "reference_io.npz"), **io)
    print("wrote", os.path.join(HERE, "reference_io.npz"))
    mesh = mesh_vectors()
    np.savez_compressed(os.path.join(HERE, "reference_mesh.npz"), **mesh)
    print("wrote", os.path.join(HERE, "reference_mesh.npz"))
    step = step_vectors()
    np.savez_compressed(os.path.join(HERE, "reference_step.npz"), **step)
    print("wrote", os.path.join(HERE, "reference_step.npz"))


def random_body_state(rng):
    """A body state of 47 floats (mass, pos, vel, P, L, omega, q, rot,
    inv_inertia_local, inv_inertia_world): unit-ish quaternion, its rotation
    matrix, a symmetric positive definite inverse inertia."""
    st = np.zeros(47, np.float32)
    st[0] = rng.uniform(0.01, 10.0)
    st[1:4] = rng.uniform(-1, 1, 3)
    st[4:7] = rng.normal(0, 1, 3)
    st[7:10] = rng.normal(0, 1, 3) * st[0]
    st[10:13] = rng.normal(0, 0.01, 3)
    st[13:16] = rng.normal(0, 1, 3)
    q = rng.normal(0, 1, 4)
    q = q / np.linalg.norm(q) * (1.0 + rng.normal(0, 1e-4))
    st[16:20] = q
    w, x, y, z = st[16:20].astype(np.float64)
    st[20:29] = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                          [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                          [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]]).ravel()
    a = rng.normal(0, 1, (3, 3))
    st[29:38] = (np.linalg.inv(a @ a.T + 0.1 * np.eye(3)) * 100.0).ravel()
    return st


def rigid_vectors(R):
    """RigidBody::UpdateMomenta + PerformStep + UpdateRotationMatrix on seeded
    states (terminal-momentum clamp active in some), and
    Matrix3x3::CalculateInverse on seeded inertia tensors."""
    fp_t = C.POINTER(C.c_float)
    R.ref_rigid_body_step.argtypes = [fp_t, fp_t, fp_t, C.c_float, C.c_float]
    R.ref_inverse3.argtypes = [fp_t, fp_t]
    R.ref_inverse3.restype = C.c_int
    rng = np.random.default_rng(20240917)
    n = 256
    st_in = np.stack([random_body_state(rng) for _ in range(n)])
    force = rng.normal(0, 5, (n, 3)).astype(np.float32)
    torque = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    dt = rng.choice(np.array([5e-4, 1e-3, 1e-2], np.float32), n).astype(np.float32)
    terminal = rng.choice(np.array([20.0, 0.5], np.float32), n).astype(np.float32)
    st_out = st_in.copy()
    for k in range(n):
        R.ref_rigid_body_step(fp(st_out[k]), fp(force[k]), fp(torque[k]), C.c_float(dt[k]), C.c_float(terminal[k]))
    mats = np.zeros((64, 9), np.float32)
    for k in range(64):
        pts = rng.normal(0, 0.1, (rng.integers(4, 40), 3))
        rr = (pts * pts).sum(1)
        inertia = sum(np.eye(3) * r2 - np.outer(p, p) for p, r2 in zip(pts, rr)) * 0.001
        mats[k] = inertia.ravel()
    inv = np.zeros_like(mats)
    ok = np.array([R.ref_inverse3(fp(mats[k]), fp(inv[k])) for k in range(64)], np.int32)
    return {"body_in": st_in, "body_force": force, "body_torque": torque, "body_dt": dt,
            "body_terminal_speed": terminal, "body_out": st_out, "inertia": mats, "inertia_inverse": inv,
            "inertia_ok": ok}


def io_positions(rng, n):
    """Positions spanning what the text writers must format: ordinary values,
    lattice values, very small and very large exponents, integers, denormals,
    signed zeros, the float extremes, infinities and NaNs."""
    pos = rng.uniform(-1, 1, (n, 4)).astype(np.float32)
    k = n // 8
    pos[:k, :3] = rng.normal(size=(k, 3))
    pos[k:2 * k, :3] = np.round(rng.uniform(0, 2, (k, 3)) / 0.01) * 0.01
    pos[2 * k:3 * k, :3] = rng.normal(size=(k, 3)) * 10.0 ** rng.integers(-30, 30, (k, 3))
    pos[3 * k:4 * k, :3] = rng.integers(-100000, 100000, (k, 3))
    pos[4 * k:5 * k, :3] = rng.uniform(-1e-3, 1e-3, (k, 3))
    special = np.array([0.0, -0.0, 1e-45, -3e-44, 1.17549435e-38, 3.4028235e38, -3.4028235e38, np.inf, -np.inf,
                        np.nan, -np.nan, 0.1, 1.0 / 3.0, 123456789.0, 1e-7], np.float32)
    rows = 5 * k + np.arange(special.size)
    pos[rows, 0] = special
    pos[rows, 1] = special[::-1]
    pos[rows, 2] = -special
    return pos.astype(np.float32)


def io_reader_text(rng, n):
    """A file in the format ReadInFluidParticlesPCISPH reads, written with
    varied number spellings and white space."""
    fmts = ["%.9g", "%e", "%+.3f", "%g", "%.2E", "%.0f.", "%.12g"]
    seps = [" ", "  ", "\t", " \t ", "\n"]
    vals = np.concatenate([rng.normal(size=(n, 8)) * 10.0 ** rng.integers(-8, 8, (n, 8)),
                           rng.integers(-3, 8, (n, 1))], axis=1)
    out = ["  %d\n" % n]
    for i in range(n):
        fields = []
        for j, col in enumerate([0, 1, 2, 8, 3, 4, 5, 6, 7]):
            if col == 8:
                t = int(vals[i, 8])
                fields.append(rng.choice(["%d", "+%d", "%03d"]) % t if t >= 0 else "%d" % t)
            else:
                fields.append(rng.choice(fmts) % float(vals[i, col]))
        special = rng.integers(0, 12)
        if special == 0:
            fields[0] = "-0"
        elif special == 1:
            fields[4] = ".5"
        elif special == 2:
            fields[7] = "1e-45"
        elif special == 3:
            fields[8] = "5e3"
        line = fields[0]
        for f in fields[1:]:
            line += rng.choice(seps) + f
        out.append(line + "\n")
    return "".join(out)


def io_vectors():
    """Inputs to the reference's text writers (UnifiedIO.cpp:14-152) and the
    bytes it wrote; a reader file and the reference reader's values
    (UnifiedIO.cpp:154-220)."""
    import tempfile
    rng = np.random.default_rng(20241203)
    n = 400
    pos = io_positions(rng, n)
    types = rng.choice(np.array([0, 1, 2, 3, 6], np.int32), n, p=[0.15, 0.05, 0.6, 0.1, 0.1]).astype(np.int32)
    nl = int(np.count_nonzero(types == 2))
    nr = int(np.count_nonzero((types == 0) | (types == 6)))
    text = io_reader_text(rng, 300)
    with tempfile.TemporaryDirectory() as d:
        liquid = pyoracle.ref_io_write("liquid", d, pos, types, nl)
        rigid = pyoracle.ref_io_write("rigid", d, pos, types, nr)
        positions = pyoracle.ref_io_write("positions", d, pos)
        path = os.path.join(d, "fluid_in.txt")
        with open(path, "w") as f:
            f.write(text)
        parsed = pyoracle.ref_io_read_pcisph(path)
    out = {"pos": pos, "type": types, "num_liquid": np.int32(nl), "num_rigid": np.int32(nr),
           "liquid_txt": np.frombuffer(liquid, np.uint8), "rigid_txt": np.frombuffer(rigid, np.uint8),
           "positions_txt": np.frombuffer(positions, np.uint8),
           "reader_txt": np.frombuffer(text.encode(), np.uint8)}
    out.update({"read_" + k: v for k, v in parsed.items()})
    return out


def mesh_cases():
    """Closed procedural meshes (the library's own, written as OBJ files) with
    the scale and spacing each is filled at: off the origin (the reference's
    lattice box always contains the origin), at negative coordinates,
    non-uniform scales, rotated, and an axis-aligned box whose faces lie on
    lattice planes (points that touch a face)."""
    from unifiedparticleframeworkcuda_b200 import scenes
    return [
        ("icosphere", scenes.mesh_icosphere(0.1, 2, (0.3, 0.2, 0.25)), (1.0, 1.0, 1.0), 0.012),
        ("torus", scenes.mesh_torus(center=(-0.2, 0.1, -0.3)), (1.5, 2.0, 1.0), 0.015),
        ("rotated_box", scenes.mesh_box(rotation_seed=5, center=(0.5, 0.4, 0.3)), (1.0, 1.0, 1.0), 0.013),
        ("icosphere_fine_scaled", scenes.mesh_icosphere(0.08, 3), (2.5, 2.5, 2.5), 0.025),
        ("torus_small", scenes.mesh_torus(0.05, 0.02, 32, 16, (0.02, 0.03, 0.01)), (0.5, 0.5, 0.5), 0.004),
        ("aligned_box", scenes.mesh_box((0.1, 0.05, 0.08), center=(0.1, 0.05, 0.08)), (1.0, 1.0, 1.0), 0.01),
    ]


def mesh_vectors():
    """The reference's ObjectLoader::LoadParticles (src/cpu/ObjectLoader.cpp,
    with its OBJ parser and Polygon tests) on each case's OBJ file."""
    import tempfile
    from unifiedparticleframeworkcuda_b200 import scenes
    R = pyoracle.ref()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, tri, scale, spacing in mesh_cases():
            path = os.path.join(d, name + ".obj")
            scenes.write_obj(path, tri)
            n = pyoracle.ref_obj_particles(path, scale, spacing)
            out[name + "_tri"] = tri
            out[name + "_scale"] = np.array(scale, np.float32)
            out[name + "_spacing"] = np.float32(spacing)
            out[name + "_pos"] = n
    return out


def rigid_contact_scene(seed=5):
    """The small coupling scene without its granular pile (the reference's
    coupling step has no grains), its three bodies moved into contact: a
    sphere half sunk into the top of the fluid, a cube beside it with half a
    spacing between their surfaces (spring-damper contacts), a torus resting
    on the collision box's floor (the rigid box force); liquid inside the
    sphere or within 0.75 spacing of a rigid particle removed. Key units of
    0.5 mm (the container is 0.42 m) keep every Morton key distinct over the
    steps the case runs."""
    from unifiedparticleframeworkcuda_b200 import GRANULAR, LIQUID, RIGID, scenes
    sc = scenes.small_coupling(seed=seed)
    p = sc.params
    s = float(p.particle_spacing)
    keep = sc.type != GRANULAR
    pos, typ, body = sc.pos[keep].copy(), sc.type[keep].copy(), sc.body[keep].copy()
    liq = typ == LIQUID
    top = pos[liq, 1].max()
    fluid_centre = pos[liq, :3].mean(0)
    floor = float(p.collision_min[1])
    pts = {b: pos[body == b, :3].astype(np.float64) for b in range(sc.num_bodies)}
    half = {b: (pts[b].max(0) - pts[b].min(0)) / 2 for b in pts}
    mid = {b: (pts[b].max(0) + pts[b].min(0)) / 2 for b in pts}
    t0 = np.array([fluid_centre[0], top, fluid_centre[2]])
    t1 = t0 + np.array([half[0][0] + half[1][0] + 0.5 * s, 0.0, 0.0])
    t2 = np.array([0.33, floor + half[2][1] + 0.2 * s, 0.15])
    for b, t in ((0, t0), (1, t1), (2, t2)):
        pos[body == b, :3] = (pts[b] - mid[b] + t).astype(np.float32)
    x = pos[:, :3].astype(np.float64)
    near = np.full(len(x), np.inf)
    for c in np.array_split(pos[typ == RIGID, :3].astype(np.float64), 8):
        near = np.minimum(near, np.sqrt(((x[:, None, :] - c[None]) ** 2).sum(-1)).min(1))
    inside = np.linalg.norm(x - t0, axis=1) < half[0].max()
    k = ~(liq & ((near < 0.75 * s) | inside))
    unit = 1024.0 * (s / 20.0)
    p.zindex_extent[:] = (unit, unit, unit)
    return scenes.Scene("rigid_contact", p, pos[k], np.zeros_like(pos[k]), typ[k], body[k], sc.num_bodies)


def step_cases():
    """(name, scene, params, method, steps, weighted boundary volumes).
    PCISPH: the dam in a box of frozen boundary particles, with the terms the
    reference's CPU coupling step applies to liquid particles (surface
    tension, penalty walls, and adhesion with Akinci boundary volumes); its
    boundary pressure term evaluates to zero (the pressure-gradient lookup is
    given the bin index as a distance, UnifiedPhysics.cpp:4245), so that
    flag is off. WCSPH: the pure-fluid step with wall weights and surface
    tension; it clamps every particle to the collision box, frozen ones
    included, so over several steps the box encloses the boundary (else
    clamped boundary particles come to share Morton keys, and the
    reference's unstable sort leaves their order unspecified), and one step
    runs with the scene's own box. Rigid: the coupling step on
    rigid_contact_scene with surface tension, penalty walls and adhesion, 20
    steps."""
    import unifiedparticleframeworkcuda_b200 as upf
    from unifiedparticleframeworkcuda_b200 import scenes
    st_pw = upf.FLAG_SURFACE_TENSION | upf.FLAG_PENALTY_WALLS
    ww_st = upf.FLAG_WALL_WEIGHT | upf.FLAG_SURFACE_TENSION
    cases = []

    def case(name, sc, flags, method, steps, wv, box=None):
        sc.params.flags = flags
        p = upf.derive_params(sc.params)
        if box is not None:
            for a in range(3):
                p.collision_min[a], p.collision_max[a] = box
        cases.append((name, sc, p, method, steps, wv))

    case("dam_st_pw", scenes.small_pcisph(), st_pw, "pcisph", 5, False)
    case("dam_st_pw_adh", scenes.small_pcisph(seed=29), st_pw | upf.FLAG_ADHESION, "pcisph", 3, True)
    case("wcsph_ww_st", scenes.small_wcsph(), ww_st, "wcsph", 1, False)
    case("wcsph_ww_st_box", scenes.small_wcsph(), ww_st, "wcsph", 5, False, box=(0.03, 0.45))
    case("rigid_contact", rigid_contact_scene(), st_pw | upf.FLAG_ADHESION, "pcisph", 20, False)
    return cases


def step_vectors():
    """The reference's own CPU step (CpuParticlePhysicsVersatileCouplingPCISPH
    or CpuParticlePhysicsPureFluidsSPH and the member functions they call,
    oracle/_ref/libupfref_physics.so) on each case: every particle's final
    position, velocity, density and pressure (PCISPH: predicted density and
    correction pressure) and type, by input index, the rigid bodies' final
    state, and the inputs."""
    from oracle import refstep
    out = {}
    for name, sc, p, method, steps, wv in step_cases():
        body = sc.body if sc.body is not None else np.full(sc.n, -1, np.int32)
        r = refstep.reference_steps(p, sc.pos, sc.vel, sc.type, steps, wv, method, body, sc.num_bodies)
        out[name + "_body_in"] = np.ascontiguousarray(body, np.int32)
        out[name + "_num_bodies"] = np.int32(sc.num_bodies)
        out[name + "_bodies"] = r["body"]
        order = np.argsort(r["id"])
        out[name + "_params"] = np.frombuffer(bytes(p), np.uint8)
        out[name + "_pos_in"] = np.ascontiguousarray(sc.pos, np.float32)
        out[name + "_vel_in"] = np.ascontiguousarray(sc.vel, np.float32)
        out[name + "_type_in"] = np.ascontiguousarray(sc.type, np.int32)
        out[name + "_steps"] = np.int32(steps)
        out[name + "_weighted_volumes"] = np.int32(1 if wv else 0)
        out[name + "_method"] = np.array(method)
        for k in ("pos", "vel", "density", "pressure", "type", "id"):
            out[name + "_" + k] = r[k][order]
    return out


if __name__ == "__main__":
    main()
