"""Seeded synthetic scenes (the reference builds its scenes in
src/sceneConfigure/Scene.cpp; no dataset is involved).

Random numbers come from an in-repo splitmix64 stream (the reference's
`drand48` macro is integer division and always 0, src/sceneConfigure/global.h:12),
so the oracle and the device path consume identical arrays.

Every generator returns a `Scene`: float32 positions/velocities (n x 4),
int32 types, and the upf parameters (not yet derived).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from ._abi import (FLAG_BOUNDARY_PRESSURE, FLAG_PENALTY_WALLS, FLAG_SURFACE_TENSION,
                   FROZEN, GRANULAR, LIQUID, METHOD_PCISPH, METHOD_WCSPH, RIGID, UpfParams)

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """The first n outputs of splitmix64 started at seed + stream * 2^32."""
    with np.errstate(over="ignore"):
        s0 = np.uint64((seed + (stream << 32)) & 0xFFFFFFFFFFFFFFFF)
        z = s0 + _GOLDEN * np.arange(1, n + 1, dtype=np.uint64)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """Uniform doubles in [0, 1)."""
    return (splitmix64(seed, n, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def normal(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """Standard normals (Box-Muller over two splitmix64 streams)."""
    u1 = uniform(seed, n, 2 * stream + 1)
    u2 = uniform(seed, n, 2 * stream + 2)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


@dataclasses.dataclass
class Scene:
    name: str
    params: UpfParams
    pos: np.ndarray    # (n, 4) float32
    vel: np.ndarray    # (n, 4) float32
    type: np.ndarray   # (n,) int32
    body: np.ndarray | None = None  # (n,) int32 body index of RIGID particles, -1 otherwise
    num_bodies: int = 0

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @property
    def n_fluid(self) -> int:
        return int(np.count_nonzero(self.type == LIQUID))

    @property
    def n_boundary(self) -> int:
        return int(np.count_nonzero(self.type == FROZEN))


def default_params() -> UpfParams:
    """UnifiedConstants::UnifiedConstants defaults
    (src/sceneConfigure/UnifiedConstants.cpp:7-159), before derivation."""
    p = UpfParams()
    p.method = METHOD_PCISPH
    p.flags = FLAG_SURFACE_TENSION | FLAG_PENALTY_WALLS
    p.particle_spacing = np.float32(1.0 / 40.0)
    p.rest_density = 1000.0
    p.gas_constant = 2000.0
    p.gamma = 7.0
    p.viscosity = 1.0
    p.gravity = 9.81
    p.dt = 0.0012
    p.density_error_fudge = -1.0
    p.max_density_error = 1.0
    p.min_loops = 3
    p.max_loops = 50
    p.surface_tension_gamma = 0.3
    p.surface_adhesion_beta = 0.0
    p.spring_coefficient = 300.0
    p.spring_coefficient_boundary = 300.0
    p.damping_coefficient = 0.5
    p.terminal_speed = 20.0
    p.granular_kr = 1.0
    p.granular_kd = 0.1
    p.granular_kt = 100.0
    p.granular_mu = 0.4
    p.zindex_extent[:] = (2.0, 2.0, 1.5)
    p.max_neighbors = 128
    return p


def _lattice(nx, ny, nz, spacing, origin, jitter, seed, stream=0):
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    g = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64)
    n = g.shape[0]
    pos = np.asarray(origin, np.float64)[None, :] + g * spacing
    if jitter:
        pos = pos + (uniform(seed, 3 * n, stream).reshape(n, 3) * 2.0 - 1.0) * jitter
    return pos


def box_shell(lo, hi, spacing, layers):
    """Boundary particles: `layers` lattice shells at `spacing` covering the six
    faces of the box [lo, hi] (the first shell on the faces, further shells
    outside)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    out = []
    for k in range(layers):
        a = lo - k * spacing
        b = hi + k * spacing
        cnt = np.rint((b - a) / spacing).astype(int) + 1
        ix, iy, iz = np.meshgrid(np.arange(cnt[0]), np.arange(cnt[1]), np.arange(cnt[2]), indexing="ij")
        on = ((ix == 0) | (ix == cnt[0] - 1) | (iy == 0) | (iy == cnt[1] - 1) |
              (iz == 0) | (iz == cnt[2] - 1))
        g = np.stack([ix[on], iy[on], iz[on]], axis=1).astype(np.float64)
        out.append(a[None, :] + g * spacing)
    return np.concatenate(out, axis=0)


def _pack(name, params, fluid, boundary, vel_fluid=None):
    nf, nb = fluid.shape[0], boundary.shape[0]
    pos = np.zeros((nf + nb, 4), np.float32)
    pos[:nf, :3] = fluid
    pos[nf:, :3] = boundary
    vel = np.zeros_like(pos)
    if vel_fluid is not None:
        vel[:nf, :3] = vel_fluid
    typ = np.concatenate([np.full(nf, LIQUID, np.int32), np.full(nb, FROZEN, np.int32)])
    return Scene(name, params, pos, vel, typ)


def _set_box(p, container_lo, container_hi):
    r = np.float32(p.particle_spacing) * np.float32(0.5)
    p.container_min[:] = container_lo
    p.container_max[:] = container_hi
    p.collision_min[:] = [np.float32(v) + r for v in container_lo]
    p.collision_max[:] = [np.float32(v) - r for v in container_hi]


def wcsph_dam(n_side=32, seed=1234, box=1.0) -> Scene:
    """WCSPH dam break, the CPU path's own method: n_side^3 fluid particles on a
    lattice (spacing 0.02, jitter U(+-0.002)) in the corner of a box x box x box
    container walled by one layer of boundary particles at the same spacing.
    h = 0.04, rest density 1000, stiffness 1000, gamma 7, viscosity 0.01,
    gravity 9.81, dt = 1e-3."""
    p = default_params()
    p.method = METHOD_WCSPH
    p.flags = 0
    s = 0.02
    p.particle_spacing = s
    p.support_radius = 0.04
    p.gas_constant = 1000.0
    p.gamma = 7.0
    p.viscosity = 0.01
    p.dt = 1e-3
    lo = np.array([0.04, 0.04, 0.04])
    hi = lo + box
    _set_box(p, lo, hi)
    p.zindex_extent[:] = (2.0, 2.0, 1.5)
    fluid = _lattice(n_side, n_side, n_side, s, lo + s, 0.002, seed)
    boundary = box_shell(lo, hi, s, 1)
    return _pack("wcsph_dam_%d" % n_side, p, fluid, boundary)


def pcisph_dam(nx=128, ny=128, nz=64, seed=4321, box=(2.0, 1.3, 1.3), layers=2,
               spacing=0.01) -> Scene:
    """PCISPH dam break: nx*ny*nz fluid particles (default 128 x 128 x 64 =
    1,048,576; spacing 0.01, jitter
    +-0.001) in the corner of a box[0] x box[1] x box[2] container with
    `layers` shells of boundary particles. h = 2 * spacing, rest density
    1000, 1% density error threshold, 3-50 iterations, dt = 5e-4."""
    p = default_params()
    p.method = METHOD_PCISPH
    p.flags = FLAG_SURFACE_TENSION | FLAG_PENALTY_WALLS | FLAG_BOUNDARY_PRESSURE
    s = spacing
    p.particle_spacing = s
    p.support_radius = 2.0 * s
    p.dt = 5e-4
    p.viscosity = 1.0
    lo = np.array([2 * s, 2 * s, 2 * s])
    hi = lo + np.asarray(box, np.float64)
    _set_box(p, lo, hi)
    ext = 1024.0 * (s / 5.0)  # 5 grid cells per spacing: 2.048 m at 0.01
    p.zindex_extent[:] = (ext, ext, ext)
    fluid = _lattice(nx, ny, nz, s, lo + s, 0.1 * s, seed)
    boundary = box_shell(lo, hi, s, layers)
    return _pack("pcisph_dam_%dx%dx%d" % (nx, ny, nz), p, fluid, boundary)


def _random_rotation(u):
    """Rotation matrix of a uniformly random unit quaternion (Shoemake) from
    three uniforms."""
    u1, u2, u3 = u
    q = np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)])
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


# ---------------------------------------------------------------- closed meshes
# Triangle meshes (n x 9 float32: three corners per row, counter-clockwise
# seen from outside) for the mesh voxeliser (upf_mesh_particles), which
# fills a closed mesh the way the reference fills its OBJ models.

def mesh_icosphere(radius=0.1, subdiv=2, center=(0.0, 0.0, 0.0)) -> np.ndarray:
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(x, np.float64) / np.linalg.norm(x) for x in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        mid = {}

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                x = v[a] + v[b]
                v.append(x / np.linalg.norm(x))
                mid[k] = len(v) - 1
            return mid[k]
        f = [g for a, b, c in f for g in ((a, m(a, b), m(c, a)), (b, m(b, c), m(a, b)), (c, m(c, a), m(b, c)),
                                          (m(a, b), m(b, c), m(c, a)))]
    pts = np.array(v) * radius + np.asarray(center, np.float64)
    return pts[np.array(f)].reshape(-1, 9).astype(np.float32)


def mesh_torus(big=0.1, small=0.035, nu=24, nv=12, center=(0.0, 0.0, 0.0)) -> np.ndarray:
    u = 2 * np.pi * np.arange(nu) / nu
    w = 2 * np.pi * np.arange(nv) / nv
    def p(i, j):
        a, b = u[i % nu], w[j % nv]
        return ((big + small * np.cos(b)) * np.cos(a), small * np.sin(b), (big + small * np.cos(b)) * np.sin(a))
    tris = []
    for i in range(nu):
        for j in range(nv):
            q00, q10, q11, q01 = p(i, j), p(i + 1, j), p(i + 1, j + 1), p(i, j + 1)
            tris += [q00 + q01 + q11, q00 + q11 + q10]
    return (np.array(tris) + np.tile(np.asarray(center, np.float64), 3)).astype(np.float32)


def mesh_box(half=(0.1, 0.06, 0.08), rotation_seed=None, center=(0.0, 0.0, 0.0)) -> np.ndarray:
    c = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float64) * np.asarray(half)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    if rotation_seed is not None:
        c = c @ _random_rotation(uniform(rotation_seed, 3)).T
    c = c + np.asarray(center, np.float64)
    tris = [c[[a, b, d]].ravel() for a, b, cc, d in quads] + [c[[b, cc, d]].ravel() for a, b, cc, d in quads]
    return np.array(tris).astype(np.float32)


def write_obj(path, tri9) -> None:
    """A Wavefront OBJ file the reference's ObjLoader reads: one vertex line
    per corner (9 significant digits: floats read back exactly), one texture
    coordinate and one normal line (its face lines index both), faces as
    v/vt/vn corners."""
    t = np.asarray(tri9, np.float32).reshape(-1, 3)
    with open(path, "w") as f:
        f.write("# closed triangle mesh, %d faces\n" % (len(t) // 3))
        for x, y, z in t:
            f.write("v %.9g %.9g %.9g\n" % (x, y, z))
        f.write("vt 0 0\nvn 0 0 1\n")
        for k in range(len(t) // 3):
            f.write("f %d/1/1 %d/1/1 %d/1/1\n" % (3 * k + 1, 3 * k + 2, 3 * k + 3))


def sample_sphere(r, n):
    """n points on a sphere of radius r (Fibonacci lattice)."""
    k = np.arange(n) + 0.5
    phi = np.arccos(1 - 2 * k / n)
    theta = np.pi * (1 + 5 ** 0.5) * k
    return r * np.stack([np.cos(theta) * np.sin(phi), np.sin(theta) * np.sin(phi), np.cos(phi)], axis=1)


def sample_box(r, n):
    """About n points on the surface of a cube of half-edge r (a k x k grid per face)."""
    k = max(2, int(round(np.sqrt(n / 6.0))))
    g = (np.arange(k) + 0.5) / k * 2 * r - r
    a, b = np.meshgrid(g, g, indexing="ij")
    a, b = a.ravel(), b.ravel()
    faces = []
    for axis in range(3):
        for sgn in (-r, r):
            p = np.zeros((a.size, 3))
            p[:, axis] = sgn
            p[:, (axis + 1) % 3] = a
            p[:, (axis + 2) % 3] = b
            faces.append(p)
    return np.concatenate(faces)


def sample_torus(r, n):
    """About n points on a torus of major radius r and minor radius r/3."""
    a = r / 3.0
    nu = max(8, int(round(np.sqrt(n * r / a))))
    nv = max(4, int(round(n / nu)))
    u = (np.arange(nu) + 0.5) / nu * 2 * np.pi
    v = (np.arange(nv) + 0.5) / nv * 2 * np.pi
    uu, vv = np.meshgrid(u, v, indexing="ij")
    uu, vv = uu.ravel(), vv.ravel()
    return np.stack([(r + a * np.cos(vv)) * np.cos(uu), (r + a * np.cos(vv)) * np.sin(uu), a * np.sin(vv)], axis=1)


def coupling_scene(fluid=(128, 64, 64), granular=(64, 32, 64), n_bodies=16, seed=99, box=(2.0, 1.3, 1.3),
                   radius=(0.05, 0.15), samples=(2000, 8000), spacing=0.01, layers=2) -> Scene:
    """Rigid-fluid coupling plus granular: a PCISPH fluid block at one end of
    the container, a granular pile (friction 0.5) at the other, and
    `n_bodies` rigid bodies (spheres, cubes and tori cycling) with radii
    uniform in `radius`, surface-sampled with 2k-8k Akinci boundary particles
    each (half the fluid spacing, clamped to `samples`), random orientations
    and positions above the fluid and the pile."""
    p = default_params()
    p.method = METHOD_PCISPH
    p.flags = FLAG_SURFACE_TENSION | FLAG_PENALTY_WALLS | FLAG_BOUNDARY_PRESSURE
    s = spacing
    p.particle_spacing = s
    p.support_radius = 2.0 * s
    p.dt = 5e-4
    p.viscosity = 1.0
    # grain contacts stiff enough to hold a pile at this dt (k omega dt < 1)
    p.granular_kr = 200.0
    p.granular_kd = 0.5
    p.granular_kt = 10.0
    p.granular_mu = 0.5
    p.max_neighbors = 160
    lo = np.array([2 * s, 2 * s, 2 * s])
    hi = lo + np.asarray(box, np.float64)
    _set_box(p, lo, hi)
    ext = 1024.0 * (s / 5.0)
    p.zindex_extent[:] = (ext, ext, ext)
    fl = _lattice(*fluid, s, lo + s, 0.1 * s, seed)
    gx = box[0] - (granular[0] + 1) * s
    gr = _lattice(*granular, s, lo + np.array([gx, s, s]), 0.1 * s, seed, stream=1)
    u = uniform(seed, 8 * n_bodies, stream=2).reshape(n_bodies, 8)
    ds = 0.5 * s
    bodies, body_ids = [], []
    top = max(fluid[1], granular[1]) * s + lo[1]
    cols = int(np.ceil(np.sqrt(n_bodies)))
    for b in range(n_bodies):
        r = radius[0] + (radius[1] - radius[0]) * u[b, 0]
        shape = b % 3
        area = (4 * np.pi * r * r, 24 * r * r, 4 * np.pi ** 2 * r * (r / 3.0))[shape]
        n = int(np.clip(round(area / ds ** 2), samples[0], samples[1]))
        pts = (sample_sphere, sample_box, sample_torus)[shape](r, n)
        pts = pts @ _random_rotation(u[b, 1:4]).T
        # slots on a grid above the fluid and the pile
        cx = lo[0] + (b % cols + 0.5) / cols * box[0]
        cz = lo[2] + ((b // cols) % cols + 0.5) / cols * box[2]
        # between the top of the fluid/pile and the ceiling, clear of both
        ylo, yhi = top + r + 2 * s, hi[1] - r - 3 * s
        cy = ylo + (yhi - ylo) * (0.25 + 0.5 * u[b, 4]) if yhi > ylo else 0.5 * (ylo + yhi)
        bodies.append(pts + np.array([cx, cy, cz]))
        body_ids.append(np.full(pts.shape[0], b, np.int32))
    rig = np.concatenate(bodies)
    bid = np.concatenate(body_ids)
    bnd = box_shell(lo, hi, s, layers)
    pos = np.zeros((fl.shape[0] + gr.shape[0] + rig.shape[0] + bnd.shape[0], 4), np.float32)
    parts = [fl, gr, rig, bnd]
    types = [LIQUID, GRANULAR, RIGID, FROZEN]
    typ, body = [], []
    o = 0
    for arr, t in zip(parts, types):
        pos[o:o + arr.shape[0], :3] = arr
        typ.append(np.full(arr.shape[0], t, np.int32))
        body.append(bid if t == RIGID else np.full(arr.shape[0], -1, np.int32))
        o += arr.shape[0]
    vel = np.zeros_like(pos)
    return Scene("coupling_%d" % fl.shape[0], p, pos, vel, np.concatenate(typ), np.concatenate(body), n_bodies)


def batch_scene(n, extent, seed, stream=0) -> Scene:
    """One scene of a batch: n liquid particles in a lattice block (jitter
    +-10% of the spacing) filling the lower half (in x) of a box of the given
    extents, walls by the collision box and penalty forces. The spacing
    follows from n and the box; h = 2 * spacing, dt = 2.5e-4 * spacing / 0.01
    (clamped to [5e-5, 1e-3]: the time step at which the collapse of these
    columns, up to 1.9 m high and without boundary particles, keeps every
    step within the 1% density error), the Morton grid spans the box."""
    lx, ly, lz = (float(v) for v in extent)
    s = (0.5 * lx * 0.8 * ly * lz / n) ** (1.0 / 3.0)
    nx = max(1, int(0.5 * lx / s))
    nz = max(1, int(lz / s) - 1)
    ny = int(np.ceil(n / (nx * nz)))
    while ny * s > 0.95 * ly - 2 * s and s > 1e-4:  # keep the block inside the box
        s *= 0.97
        nx = max(1, int(0.5 * lx / s))
        nz = max(1, int(lz / s) - 1)
        ny = int(np.ceil(n / (nx * nz)))
    p = default_params()
    p.method = METHOD_PCISPH
    p.flags = FLAG_SURFACE_TENSION | FLAG_PENALTY_WALLS
    p.particle_spacing = s
    p.support_radius = 2.0 * s
    p.dt = float(np.clip(2.5e-4 * s / 0.01, 5e-5, 1e-3))
    p.viscosity = 1.0
    lo = np.array([2 * s, 2 * s, 2 * s])
    hi = lo + np.array([lx, ly, lz])
    _set_box(p, lo, hi)
    ext = max(lx, ly, lz) + 4 * s
    p.zindex_extent[:] = (ext, ext, ext)
    pts = _lattice(nx, ny, nz, s, lo + s, 0.1 * s, seed, stream)
    # lattice order is x-major: keep the first n in y-layers from the bottom
    order = np.lexsort((pts[:, 2], pts[:, 0], pts[:, 1]))
    fluid = pts[order[:n]]
    return _pack("batch_%d" % n, p, fluid, np.zeros((0, 3)))


def batch_scenes(num=256, seed=2024, counts=(2048, 65536), extents=(0.5, 2.0)) -> list:
    """A batch of independent scenes: particle counts log-uniform in `counts`,
    box extents uniform in `extents` per axis, from the seed."""
    u = uniform(seed, 4 * num, stream=7).reshape(num, 4)
    lo, hi = np.log(counts[0]), np.log(counts[1])
    out = []
    for k in range(num):
        n = int(round(np.exp(lo + (hi - lo) * u[k, 0])))
        ext = extents[0] + (extents[1] - extents[0]) * u[k, 1:4]
        out.append(batch_scene(n, ext, seed + 17 * k, stream=k + 1))
    return out


def adjoint_scene(nx=32, ny=32, nz=64, seed=77, spacing=0.01, dt=1e-3, vel_sigma=0.1) -> Scene:
    """The differentiation workload: an nx x ny x nz liquid block (default
    65,536; jitter +-10% of the spacing) in the middle of a 2 m box it does
    not reach within 200 steps, initial velocities N(0, vel_sigma) m/s per
    component from the seed, h = 2 * spacing, dt, no surface tension or wall
    forces (the trajectory the adjoint differentiates)."""
    p = default_params()
    p.method = METHOD_PCISPH
    p.flags = 0
    s = spacing
    p.particle_spacing = s
    p.support_radius = 2.0 * s
    p.dt = dt
    p.viscosity = 1.0
    lo = np.array([0.02, 0.02, 0.02])
    hi = lo + 2.0
    _set_box(p, lo, hi)
    p.zindex_extent[:] = (2.048, 2.048, 2.048)
    block = np.array([nx, ny, nz], np.float64) * s
    origin = lo + 1.0 - 0.5 * block + np.array([0.0, 0.5, 0.0])  # above the centre: it falls during the run
    fluid = _lattice(nx, ny, nz, s, origin, 0.1 * s, seed)
    vel = normal(seed, 3 * fluid.shape[0], stream=5).reshape(-1, 3) * vel_sigma
    return _pack("adjoint_%dx%dx%d" % (nx, ny, nz), p, fluid, np.zeros((0, 3)), vel_fluid=vel)


def small_coupling(seed=5) -> Scene:
    """A small coupling scene (oracle-sized): 12^3 fluid, an 8x4x8 pile and
    three small bodies."""
    return coupling_scene(fluid=(12, 12, 12), granular=(8, 4, 8), n_bodies=3, seed=seed, box=(0.4, 0.35, 0.25),
                          radius=(0.03, 0.05), samples=(150, 400))


def small_pcisph(n_side=12, seed=7, layers=2, box=(0.3, 0.2, 0.2)) -> Scene:
    """A small PCISPH dam (oracle-sized) with the same physics as pcisph_dam."""
    return pcisph_dam(n_side, n_side, n_side, seed=seed, box=box, layers=layers)


def small_wcsph(n_side=12, seed=11) -> Scene:
    """A small WCSPH dam (oracle-sized) with the same physics as wcsph_dam."""
    return wcsph_dam(n_side, seed=seed, box=0.4)
