"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (liboracle.so)
and the reference pin library (_ref/libupfref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker. The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from unifiedparticleframeworkcuda_b200._abi import UpfParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REFLIB = os.path.join(HERE, "_ref", "libupfref.so")


_lib = None
_ref = None


def reference_dir() -> str:
    """The reference tree oracle/Makefile compiles the pins from: the
    environment's UPF_REFERENCE, else the recipe's default location."""
    r = subprocess.run(["make", "-s", "-C", HERE, "refdir"], capture_output=True, text=True, check=True)
    return r.stdout.strip()


def reference_present() -> bool:
    return os.path.isdir(os.path.join(reference_dir(), "src"))


def build(with_ref: bool = True) -> None:
    """Compile the oracle (and the reference pins when the reference tree is
    present) with oracle/Makefile."""
    targets = ["all"]
    if with_ref and reference_present():
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


# the reference's own rule where the restatement deviates (orc_set_reference_literal)
LITERAL_GRANULAR_TANGENTIAL_ONLY = 1
LITERAL_OWN_BODY_SPRING = 2
LITERAL_ZERO_INVERSE_INERTIA = 4
LITERAL_WCSPH_CLAMP_ALL = 8
LITERAL_FLOAT_RIGID_ASSEMBLY = 16
LITERAL_FLOAT_BODY_SUMS = 32
LITERAL_STALE_RIGID_KEYS = 64
LITERAL_STALE_RIGID_PREDICTED = 128


class StepInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("max_predicted_density", C.c_float),
        ("density_error_percent", C.c_float),
        ("max_neighbor_count", C.c_uint32),
        ("kinetic_energy", C.c_double),
        ("momentum", C.c_double * 3),
        ("iteration_max_density", C.c_float * 64),
    ]


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build(with_ref=False)
        L = C.CDLL(LIB)
        P = C.POINTER(UpfParams)
        fp, u32p, i32p = C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.POINTER(C.c_int32)
        L.orc_default_params.argtypes = [P]
        L.orc_params_derive.argtypes = [P]
        L.orc_params_derive.restype = C.c_int
        L.orc_density_error_factor.argtypes = [P, C.c_int]
        L.orc_density_error_factor.restype = C.c_double
        L.orc_build_luts.argtypes = [P, fp]
        L.orc_morton.argtypes = [P, C.c_float, C.c_float, C.c_float]
        L.orc_morton.restype = C.c_uint32
        L.orc_morton_table.argtypes = [u32p]
        L.orc_box_query.argtypes = [C.c_uint32, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), u32p, u32p, C.c_int]
        L.orc_box_query.restype = C.c_int
        L.orc_create.argtypes = [P, fp, fp, i32p, C.c_uint32, C.c_int, C.c_int]
        L.orc_create.restype = C.c_void_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.POINTER(StepInfo)]
        L.orc_step.restype = C.c_int
        L.orc_count.argtypes = [C.c_void_p]
        L.orc_count.restype = C.c_uint32
        L.orc_keep_fields.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_reference_literal.argtypes = [C.c_void_p, C.c_uint32]
        L.orc_set_reference_literal.restype = None
        L.orc_set_lagged.argtypes = [C.c_void_p, fp, fp, fp]
        L.orc_set_lagged.restype = None
        L.orc_get_lagged.argtypes = [C.c_void_p, fp, fp, fp]
        L.orc_get_lagged.restype = None
        L.orc_get.argtypes = [C.c_void_p, fp, fp, fp, fp, i32p, u32p, u32p]
        L.orc_get_step_fields.argtypes = [C.c_void_p, fp, fp, fp, fp, fp, fp, u32p]
        L.orc_neighbors.argtypes = [C.c_void_p, u32p, u32p, C.c_uint32]
        L.orc_neighbors.restype = C.c_uint32
        L.orc_set_rigid_bodies.argtypes = [C.c_void_p, i32p, C.c_uint32, C.c_uint32]
        L.orc_set_rigid_bodies.restype = C.c_int
        L.orc_get_rigid.argtypes = [C.c_void_p, fp, fp, fp, fp]
        L.orc_get_rigid.restype = C.c_int
        L.orc_rigid_body_step.argtypes = [fp, fp, fp, C.c_float, C.c_float]
        L.orc_inverse3.argtypes = [fp, fp]
        L.orc_inverse3.restype = C.c_int
        dp = C.POINTER(C.c_double)
        L.orc_adjoint_run.argtypes = [P, dp, dp, C.c_uint32, C.c_int32, C.c_int32, dp, C.c_double, C.c_double,
                                      C.c_double, C.c_double, dp, dp, dp]
        L.orc_adjoint_run.restype = C.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REFLIB)


def ref():
    """The reference's own CPU code (zIndex, WeightingKernel, UnifiedConstants)."""
    global _ref
    if _ref is None:
        L = C.CDLL(REFLIB)
        fp, u32p = C.POINTER(C.c_float), C.POINTER(C.c_uint32)
        L.ref_morton_table.argtypes = [u32p]
        L.ref_box_query.argtypes = [C.c_uint32, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), u32p, u32p, C.c_int]
        L.ref_box_query.restype = C.c_int
        L.ref_block_size.argtypes = [C.c_int]
        L.ref_block_size.restype = C.c_uint32
        L.ref_luts.argtypes = [C.c_float, fp]
        L.ref_kernels.argtypes = [C.c_float, C.c_float, fp]
        L.ref_lut_lookup.argtypes = [C.c_float, fp, C.c_int, fp]
        L.ref_default_constants.argtypes = [fp]
        ip = C.POINTER(C.c_int)
        for name in ("ref_io_save_liquid", "ref_io_save_rigid"):
            getattr(L, name).argtypes = [C.c_char_p, fp, ip, C.c_int, C.c_int, C.c_char_p, C.c_int]
            getattr(L, name).restype = C.c_int
        L.ref_io_save_positions.argtypes = [C.c_char_p, fp, C.c_int, C.c_char_p, C.c_int]
        L.ref_io_save_positions.restype = C.c_int
        L.ref_io_read_num.argtypes = [C.c_char_p]
        L.ref_io_read_num.restype = C.c_int
        L.ref_io_read_pcisph.argtypes = [C.c_char_p, fp, fp, ip, fp, fp]
        L.ref_obj_particles.argtypes = [C.c_char_p, C.c_float, C.c_float, C.c_float, C.c_float, fp, C.c_int]
        L.ref_obj_particles.restype = C.c_int
        _ref = L
    return _ref


# ---------------------------------------------------------------- helpers
def default_params() -> UpfParams:
    p = UpfParams()
    lib().orc_default_params(C.byref(p))
    return p


def derive(p: UpfParams) -> UpfParams:
    q = p.copy()
    rc = lib().orc_params_derive(C.byref(q))
    if rc != 0:
        raise ValueError("orc_params_derive failed")
    return q


def luts(p: UpfParams) -> np.ndarray:
    out = np.zeros((5, 301), np.float32)
    lib().orc_build_luts(C.byref(p), _ptr(out, C.c_float))
    return out


def rigid_body_step(state, force, torque, dt, terminal_speed) -> np.ndarray:
    """One FP32 body update of a 47-float body state (see orc_rigid_body_step)."""
    st = np.array(state, np.float32).copy()
    f = np.ascontiguousarray(force, np.float32)
    t = np.ascontiguousarray(torque, np.float32)
    lib().orc_rigid_body_step(_ptr(st, C.c_float), _ptr(f, C.c_float), _ptr(t, C.c_float), float(dt),
                              float(terminal_speed))
    return st


def inverse3(m9) -> np.ndarray:
    a = np.ascontiguousarray(m9, np.float32).reshape(9)
    out = np.zeros(9, np.float32)
    lib().orc_inverse3(_ptr(a, C.c_float), _ptr(out, C.c_float))
    return out


def adjoint_run(params, pos, vel, steps, iterations, target, com_weight, density_weight, viscosity, grad=True,
                eps_rho=1e-2):
    """FP64 differentiable PCISPH trajectory (the library's upf_adjoint model):
    (loss, dL/dv0 (n,3), dL/dviscosity) or just the loss when grad is False."""
    pos = np.ascontiguousarray(np.asarray(pos, np.float64)[:, :3])
    vel = np.ascontiguousarray(np.asarray(vel, np.float64)[:, :3])
    n = pos.shape[0]
    tgt = np.ascontiguousarray(target, np.float64)
    loss = C.c_double()
    gv = np.zeros((n, 3), np.float64) if grad else None
    gm = C.c_double()
    rc = lib().orc_adjoint_run(C.byref(params), _ptr(pos, C.c_double), _ptr(vel, C.c_double), n, int(steps),
                               int(iterations), _ptr(tgt, C.c_double), float(com_weight), float(density_weight),
                               float(viscosity), float(eps_rho), C.byref(loss), _ptr(gv, C.c_double) if grad else None,
                               C.byref(gm) if grad else None)
    if rc != 0:
        raise RuntimeError("orc_adjoint_run failed")
    return (loss.value, gv, gm.value) if grad else loss.value


def morton_table() -> np.ndarray:
    out = np.zeros((1024, 3), np.uint32)
    lib().orc_morton_table(_ptr(out, C.c_uint32))
    return out


def box_query(block_size, mn, mx, cap=4096):
    a = np.asarray(mn, np.uint16)
    b = np.asarray(mx, np.uint16)
    f = np.zeros(cap, np.uint32)
    l = np.zeros(cap, np.uint32)
    n = lib().orc_box_query(block_size, _ptr(a, C.c_uint16), _ptr(b, C.c_uint16), _ptr(f, C.c_uint32), _ptr(l, C.c_uint32), cap)
    return f[:n].copy(), l[:n].copy()


class OracleSim:
    """One oracle simulation (all particle types in one array, as in the
    reference's UnifiedPhysics)."""

    def __init__(self, params: UpfParams, pos4, vel4, types, fp64=False, threads=0, keep_fields=True):
        self.params = params
        pos4 = np.ascontiguousarray(pos4, np.float32)
        vel4 = np.ascontiguousarray(vel4, np.float32)
        types = np.ascontiguousarray(types, np.int32)
        self.n = pos4.shape[0]
        self._h = lib().orc_create(C.byref(params), _ptr(pos4, C.c_float), _ptr(vel4, C.c_float),
                                   _ptr(types, C.c_int32), self.n, int(fp64), int(threads))
        lib().orc_keep_fields(self._h, int(keep_fields))

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_reference_literal(self, mask: int):
        """Switch deviations back to the reference's literal rule (the
        LITERAL_* bits; before set_rigid_bodies for the inertia and assembly bits)."""
        lib().orc_set_reference_literal(self._h, int(mask))

    def set_lagged(self, pressure_prev, pressure, density):
        """Continue from another run's state, per particle in creation order:
        the final correction pressure of the step before last and of the last
        step, and the last step's predicted density."""
        arrs = [np.ascontiguousarray(a, np.float32) for a in (pressure_prev, pressure, density)]
        assert all(a.shape == (self.n,) for a in arrs)
        lib().orc_set_lagged(self._h, *[_ptr(a, C.c_float) for a in arrs])

    def lagged(self):
        """(pressure_prev, pressure, density) of the current state, per
        particle in creation order (what set_lagged takes)."""
        arrs = [np.zeros(self.n, np.float32) for _ in range(3)]
        lib().orc_get_lagged(self._h, *[_ptr(a, C.c_float) for a in arrs])
        return tuple(arrs)

    def step(self) -> StepInfo:
        info = StepInfo()
        rc = lib().orc_step(self._h, C.byref(info))
        if rc != 0:
            raise RuntimeError("oracle step failed")
        return info

    def set_rigid_bodies(self, body, num_bodies):
        body = np.ascontiguousarray(body, np.int32)
        rc = lib().orc_set_rigid_bodies(self._h, _ptr(body, C.c_int32), body.shape[0], num_bodies)
        if rc != 0:
            raise RuntimeError("oracle rigid bodies not supported for this scene")
        self.num_bodies = int(num_bodies)

    def rigid(self):
        """(pos (nb,3), vel (nb,3), omega (nb,3), quat (nb,4) as (s,x,y,z))."""
        nb = getattr(self, "num_bodies", 0)
        pos = np.zeros((nb, 3), np.float32)
        vel = np.zeros((nb, 3), np.float32)
        om = np.zeros((nb, 3), np.float32)
        q = np.zeros((nb, 4), np.float32)
        if nb:
            lib().orc_get_rigid(self._h, _ptr(pos, C.c_float), _ptr(vel, C.c_float), _ptr(om, C.c_float),
                                _ptr(q, C.c_float))
        return pos, vel, om, q

    def state(self):
        n = self.n
        pos = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        den = np.zeros(n, np.float32)
        pre = np.zeros(n, np.float32)
        typ = np.zeros(n, np.int32)
        ids = np.zeros(n, np.uint32)
        key = np.zeros(n, np.uint32)
        lib().orc_get(self._h, _ptr(pos, C.c_float), _ptr(vel, C.c_float), _ptr(den, C.c_float),
                      _ptr(pre, C.c_float), _ptr(typ, C.c_int32), _ptr(ids, C.c_uint32), _ptr(key, C.c_uint32))
        return dict(pos=pos, vel=vel, density=den, pressure=pre, type=typ, id=ids, key=key)

    def step_fields(self):
        n = self.n
        f = np.zeros((n, 4), np.float32)
        fp = np.zeros((n, 4), np.float32)
        rs = np.zeros(n, np.float32)
        pc = np.zeros(n, np.float32)
        den = np.zeros(n, np.float32)
        pr = np.zeros(n, np.float32)
        ids = np.zeros(n, np.uint32)
        lib().orc_get_step_fields(self._h, _ptr(f, C.c_float), _ptr(fp, C.c_float), _ptr(rs, C.c_float),
                                  _ptr(pc, C.c_float), _ptr(den, C.c_float), _ptr(pr, C.c_float),
                                  _ptr(ids, C.c_uint32))
        return dict(force=f, pforce=fp, predicted_density=rs, corr_pressure=pc, density=den,
                    pressure=pr, id=ids)

    def neighbors(self):
        """CSR neighbour lists of the current order, as particle ids."""
        n = self.n
        off = np.zeros(n + 1, np.uint32)
        total = lib().orc_neighbors(self._h, _ptr(off, C.c_uint32), None, 0)
        ids = np.zeros(max(total, 1), np.uint32)
        lib().orc_neighbors(self._h, _ptr(off, C.c_uint32), _ptr(ids, C.c_uint32), total)
        return off, ids[:total]


# ---------------------------------------------------------------- reference file I/O
def ref_io_write(kind: str, workdir: str, pos4, type_=None, count: int = 0) -> bytes:
    """The bytes the reference's UnifiedIO writer `kind` ("liquid", "rigid",
    "positions") produces for these arrays (written under workdir)."""
    R = ref()
    pos4 = np.ascontiguousarray(pos4, np.float32)
    name = C.create_string_buffer(512)
    d = os.fsencode(workdir)
    if kind == "positions":
        rc = R.ref_io_save_positions(d, _ptr(pos4, C.c_float), len(pos4), name, 512)
    else:
        t = np.ascontiguousarray(type_, np.int32)
        fn = R.ref_io_save_liquid if kind == "liquid" else R.ref_io_save_rigid
        rc = fn(d, _ptr(pos4, C.c_float), _ptr(t, C.c_int), len(t), int(count), name, 512)
    if rc != 0:
        raise RuntimeError("reference writer failed")
    with open(os.path.join(workdir, name.value.decode()), "rb") as f:
        return f.read()


def ref_io_read_pcisph(path: str) -> dict:
    """UnifiedIO::ReadInFluidParticleNum + ReadInFluidParticlesPCISPH on path
    (which must exist: the reference exits the process otherwise)."""
    R = ref()
    n = R.ref_io_read_num(os.fsencode(path))
    out = {"pos": np.zeros((n, 3), np.float32), "vel": np.zeros((n, 3), np.float32), "type": np.zeros(n, np.int32),
           "corr_pressure": np.zeros(n, np.float32), "predicted_density": np.zeros(n, np.float32)}
    R.ref_io_read_pcisph(os.fsencode(path), _ptr(out["pos"], C.c_float), _ptr(out["vel"], C.c_float),
                         _ptr(out["type"], C.c_int), _ptr(out["corr_pressure"], C.c_float),
                         _ptr(out["predicted_density"], C.c_float))
    return out


# ---------------------------------------------------------------- reference mesh voxeliser
def ref_obj_particles(path: str, scale, spacing: float) -> np.ndarray:
    """ObjLoader::GetInstance().LoadParticles on an OBJ file: particle
    positions (n x 3) in the reference's order."""
    R = ref()
    sx, sy, sz = (float(v) for v in scale)
    cap = 1 << 16
    while True:
        buf = np.zeros((cap, 3), np.float32)
        n = R.ref_obj_particles(os.fsencode(path), sx, sy, sz, float(spacing), _ptr(buf, C.c_float), cap)
        if n <= cap:
            return buf[:n].copy()
        cap = n


# ---------------------------------------------------------------- scene generators (restated)
def scene_fluid_block(box_min, box_max, spacing, jitter, offset) -> np.ndarray:
    """Scene::createFluidObject restated (oracle/scene_oracle.cpp): n x 4."""
    L = lib()
    f3 = lambda v: np.ascontiguousarray(v, np.float32)  # noqa: E731
    a, b, o = f3(box_min), f3(box_max), f3(offset)
    L.orc_scene_fluid_block.restype = C.c_int64
    L.orc_scene_fluid_block.argtypes = [C.POINTER(C.c_float)] * 2 + [C.c_float, C.c_float, C.POINTER(C.c_float),
                                                                     C.POINTER(C.c_float), C.c_int64]
    n = L.orc_scene_fluid_block(_ptr(a, C.c_float), _ptr(b, C.c_float), spacing, jitter, _ptr(o, C.c_float), None, 0)
    out = np.zeros((max(n, 0), 4), np.float32)
    L.orc_scene_fluid_block(_ptr(a, C.c_float), _ptr(b, C.c_float), spacing, jitter, _ptr(o, C.c_float),
                            _ptr(out, C.c_float), n)
    return out


def scene_box_boundary(cmin, cmax, zstart, spacing, support_radius, dist_frozen, layers):
    """Scene::createBoxBoundaryFrozenParticles(MultiLayers) restated: (pos n x 4,
    normals n x 4), or None where the reference aborts."""
    L = lib()
    f3 = lambda v: np.ascontiguousarray(v, np.float32)  # noqa: E731
    a, b, z = f3(cmin), f3(cmax), f3(zstart)
    fp = C.POINTER(C.c_float)
    L.orc_scene_box_boundary.restype = C.c_int64
    L.orc_scene_box_boundary.argtypes = [fp, fp, fp, C.c_float, C.c_float, C.c_float, C.c_int, fp, fp, C.c_int64]
    n = L.orc_scene_box_boundary(_ptr(a, C.c_float), _ptr(b, C.c_float), _ptr(z, C.c_float), spacing,
                                 support_radius, dist_frozen, layers, None, None, 0)
    if n < 0:
        return None
    pos = np.zeros((n, 4), np.float32)
    nrm = np.zeros((n, 4), np.float32)
    L.orc_scene_box_boundary(_ptr(a, C.c_float), _ptr(b, C.c_float), _ptr(z, C.c_float), spacing, support_radius,
                             dist_frozen, layers, _ptr(pos, C.c_float), _ptr(nrm, C.c_float), n)
    return pos, nrm
