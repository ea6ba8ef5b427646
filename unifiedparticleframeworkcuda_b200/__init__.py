"""B200-native per-step particle pipeline (SPH / WCSPH / PCISPH).

Python host mirror of the C ABI in include/upf.h, over ctypes. The compute
path is the in-tree CUDA library libupf.so (sm_100a); there is no CPU
fallback: if the library is missing or no GPU is present, the calls fail.

The reference drives its GPU path from the C++ facade UnifiedPhysics
(src/cpu/UnifiedPhysics.cpp:615-643 InitCudaVariables, 4051-4141
CudaParticlePhysics, 404-407 CopyGPUParticles). `ParticleSystem` mirrors
that: construct with parameters, upload particles, step, copy back.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._abi import (FLAG_ADHESION, FLAG_BOUNDARY_PRESSURE, FLAG_PENALTY_WALLS,  # noqa: F401
                   FLAG_RECORD_ITERATIONS, FLAG_SURFACE_TENSION, FLAG_WALL_WEIGHT, FROZEN,
                   GRANULAR, LIQUID, METHOD_PCISPH, METHOD_WCSPH, RIGID, STATUS, UpfParams,
                   UpfAdjointOptions, UpfDeviceState, UpfLaunchConfig, UpfPhaseTimes, UpfStepStats)

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libupf.so")

_lib = None


class UpfError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__("%s: %s: %s" % (where, STATUS.get(status, status), message))


def lib():
    """Load libupf.so (build it first with `python -m unifiedparticleframeworkcuda_b200.build`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError("libupf.so not built: run python -m unifiedparticleframeworkcuda_b200.build")
        L = C.CDLL(LIBPATH)
        P = C.POINTER(UpfParams)
        vp, fp = C.c_void_p, C.POINTER(C.c_float)
        u32p, i32p = C.POINTER(C.c_uint32), C.POINTER(C.c_int32)
        sig = {
            "upf_default_params": [P],
            "upf_params_derive": [P],
            "upf_density_error_factor": [P, C.POINTER(C.c_double)],
            "upf_build_luts": [P, fp],
            "upf_build_bin_thresholds": [P, fp],
            "upf_create": [P, C.c_int, C.c_uint32, C.POINTER(vp)],
            "upf_destroy": [vp],
            "upf_get_params": [vp, P],
            "upf_set_stream": [vp, vp],
            "upf_set_particles": [vp, fp, fp, i32p, C.c_uint32],
            "upf_set_rigid_bodies": [vp, i32p, C.c_uint32, C.c_uint32],
            "upf_step": [vp, C.c_int32],
            "upf_synchronize": [vp],
            "upf_get_step_stats": [vp, C.POINTER(UpfStepStats)],
            "upf_phase_sort": [vp],
            "upf_phase_neighbors": [vp],
            "upf_phase_forces": [vp],
            "upf_phase_predict_correct": [vp],
            "upf_phase_integrate": [vp],
            "upf_phase_loop_begin": [vp],
            "upf_phase_density": [vp],
            "upf_phase_pressure_force": [vp],
            "upf_phase_loop_control": [vp, i32p],
            "upf_get_device_state": [vp, C.POINTER(UpfDeviceState)],
            "upf_set_dynamic_device": [vp, fp, fp, fp, i32p, u32p, C.c_uint32],
            "upf_gather_rows": [vp, C.c_uint32, vp, C.c_uint32, vp, vp],
            "upf_scatter_rows": [vp, C.c_uint32, vp, C.c_uint32, vp, vp],
            "upf_get_particles": [vp, fp, fp, fp, fp, i32p, u32p, u32p],
            "upf_get_particles_input_order": [vp, fp, fp, fp, fp, i32p, C.c_uint32],
            "upf_get_lagged_state": [vp, fp, C.c_uint32],
            "upf_get_step_fields": [vp, fp, fp, fp, u32p, u32p],
            "upf_get_neighbors": [vp, u32p, u32p, C.c_uint32, u32p],
            "upf_get_sorted_keys": [vp, u32p, u32p, u32p],
            "upf_get_cell_ranges": [vp, u32p, u32p, u32p],
            "upf_get_rigid_bodies": [vp, fp, fp, fp, fp, u32p],
            "upf_batch_create": [P, u32p, C.c_uint32, C.c_int, C.POINTER(vp)],
            "upf_batch_destroy": [vp],
            "upf_batch_set_stream": [vp, vp],
            "upf_batch_set_particles": [vp, fp, fp],
            "upf_batch_step": [vp, C.c_int32],
            "upf_batch_synchronize": [vp],
            "upf_batch_get_stats": [vp, C.POINTER(UpfStepStats)],
            "upf_batch_reset_counters": [vp],
            "upf_batch_get_particles": [vp, C.c_uint32, fp, fp, fp, fp, u32p, u32p],
            "upf_batch_checkpoint": [vp, C.c_int32],
            "upf_batch_restore": [vp, C.c_int32],
            "upf_batch_upload_state": [vp, fp, fp],
            "upf_batch_download_state": [vp, fp, fp],
            "upf_batch_profile_step": [vp, C.POINTER(UpfPhaseTimes), C.POINTER(C.c_uint64)],
            "upf_get_launch_config": [vp, C.POINTER(UpfLaunchConfig)],
            "upf_set_launch_config": [vp, C.POINTER(UpfLaunchConfig)],
            "upf_autotune": [vp, C.c_int32, C.POINTER(UpfLaunchConfig)],
            "upf_batch_get_launch_config": [vp, C.POINTER(UpfLaunchConfig)],
            "upf_batch_set_launch_config": [vp, C.POINTER(UpfLaunchConfig)],
            "upf_batch_autotune": [vp, C.c_int32, C.POINTER(UpfLaunchConfig)],
            "upf_adjoint_create": [P, C.POINTER(UpfAdjointOptions), fp, fp, C.c_uint32, C.c_int, C.POINTER(vp)],
            "upf_adjoint_destroy": [vp],
            "upf_adjoint_set_stream": [vp, vp],
            "upf_adjoint_forward": [vp, fp, C.c_float, C.POINTER(C.c_double)],
            "upf_adjoint_backward": [vp, fp, C.POINTER(C.c_double)],
            "upf_adjoint_get_state": [vp, fp, fp],
            "upf_adjoint_times": [vp, fp, fp],
            "upf_test_fail_allocation": [C.c_int32],
            "upf_test_stage_union_cap": [vp, C.c_uint32],
            "upf_selftest_bounded_wait": [C.c_int, C.c_uint32],
            "upf_selftest_support_bins": [C.c_int, P, fp, C.c_uint32, i32p],
            "upf_morton_keys": [vp, C.c_uint32, fp, fp, vp, vp],
            "upf_radix_sort_pairs": [vp, vp, C.c_uint32, C.c_int32, vp, C.c_size_t, vp],
            "upf_radix_sort_pairs_noalloc": [vp, vp, C.c_uint32, C.c_int32, vp],
            "upf_cell_ranges": [vp, C.c_uint32, C.c_int32, C.c_uint32, vp, vp, vp],
            "upf_upload_state": [vp, fp, fp, C.c_uint32],
            "upf_upload_state_async": [vp, fp, fp, C.c_uint32],
            "upf_get_particles_async": [vp, fp, fp, fp, fp, i32p, u32p, u32p],
            "upf_wait_frames": [vp],
            "upf_exchange_frame_async": [vp, fp, fp, fp, fp, i32p, u32p, C.c_uint32, u32p],
            "upf_batch_upload_state_async": [vp, fp, fp],
            "upf_batch_download_state_async": [vp, fp, fp],
            "upf_batch_wait_frames": [vp],
            "upf_profile_step": [vp, C.POINTER(UpfPhaseTimes)],
            "upf_reset_counters": [vp],
            "upf_checkpoint": [vp, C.c_int32],
            "upf_restore": [vp, C.c_int32],
            "upf_state_save": [vp, vp, C.c_size_t],
            "upf_state_load": [vp, vp, C.c_size_t],
            "upf_state_write_file": [vp, C.c_char_p],
            "upf_state_read_file": [vp, C.c_char_p],
            "upf_state_file_info": [C.c_char_p, P, u32p, u32p, C.POINTER(C.c_uint64)],
            "upf_io_save_liquid_info_full": [C.c_char_p, fp, i32p, C.c_int32, C.c_int32],
            "upf_io_save_rigid_info_full": [C.c_char_p, fp, i32p, C.c_int32, C.c_int32],
            "upf_io_save_particle_positions": [C.c_char_p, fp, C.c_uint32],
            "upf_io_save_scene_particles": [C.c_char_p, fp, fp, fp, i32p, C.c_uint32, C.c_float, C.c_float],
            "upf_io_save_fluid_particles_pcisph": [C.c_char_p, fp, fp, i32p, fp, fp, C.c_uint32],
            "upf_io_read_fluid_particle_num": [C.c_char_p, i32p],
            "upf_io_read_fluid_particles_pcisph": [C.c_char_p, fp, fp, i32p, fp, fp, C.c_int32, i32p],
            "upf_io_read_scene_particles": [C.c_char_p, fp, fp, fp, i32p, C.c_uint32, u32p],
            "upf_obj_read_triangles": [C.c_char_p, fp, C.c_uint32, u32p],
            "upf_scene_fluid_block": [C.c_int, fp, fp, C.c_float, C.c_float, fp, fp, C.c_uint32, u32p],
            "upf_scene_rigid_surface": [C.c_int, C.c_int32, C.c_float, C.c_uint32, fp, fp, fp, C.c_uint32, u32p],
            "upf_scene_box_boundary": [C.c_int, fp, fp, fp, C.c_float, C.c_float, C.c_float, C.c_int32, fp, fp,
                                       C.c_uint32, u32p],
            "upf_mesh_particles": [C.c_int, fp, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float, fp,
                                   C.c_uint32, u32p],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.upf_state_bytes.argtypes = [vp]
        L.upf_state_bytes.restype = C.c_size_t
        L.upf_radix_sort_temp_bytes.argtypes = [C.c_uint32]
        L.upf_radix_sort_temp_bytes.restype = C.c_size_t
        L.upf_last_error.restype = C.c_char_p
        L.upf_status_string.argtypes = [C.c_int]
        L.upf_status_string.restype = C.c_char_p
        L.upf_abi_version.restype = C.c_int32
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != 0:
        raise UpfError(status, where, lib().upf_last_error().decode())


def _p(a, ctype):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def default_params() -> UpfParams:
    p = UpfParams()
    check(lib().upf_default_params(C.byref(p)), "upf_default_params")
    return p


def derive_params(p: UpfParams) -> UpfParams:
    q = p.copy()
    check(lib().upf_params_derive(C.byref(q)), "upf_params_derive")
    return q


def density_error_factor(p: UpfParams) -> float:
    out = C.c_double()
    check(lib().upf_density_error_factor(C.byref(p), C.byref(out)), "upf_density_error_factor")
    return out.value


def build_luts(p: UpfParams) -> np.ndarray:
    out = np.zeros((5, 301), np.float32)
    check(lib().upf_build_luts(C.byref(p), _p(out, C.c_float)), "upf_build_luts")
    return out


def bin_thresholds(p: UpfParams) -> np.ndarray:
    out = np.zeros(302, np.float32)
    check(lib().upf_build_bin_thresholds(C.byref(p), _p(out, C.c_float)), "upf_build_bin_thresholds")
    return out


def obj_triangles(path) -> np.ndarray:
    """The triangles of a Wavefront OBJ file (upf_obj_read_triangles), n x 9."""
    n = C.c_uint32()
    fs = os.fsencode(str(path))
    check(lib().upf_obj_read_triangles(fs, None, 0, C.byref(n)), "upf_obj_read_triangles")
    out = np.zeros((n.value, 9), np.float32)
    check(lib().upf_obj_read_triangles(fs, _p(out, C.c_float), n.value, C.byref(n)), "upf_obj_read_triangles")
    return out


def _f3(v):
    return np.ascontiguousarray(v, np.float32).reshape(3)


def scene_fluid_block(box_min, box_max, spacing: float, jitter: float = 0.0, offset=(0.0, 0.0, 0.0),
                      device: int = 0) -> np.ndarray:
    """The reference's Scene::createFluidObject lattice on the GPU
    (upf_scene_fluid_block), n x 4."""
    a, b, o = _f3(box_min), _f3(box_max), _f3(offset)
    n = C.c_uint32()
    args = (device, _p(a, C.c_float), _p(b, C.c_float), float(spacing), float(jitter), _p(o, C.c_float))
    check(lib().upf_scene_fluid_block(*args, None, 0, C.byref(n)), "upf_scene_fluid_block")
    out = np.zeros((n.value, 4), np.float32)
    check(lib().upf_scene_fluid_block(*args, _p(out, C.c_float), n.value, C.byref(n)), "upf_scene_fluid_block")
    return out


def scene_rigid_surface(shape: int, radius: float, n_target: int, rotation=None, center=(0.0, 0.0, 0.0),
                        device: int = 0) -> np.ndarray:
    """A procedural rigid body's surface particles on the GPU
    (upf_scene_rigid_surface; shape 0 sphere, 1 cube, 2 torus), n x 4."""
    R = np.ascontiguousarray(np.eye(3) if rotation is None else rotation, np.float32).reshape(9)
    c = _f3(center)
    n = C.c_uint32()
    args = (device, int(shape), float(radius), int(n_target), _p(R, C.c_float), _p(c, C.c_float))
    check(lib().upf_scene_rigid_surface(*args, None, 0, C.byref(n)), "upf_scene_rigid_surface")
    out = np.zeros((n.value, 4), np.float32)
    check(lib().upf_scene_rigid_surface(*args, _p(out, C.c_float), n.value, C.byref(n)), "upf_scene_rigid_surface")
    return out


def scene_box_boundary(container_min, container_max, zindex_start, spacing: float, support_radius: float,
                       distance_frozen_to_boundary: float, layers: int = 2, device: int = 0):
    """The reference's Scene::createBoxBoundaryFrozenParticles(MultiLayers)
    walls on the GPU (upf_scene_box_boundary): (positions n x 4, normals n x 4)."""
    a, b, z = _f3(container_min), _f3(container_max), _f3(zindex_start)
    n = C.c_uint32()
    args = (device, _p(a, C.c_float), _p(b, C.c_float), _p(z, C.c_float), float(spacing), float(support_radius),
            float(distance_frozen_to_boundary), int(layers))
    check(lib().upf_scene_box_boundary(*args, None, None, 0, C.byref(n)), "upf_scene_box_boundary")
    pos = np.zeros((n.value, 4), np.float32)
    nrm = np.zeros((n.value, 4), np.float32)
    check(lib().upf_scene_box_boundary(*args, _p(pos, C.c_float), _p(nrm, C.c_float), n.value, C.byref(n)),
          "upf_scene_box_boundary")
    return pos, nrm


def mesh_particles(tri9, spacing: float, scale=(1.0, 1.0, 1.0), device: int = 0) -> np.ndarray:
    """Particles filling a closed triangle mesh on the GPU (upf_mesh_particles,
    the reference's ObjectLoader::LoadParticles), n x 4."""
    t = np.ascontiguousarray(tri9, np.float32).reshape(-1, 9)
    sx, sy, sz = (float(v) for v in scale)
    n = C.c_uint32()
    # at most one particle per lattice point: one pass when that bound is modest
    if len(t):
        v = t.reshape(-1, 3).astype(np.float64)
        ext = (np.maximum(v.max(0), 0.0) - np.minimum(v.min(0), 0.0)) * np.array([sx, sy, sz])
        bound = int(np.prod(np.floor(ext / float(spacing)) + 2))
    else:
        bound = 0
    if 0 < bound <= (1 << 24):
        out = np.zeros((bound, 4), np.float32)
        check(lib().upf_mesh_particles(device, _p(t, C.c_float), len(t), sx, sy, sz, float(spacing),
                                       _p(out, C.c_float), bound, C.byref(n)), "upf_mesh_particles")
        return out[: n.value].copy()
    check(lib().upf_mesh_particles(device, _p(t, C.c_float), len(t), sx, sy, sz, float(spacing), None, 0,
                                   C.byref(n)), "upf_mesh_particles")
    out = np.zeros((n.value, 4), np.float32)
    check(lib().upf_mesh_particles(device, _p(t, C.c_float), len(t), sx, sy, sz, float(spacing), _p(out, C.c_float),
                                   n.value, C.byref(n)), "upf_mesh_particles")
    return out


class ParticleSystem:
    """One simulation on one GPU (the reference's UnifiedPhysics + dataPointers)."""

    def __init__(self, params: UpfParams, capacity: int, device: int = 0, derive: bool = True):
        self.params = derive_params(params) if derive else params.copy()
        h = C.c_void_p()
        check(lib().upf_create(C.byref(self.params), int(device), int(capacity), C.byref(h)), "upf_create")
        self._h = h
        self.n_dynamic = 0

    # lifetime
    def close(self):
        if getattr(self, "_h", None):
            lib().upf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # uploads
    def set_particles(self, pos4, vel4, types):
        pos4 = np.ascontiguousarray(pos4, np.float32)
        vel4 = np.ascontiguousarray(vel4, np.float32)
        types = np.ascontiguousarray(types, np.int32)
        n = pos4.shape[0]
        if pos4.shape != (n, 4) or vel4.shape != (n, 4) or types.shape != (n,):
            raise ValueError("pos4/vel4 must be (n,4) and types (n,)")
        check(lib().upf_set_particles(self._h, _p(pos4, C.c_float), _p(vel4, C.c_float), _p(types, C.c_int32), n),
              "upf_set_particles")
        self.n_dynamic = int(np.count_nonzero(types != FROZEN))
        self.n_input = n
        self.n_bodies = 0

    def set_rigid_bodies(self, body_of_particle, n_bodies: int | None = None):
        """Group RIGID particles into bodies (body index per particle of the
        last set_particles call, -1 for none); PCISPH only, before the first
        step."""
        b = np.ascontiguousarray(body_of_particle, np.int32)
        if b.shape != (self.n_input,):
            raise ValueError("need one body index per uploaded particle")
        nb = int(b.max()) + 1 if n_bodies is None and b.size else int(n_bodies or 0)
        check(lib().upf_set_rigid_bodies(self._h, _p(b, C.c_int32), b.shape[0], nb), "upf_set_rigid_bodies")
        self.n_bodies = nb

    def rigid_bodies(self):
        """(pos (nb,3), vel (nb,3), omega (nb,3), quat (nb,4) as (s,x,y,z))."""
        nb = self.n_bodies
        pos = np.zeros((nb, 3), np.float32)
        vel = np.zeros((nb, 3), np.float32)
        om = np.zeros((nb, 3), np.float32)
        q = np.zeros((nb, 4), np.float32)
        cnt = C.c_uint32()
        check(lib().upf_get_rigid_bodies(self._h, _p(pos, C.c_float), _p(vel, C.c_float), _p(om, C.c_float),
                                         _p(q, C.c_float), C.byref(cnt)), "upf_get_rigid_bodies")
        return pos, vel, om, q

    # stepping
    def step(self, nsteps: int = 1):
        check(lib().upf_step(self._h, int(nsteps)), "upf_step")

    def synchronize(self):
        check(lib().upf_synchronize(self._h), "upf_synchronize")

    def stats(self) -> UpfStepStats:
        s = UpfStepStats()
        check(lib().upf_get_step_stats(self._h, C.byref(s)), "upf_get_step_stats")
        return s

    # checkpoint / resume
    def checkpoint(self, slot: int = 0):
        check(lib().upf_checkpoint(self._h, int(slot)), "upf_checkpoint")

    def restore(self, slot: int = 0):
        check(lib().upf_restore(self._h, int(slot)), "upf_restore")

    def save_state(self) -> bytes:
        n = lib().upf_state_bytes(self._h)
        buf = C.create_string_buffer(n)
        check(lib().upf_state_save(self._h, buf, n), "upf_state_save")
        return buf.raw

    def load_state(self, data: bytes):
        buf = C.create_string_buffer(data, len(data))
        check(lib().upf_state_load(self._h, buf, len(data)), "upf_state_load")

    def write_state_file(self, path: str):
        """Snapshot file (upf_state_write_file): resume with read_state_file."""
        check(lib().upf_state_write_file(self._h, os.fsencode(path)), "upf_state_write_file")

    def read_state_file(self, path: str):
        check(lib().upf_state_read_file(self._h, os.fsencode(path)), "upf_state_read_file")

    def reset_counters(self):
        check(lib().upf_reset_counters(self._h), "upf_reset_counters")

    def set_stream(self, stream_handle: int | None):
        """Run on a caller's cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
        check(lib().upf_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None), "upf_set_stream")

    def upload_state(self, pos4, vel4):
        """Host -> device copy of positions/velocities in the current device order."""
        pos4 = np.ascontiguousarray(pos4, np.float32)
        vel4 = np.ascontiguousarray(vel4, np.float32)
        check(lib().upf_upload_state(self._h, _p(pos4, C.c_float), _p(vel4, C.c_float), pos4.shape[0]),
              "upf_upload_state")

    def profile_step(self) -> UpfPhaseTimes:
        t = UpfPhaseTimes()
        check(lib().upf_profile_step(self._h, C.byref(t)), "upf_profile_step")
        return t

    def phase(self, name: str):
        check(getattr(lib(), "upf_phase_" + name)(self._h), "upf_phase_" + name)

    # readback
    def launch_config(self) -> UpfLaunchConfig:
        c = UpfLaunchConfig()
        check(lib().upf_get_launch_config(self._h, C.byref(c)), "upf_get_launch_config")
        return c

    def set_launch_config(self, cfg: UpfLaunchConfig):
        check(lib().upf_set_launch_config(self._h, C.byref(cfg)), "upf_set_launch_config")

    def autotune(self, repeats: int = 3) -> UpfLaunchConfig:
        """Times every launch shape of the tunable passes on the current state
        and keeps the fastest (the state is left unchanged)."""
        c = UpfLaunchConfig()
        check(lib().upf_autotune(self._h, int(repeats), C.byref(c)), "upf_autotune")
        return c

    def particles(self):
        n = self.n_dynamic
        pos = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        den = np.zeros(n, np.float32)
        pre = np.zeros(n, np.float32)
        typ = np.zeros(n, np.int32)
        ids = np.zeros(n, np.uint32)
        cnt = C.c_uint32()
        check(lib().upf_get_particles(self._h, _p(pos, C.c_float), _p(vel, C.c_float), _p(den, C.c_float),
                                      _p(pre, C.c_float), _p(typ, C.c_int32), _p(ids, C.c_uint32), C.byref(cnt)),
              "upf_get_particles")
        return dict(pos=pos, vel=vel, density=den, pressure=pre, type=typ, id=ids)

    def lagged_state(self):
        """The dynamic particles' lagged PCISPH state, in the order of
        particles(): (final correction pressure of the step before last, of
        the last step, last predicted density, 0) per particle."""
        out = np.zeros((self.n_dynamic, 4), np.float32)
        check(lib().upf_get_lagged_state(self._h, _p(out, C.c_float), self.n_dynamic), "upf_get_lagged_state")
        return out

    def particles_input_order(self):
        """Every particle of the last set_particles call at its input index
        (boundary particles included; pos.w = the Morton key), permuted back
        on the device."""
        n = self.n_input
        pos = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        den = np.zeros(n, np.float32)
        pre = np.zeros(n, np.float32)
        typ = np.zeros(n, np.int32)
        check(lib().upf_get_particles_input_order(self._h, _p(pos, C.c_float), _p(vel, C.c_float),
                                                  _p(den, C.c_float), _p(pre, C.c_float), _p(typ, C.c_int32), n),
              "upf_get_particles_input_order")
        return dict(pos=pos, vel=vel, density=den, pressure=pre, type=typ)

    def step_fields(self):
        n = self.n_dynamic
        f = np.zeros((n, 4), np.float32)
        fp = np.zeros((n, 4), np.float32)
        rs = np.zeros(n, np.float32)
        ids = np.zeros(n, np.uint32)
        cnt = C.c_uint32()
        check(lib().upf_get_step_fields(self._h, _p(f, C.c_float), _p(fp, C.c_float), _p(rs, C.c_float),
                                        _p(ids, C.c_uint32), C.byref(cnt)), "upf_get_step_fields")
        return dict(force=f, pforce=fp, predicted_density=rs, id=ids)

    def neighbors(self):
        n = self.n_dynamic
        cap = int(self.params.max_neighbors)
        counts = np.zeros(n, np.uint32)
        lists = np.zeros((n, cap), np.uint32)
        cnt = C.c_uint32()
        check(lib().upf_get_neighbors(self._h, _p(counts, C.c_uint32), _p(lists, C.c_uint32), cap, C.byref(cnt)),
              "upf_get_neighbors")
        return counts, lists

    def sorted_keys(self):
        n = self.n_dynamic
        keys = np.zeros(n, np.uint32)
        ids = np.zeros(n, np.uint32)
        cnt = C.c_uint32()
        check(lib().upf_get_sorted_keys(self._h, _p(keys, C.c_uint32), _p(ids, C.c_uint32), C.byref(cnt)),
              "upf_get_sorted_keys")
        return keys, ids

    def cell_ranges(self):
        cnt = C.c_uint32()
        check(lib().upf_get_cell_ranges(self._h, None, None, C.byref(cnt)), "upf_get_cell_ranges")
        nc = int(cnt.value)
        start = np.zeros(nc, np.uint32)
        end = np.zeros(nc, np.uint32)
        cnt = C.c_uint32()
        check(lib().upf_get_cell_ranges(self._h, _p(start, C.c_uint32), _p(end, C.c_uint32), C.byref(cnt)),
              "upf_get_cell_ranges")
        return start, end


class ParticleBatch:
    """Many independent PCISPH scenes advanced together (upf_batch_*): one
    launch per pass over all scenes, one CUDA graph per step."""

    def __init__(self, params_list, counts, device: int = 0, derive: bool = True):
        ps = [derive_params(p) if derive else p.copy() for p in params_list]
        self.params = ps
        arr = (UpfParams * len(ps))(*ps)
        self.counts = np.ascontiguousarray(counts, np.uint32)
        if self.counts.shape != (len(ps),):
            raise ValueError("one count per scene")
        h = C.c_void_p()
        check(lib().upf_batch_create(arr, _p(self.counts, C.c_uint32), len(ps), int(device), C.byref(h)),
              "upf_batch_create")
        self._h = h
        self.n_scenes = len(ps)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts.astype(np.int64))])

    @classmethod
    def from_scenes(cls, scene_list, device: int = 0):
        b = cls([sc.params for sc in scene_list], [sc.n for sc in scene_list], device=device)
        b.set_particles(np.concatenate([sc.pos for sc in scene_list]), np.concatenate([sc.vel for sc in scene_list]))
        return b

    def close(self):
        if getattr(self, "_h", None):
            lib().upf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_handle: int | None):
        check(lib().upf_batch_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None),
              "upf_batch_set_stream")

    def set_particles(self, pos4, vel4):
        pos4 = np.ascontiguousarray(pos4, np.float32)
        vel4 = np.ascontiguousarray(vel4, np.float32)
        n = int(self.offsets[-1])
        if pos4.shape != (n, 4) or vel4.shape != (n, 4):
            raise ValueError("pos4/vel4 must be (sum(counts), 4)")
        check(lib().upf_batch_set_particles(self._h, _p(pos4, C.c_float), _p(vel4, C.c_float)),
              "upf_batch_set_particles")

    def step(self, nsteps: int = 1):
        check(lib().upf_batch_step(self._h, int(nsteps)), "upf_batch_step")

    def synchronize(self):
        check(lib().upf_batch_synchronize(self._h), "upf_batch_synchronize")

    def stats(self):
        out = (UpfStepStats * self.n_scenes)()
        check(lib().upf_batch_get_stats(self._h, out), "upf_batch_get_stats")
        return list(out)

    def reset_counters(self):
        check(lib().upf_batch_reset_counters(self._h), "upf_batch_reset_counters")

    def checkpoint(self, slot: int = 0):
        check(lib().upf_batch_checkpoint(self._h, int(slot)), "upf_batch_checkpoint")

    def restore(self, slot: int = 0):
        check(lib().upf_batch_restore(self._h, int(slot)), "upf_batch_restore")

    def launch_config(self) -> UpfLaunchConfig:
        c = UpfLaunchConfig()
        check(lib().upf_batch_get_launch_config(self._h, C.byref(c)), "upf_batch_get_launch_config")
        return c

    def set_launch_config(self, cfg: UpfLaunchConfig):
        check(lib().upf_batch_set_launch_config(self._h, C.byref(cfg)), "upf_batch_set_launch_config")

    def autotune(self, repeats: int = 3) -> UpfLaunchConfig:
        c = UpfLaunchConfig()
        check(lib().upf_batch_autotune(self._h, int(repeats), C.byref(c)), "upf_batch_autotune")
        return c

    def profile_step(self):
        """(phase times of one step, particles processed by the loop passes)."""
        t = UpfPhaseTimes()
        act = C.c_uint64()
        check(lib().upf_batch_profile_step(self._h, C.byref(t), C.byref(act)), "upf_batch_profile_step")
        return t, int(act.value)

    def particles(self, scene: int):
        n = int(self.counts[scene])
        pos = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        den = np.zeros(n, np.float32)
        pre = np.zeros(n, np.float32)
        ids = np.zeros(n, np.uint32)
        cnt = C.c_uint32()
        check(lib().upf_batch_get_particles(self._h, int(scene), _p(pos, C.c_float), _p(vel, C.c_float),
                                            _p(den, C.c_float), _p(pre, C.c_float), _p(ids, C.c_uint32),
                                            C.byref(cnt)), "upf_batch_get_particles")
        return dict(pos=pos, vel=vel, density=den, pressure=pre, id=ids)


class Adjoint:
    """A differentiable PCISPH trajectory and its adjoint (upf_adjoint_*):
    forward() returns the loss, backward() its gradient with respect to the
    initial velocities and the viscosity."""

    def __init__(self, params, pos4, vel4, steps: int, checkpoint_interval: int = 20, loop_iterations: int = 3,
                 target=(0.0, 0.0, 0.0), com_weight: float = 1.0, density_weight: float = 1e-6,
                 density_smoothing: float = 1e-2, device: int = 0, derive: bool = True):
        self.params = derive_params(params) if derive else params.copy()
        pos4 = np.ascontiguousarray(pos4, np.float32)
        vel4 = np.ascontiguousarray(vel4, np.float32)
        self.n = pos4.shape[0]
        if pos4.shape != (self.n, 4) or vel4.shape != (self.n, 4):
            raise ValueError("pos4/vel4 must be (n, 4)")
        o = UpfAdjointOptions()
        o.steps, o.checkpoint_interval, o.loop_iterations = int(steps), int(checkpoint_interval), int(loop_iterations)
        o.target[:] = [float(t) for t in target]
        o.com_weight, o.density_weight = float(com_weight), float(density_weight)
        o.density_smoothing = float(density_smoothing)
        self.options = o
        h = C.c_void_p()
        check(lib().upf_adjoint_create(C.byref(self.params), C.byref(o), _p(pos4, C.c_float), _p(vel4, C.c_float),
                                       self.n, int(device), C.byref(h)), "upf_adjoint_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().upf_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle: int | None):
        check(lib().upf_adjoint_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None),
              "upf_adjoint_set_stream")

    def forward(self, vel4=None, viscosity: float | None = None) -> float:
        v = None if vel4 is None else np.ascontiguousarray(vel4, np.float32)
        if v is not None and v.shape != (self.n, 4):
            raise ValueError("vel4 must be (n, 4)")
        mu = self.params.viscosity if viscosity is None else float(viscosity)
        loss = C.c_double()
        check(lib().upf_adjoint_forward(self._h, _p(v, C.c_float), mu, C.byref(loss)), "upf_adjoint_forward")
        return loss.value

    def backward(self):
        """(dL/dv0 as (n, 3), dL/dviscosity)."""
        g = np.zeros((self.n, 4), np.float32)
        gm = C.c_double()
        check(lib().upf_adjoint_backward(self._h, _p(g, C.c_float), C.byref(gm)), "upf_adjoint_backward")
        return g[:, :3].copy(), gm.value

    def state(self):
        pos = np.zeros((self.n, 4), np.float32)
        vel = np.zeros((self.n, 4), np.float32)
        check(lib().upf_adjoint_get_state(self._h, _p(pos, C.c_float), _p(vel, C.c_float)), "upf_adjoint_get_state")
        return pos, vel

    def times(self):
        f = C.c_float()
        b = C.c_float()
        check(lib().upf_adjoint_times(self._h, C.byref(f), C.byref(b)), "upf_adjoint_times")
        return f.value, b.value

