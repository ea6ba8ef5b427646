"""Particle files in the reference's text formats (src/cpu/UnifiedIO.cpp,
src/sceneConfigure/Scene.cpp) and the library's snapshot files, over the
C ABI (upf_io_*, upf_state_file_info). Arrays are numpy; positions and
velocities are n x 4 float32 (x, y, z, unused) on the way in."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import LIQUID, UpfParams, _p, check, lib


def _f4(a) -> np.ndarray:
    a = np.ascontiguousarray(a, np.float32)
    if a.ndim != 2 or a.shape[1] not in (3, 4):
        raise ValueError("positions / velocities must be n x 3 or n x 4")
    if a.shape[1] == 3:
        a = np.concatenate([a, np.zeros((a.shape[0], 1), np.float32)], axis=1)
    return a


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, np.int32)


def save_liquid_info_full(path, pos, type_, num_liquid: int | None = None) -> None:
    """UnifiedIO::SaveLiquidParticleInfoFull (UnifiedIO.cpp:60-105)."""
    pos, type_ = _f4(pos), _i32(type_)
    nl = int(np.count_nonzero(type_ == LIQUID)) if num_liquid is None else int(num_liquid)
    check(lib().upf_io_save_liquid_info_full(os.fsencode(path), _p(pos, C.c_float), _p(type_, C.c_int32),
                                             len(type_), nl), "upf_io_save_liquid_info_full")


def save_rigid_info_full(path, pos, type_, header_count: int) -> None:
    """UnifiedIO::SaveRigidParticleInfoFull (UnifiedIO.cpp:107-152)."""
    pos, type_ = _f4(pos), _i32(type_)
    check(lib().upf_io_save_rigid_info_full(os.fsencode(path), _p(pos, C.c_float), _p(type_, C.c_int32),
                                            len(type_), int(header_count)), "upf_io_save_rigid_info_full")


def save_particle_positions(path, pos) -> None:
    """UnifiedIO::SaveParticlePositions (UnifiedIO.cpp:14-58)."""
    pos = _f4(pos)
    check(lib().upf_io_save_particle_positions(os.fsencode(path), _p(pos, C.c_float), len(pos)),
          "upf_io_save_particle_positions")


def save_scene_particles(path, pos, type_, rest_density=1000.0, mass=1.0) -> None:
    """Scene::saveParticles (Scene.cpp:247-279); rest_density / mass: one
    value for all particles or one per particle."""
    pos, type_ = _f4(pos), _i32(type_)
    rd = np.ascontiguousarray(rest_density, np.float32) if np.ndim(rest_density) else None
    ms = np.ascontiguousarray(mass, np.float32) if np.ndim(mass) else None
    check(lib().upf_io_save_scene_particles(os.fsencode(path), _p(pos, C.c_float), _p(rd, C.c_float),
                                            _p(ms, C.c_float), _p(type_, C.c_int32), len(pos),
                                            float(rest_density) if rd is None else 0.0,
                                            float(mass) if ms is None else 0.0), "upf_io_save_scene_particles")


def save_fluid_particles_pcisph(path, pos, vel, type_, corr_pressure=None, predicted_density=None) -> None:
    """The file UnifiedIO::ReadInFluidParticlesPCISPH reads."""
    pos, vel, type_ = _f4(pos), _f4(vel), _i32(type_)
    pc = None if corr_pressure is None else np.ascontiguousarray(corr_pressure, np.float32)
    pd = None if predicted_density is None else np.ascontiguousarray(predicted_density, np.float32)
    check(lib().upf_io_save_fluid_particles_pcisph(os.fsencode(path), _p(pos, C.c_float), _p(vel, C.c_float),
                                                   _p(type_, C.c_int32), _p(pc, C.c_float), _p(pd, C.c_float),
                                                   len(pos)), "upf_io_save_fluid_particles_pcisph")


def read_fluid_particle_num(path) -> int:
    """UnifiedIO::ReadInFluidParticleNum (UnifiedIO.cpp:154-177)."""
    n = C.c_int32()
    check(lib().upf_io_read_fluid_particle_num(os.fsencode(path), C.byref(n)), "upf_io_read_fluid_particle_num")
    return n.value


def read_fluid_particles_pcisph(path) -> dict:
    """UnifiedIO::ReadInFluidParticlesPCISPH (UnifiedIO.cpp:179-220): pos and
    vel n x 3, type, corr_pressure, predicted_density."""
    n = max(read_fluid_particle_num(path), 0)
    out = {"pos": np.zeros((n, 3), np.float32), "vel": np.zeros((n, 3), np.float32),
           "type": np.zeros(n, np.int32), "corr_pressure": np.zeros(n, np.float32),
           "predicted_density": np.zeros(n, np.float32)}
    got = C.c_int32()
    check(lib().upf_io_read_fluid_particles_pcisph(os.fsencode(path), _p(out["pos"], C.c_float),
                                                   _p(out["vel"], C.c_float), _p(out["type"], C.c_int32),
                                                   _p(out["corr_pressure"], C.c_float),
                                                   _p(out["predicted_density"], C.c_float), n, C.byref(got)),
          "upf_io_read_fluid_particles_pcisph")
    return out


def read_scene_particles(path) -> dict:
    """Scene::readInParticles (Scene.cpp:218-243): pos n x 4, density, mass,
    type, granular records skipped."""
    n = C.c_uint32()
    fs = os.fsencode(path)
    check(lib().upf_io_read_scene_particles(fs, None, None, None, None, 0, C.byref(n)), "upf_io_read_scene_particles")
    k = n.value
    out = {"pos": np.zeros((k, 4), np.float32), "density": np.zeros(k, np.float32),
           "mass": np.zeros(k, np.float32), "type": np.zeros(k, np.int32)}
    check(lib().upf_io_read_scene_particles(fs, _p(out["pos"], C.c_float), _p(out["density"], C.c_float),
                                            _p(out["mass"], C.c_float), _p(out["type"], C.c_int32), k, C.byref(n)),
          "upf_io_read_scene_particles")
    return out


def state_file_info(path) -> dict:
    """Header of a snapshot file (upf_state_file_info): the saving system's
    parameters, dynamic-particle and rigid-body counts, state bytes."""
    prm = UpfParams()
    nd, nb = C.c_uint32(), C.c_uint32()
    sb = C.c_uint64()
    check(lib().upf_state_file_info(os.fsencode(path), C.byref(prm), C.byref(nd), C.byref(nb), C.byref(sb)),
          "upf_state_file_info")
    return {"params": prm, "n_dynamic": nd.value, "num_bodies": nb.value, "state_bytes": sb.value}
