"""TEST INFRASTRUCTURE: the reference's own CPU step, compiled by
oracle/Makefile from src/cpu/UnifiedPhysics.cpp into
oracle/_ref/libupfref_physics.so (see ref_pins_physics.cpp), run on a scene.

The reference keeps function-local statics (collision box, time step,
particle count, the lookup tables' distance factor) from the first scene a
process runs, so every call runs in a fresh Python process.

    reference_time(params, pos4, vel4, type, lagged, method, threads, warmup, steps, max_seconds)
        -> dict(seconds, iterations, error_percent) per timed step

    reference_steps(params, pos4, vel4, type, steps, weighted_volumes, method, body, num_bodies, lagged)
        -> dict(pos, vel, density, pressure, type, id, body), particles in
           the reference's final order (ascending Morton key); id = input
           index; body = per rigid body position, velocity, angular
           velocity, mass, quaternion (16 floats)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libupfref_physics.so")


def available() -> bool:
    return os.path.exists(LIB)


def reference_steps(params, pos4, vel4, type_, steps, weighted_volumes=False, method="pcisph", body=None,
                    num_bodies=0, lagged=None):
    if body is None:
        body = np.full(len(type_), -1, np.int32)
    lag = np.zeros((3, len(type_)), np.float32) if lagged is None else np.asarray(lagged, np.float32)
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.npz"), os.path.join(d, "out.npz")
        np.savez(src, params=np.frombuffer(bytes(params), np.uint8), pos=np.ascontiguousarray(pos4, np.float32),
                 vel=np.ascontiguousarray(vel4, np.float32), type=np.ascontiguousarray(type_, np.int32),
                 steps=np.int32(steps), wv=np.int32(1 if weighted_volumes else 0),
                 wcsph=np.int32(1 if method == "wcsph" else 0), body=np.ascontiguousarray(body, np.int32),
                 num_bodies=np.int32(num_bodies), lag=np.ascontiguousarray(lag),
                 have_lag=np.int32(lagged is not None))
        r = subprocess.run([sys.executable, os.path.abspath(__file__), src, dst], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference step failed: " + r.stderr[-2000:])
        out = np.load(dst)
        return {k: out[k] for k in out.files}


def reference_time(params, pos4, vel4, type_, lagged=None, method="pcisph", threads=1, warmup=1, steps=5,
                   max_seconds=60.0, min_steps=1):
    """The reference's step timed on the host cores (ref_physics_time): per
    timed step its wall seconds, and for PCISPH its iteration count and final
    density error in percent. lagged = (previous correction pressure, last
    correction pressure, last predicted density) per input particle, or None
    for a run from rest. Timed steps run until `steps`, or until at least
    `min_steps` and `max_seconds`."""
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.npz"), os.path.join(d, "out.npz")
        lag = np.zeros((3, len(type_)), np.float32) if lagged is None else np.asarray(lagged, np.float32)
        np.savez(src, params=np.frombuffer(bytes(params), np.uint8), pos=np.ascontiguousarray(pos4, np.float32),
                 vel=np.ascontiguousarray(vel4, np.float32), type=np.ascontiguousarray(type_, np.int32),
                 lag=np.ascontiguousarray(lag), have_lag=np.int32(lagged is not None),
                 wcsph=np.int32(1 if method == "wcsph" else 0), threads=np.int32(threads),
                 warmup=np.int32(warmup), steps=np.int32(steps), max_seconds=np.float64(max_seconds),
                 min_steps=np.int32(min_steps))
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "time", src, dst], capture_output=True,
                           text=True)
        if r.returncode != 0:
            raise RuntimeError("reference timing failed: " + r.stderr[-2000:])
        out = np.load(dst)
        return {k: out[k] for k in out.files}


def _time(src, dst):
    import ctypes as C
    sys.path.insert(0, os.path.dirname(HERE))
    from unifiedparticleframeworkcuda_b200._abi import UpfParams
    a = np.load(src)
    p = UpfParams.from_buffer_copy(a["params"].tobytes())
    n = a["pos"].shape[0]
    steps = int(a["steps"])
    L = C.CDLL(LIB)
    L.ref_physics_time.restype = C.c_int
    sec = np.zeros(steps, np.float64)
    its = np.zeros(steps, np.int32)
    err = np.zeros(steps, np.float32)
    vp = C.c_void_p
    lag = [a["lag"][k].ctypes.data_as(vp) if int(a["have_lag"]) else None for k in range(3)]
    done = L.ref_physics_time(C.c_int32(int(a["wcsph"])), C.byref(p), a["pos"].ctypes.data_as(vp),
                              a["vel"].ctypes.data_as(vp), a["type"].ctypes.data_as(vp), C.c_uint32(n), *lag,
                              C.c_int32(int(a["threads"])), C.c_int32(int(a["warmup"])), C.c_int32(steps),
                              C.c_int32(int(a["min_steps"])), C.c_double(float(a["max_seconds"])), sec.ctypes.data_as(vp), its.ctypes.data_as(vp),
                              err.ctypes.data_as(vp))
    if done < 1:
        raise SystemExit("ref_physics_time returned %d" % done)
    np.savez(dst, seconds=sec[:done], iterations=its[:done], error_percent=err[:done])


def _main(src, dst):
    import ctypes as C
    sys.path.insert(0, os.path.dirname(HERE))
    from unifiedparticleframeworkcuda_b200._abi import UpfParams
    a = np.load(src)
    p = UpfParams.from_buffer_copy(a["params"].tobytes())
    n = a["pos"].shape[0]
    L = C.CDLL(LIB)
    out = {"pos": np.zeros((n, 4), np.float32), "vel": np.zeros((n, 4), np.float32),
           "density": np.zeros(n, np.float32), "pressure": np.zeros(n, np.float32),
           "type": np.zeros(n, np.int32), "id": np.zeros(n, np.uint32),
           "body": np.zeros((int(a["num_bodies"]), 16), np.float32)}
    vp = C.c_void_p
    head = [C.byref(p), a["pos"].ctypes.data_as(vp), a["vel"].ctypes.data_as(vp), a["type"].ctypes.data_as(vp)]
    tail = [C.c_uint32(n), C.c_int32(int(a["steps"]))]
    outs = [out[k].ctypes.data_as(vp) for k in ("pos", "vel", "density", "pressure", "type", "id")]
    if int(a["wcsph"]):
        rc = L.ref_physics_wcsph_steps(*head, *tail, *outs)
    else:
        lag = [a["lag"][k].ctypes.data_as(vp) if int(a["have_lag"]) else None for k in range(3)]
        rc = L.ref_physics_pcisph_steps(*head, *lag, a["body"].ctypes.data_as(vp), C.c_uint32(int(a["num_bodies"])),
                                        *tail, C.c_int32(int(a["wv"])), *outs, out["body"].ctypes.data_as(vp))
    if rc != 0:
        raise SystemExit("reference step returned %d (1: equal Morton keys, 3: arguments)" % rc)
    np.savez(dst, **out)


if __name__ == "__main__":
    if sys.argv[1] == "time":
        _time(sys.argv[2], sys.argv[3])
    else:
        _main(sys.argv[1], sys.argv[2])
