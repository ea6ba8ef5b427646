"""TEST INFRASTRUCTURE: the reference's own CPU step, compiled by
oracle/Makefile from src/cpu/UnifiedPhysics.cpp into
oracle/_ref/libupfref_physics.so (see ref_pins_physics.cpp), run on a scene.

The reference keeps function-local statics (collision box, time step,
particle count, the lookup tables' distance factor) from the first scene a
process runs, so every call runs in a fresh Python process.

    reference_steps(params, pos4, vel4, type, steps, weighted_volumes, method, body, num_bodies)
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
                    num_bodies=0):
    if body is None:
        body = np.full(len(type_), -1, np.int32)
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.npz"), os.path.join(d, "out.npz")
        np.savez(src, params=np.frombuffer(bytes(params), np.uint8), pos=np.ascontiguousarray(pos4, np.float32),
                 vel=np.ascontiguousarray(vel4, np.float32), type=np.ascontiguousarray(type_, np.int32),
                 steps=np.int32(steps), wv=np.int32(1 if weighted_volumes else 0),
                 wcsph=np.int32(1 if method == "wcsph" else 0), body=np.ascontiguousarray(body, np.int32),
                 num_bodies=np.int32(num_bodies))
        r = subprocess.run([sys.executable, os.path.abspath(__file__), src, dst], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference step failed: " + r.stderr[-2000:])
        out = np.load(dst)
        return {k: out[k] for k in out.files}


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
        rc = L.ref_physics_pcisph_steps(*head, a["body"].ctypes.data_as(vp), C.c_uint32(int(a["num_bodies"])),
                                        *tail, C.c_int32(int(a["wv"])), *outs, out["body"].ctypes.data_as(vp))
    if rc != 0:
        raise SystemExit("reference step returned %d (1: equal Morton keys, 3: arguments)" % rc)
    np.savez(dst, **out)


if __name__ == "__main__":
    _main(sys.argv[1], sys.argv[2])
