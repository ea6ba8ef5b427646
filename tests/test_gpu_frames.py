"""Asynchronous per-frame exchange (upf_upload_state_async,
upf_get_particles_async, upf_wait_frames): a pipelined loop, uploads and
readbacks in flight while the steps run, gives every frame bit for bit what
the synchronous calls (upf_upload_state, upf_get_particles) give."""
import ctypes as C

import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import scenes

pytestmark = pytest.mark.gpu
FIELDS = ("pos", "vel", "density", "pressure", "type", "id")


def _ptr(t, ctype):
    return C.cast(t.data_ptr(), C.POINTER(ctype))


def _host(torch, n):
    return {"pos": torch.zeros((n, 4), dtype=torch.float32, pin_memory=True),
            "vel": torch.zeros((n, 4), dtype=torch.float32, pin_memory=True),
            "density": torch.zeros(n, dtype=torch.float32, pin_memory=True),
            "pressure": torch.zeros(n, dtype=torch.float32, pin_memory=True),
            "type": torch.zeros(n, dtype=torch.int32, pin_memory=True),
            "id": torch.zeros(n, dtype=torch.int32, pin_memory=True)}


@pytest.mark.parametrize("scene", ["small_pcisph", "small_coupling"])
def test_pipelined_frames_equal_synchronous_frames(upf_lib, scene):
    torch = pytest.importorskip("torch")
    L = upf_lib.lib()
    sc = getattr(scenes, scene)()
    p = upf_lib.derive_params(sc.params)
    frames = 4

    def system():
        s = upf_lib.ParticleSystem(p, capacity=sc.n, derive=False)
        s.set_particles(sc.pos, sc.vel, sc.type)
        if getattr(sc, "num_bodies", 0):
            s.set_rigid_bodies(sc.body, sc.num_bodies)
        s.step(1)
        return s

    # synchronous reference run; each frame's input is the last result with
    # the velocities damped by 1%, so every upload changes the state
    inputs, want = [], []
    with system() as a:
        st = a.particles()
        for k in range(frames):
            pos = st["pos"].copy()
            vel = (st["vel"] * np.float32(0.99)).astype(np.float32)
            inputs.append((pos, vel))
            upf_lib.check(L.upf_upload_state(a.handle, pos.ctypes.data_as(C.POINTER(C.c_float)),
                                             vel.ctypes.data_as(C.POINTER(C.c_float)), len(pos)), "upload")
            a.step(1)
            st = a.particles()
            want.append(st)
    # pipelined run: every upload, step and readback issued before any wait
    with system() as b:
        n = b.n_dynamic
        ins = []
        for pos, vel in inputs:
            hp = torch.from_numpy(pos).pin_memory()
            hv = torch.from_numpy(vel).pin_memory()
            ins.append((hp, hv))
        outs = [_host(torch, n) for _ in range(frames)]
        cnt = C.c_uint32()
        for k in range(frames):
            hp, hv = ins[k]
            upf_lib.check(L.upf_upload_state_async(b.handle, _ptr(hp, C.c_float), _ptr(hv, C.c_float), n),
                          "upf_upload_state_async")
            b.step(1)
            o = outs[k]
            upf_lib.check(L.upf_get_particles_async(b.handle, _ptr(o["pos"], C.c_float), _ptr(o["vel"], C.c_float),
                                                    _ptr(o["density"], C.c_float), _ptr(o["pressure"], C.c_float),
                                                    _ptr(o["type"], C.c_int32), _ptr(o["id"], C.c_uint32),
                                                    C.byref(cnt)), "upf_get_particles_async")
        upf_lib.check(L.upf_wait_frames(b.handle), "upf_wait_frames")
        b.synchronize()
        for k in range(frames):
            for f in FIELDS:
                got = outs[k][f].numpy()
                ref = want[k][f]
                assert np.array_equal(got.view(np.uint32) if got.dtype != np.int32 else got,
                                      np.asarray(ref).view(np.uint32) if np.asarray(ref).dtype != np.int32
                                      else ref), (k, f)


def test_partial_readback_and_idle_wait(upf_lib):
    torch = pytest.importorskip("torch")
    L = upf_lib.lib()
    sc = scenes.small_pcisph()
    with upf_lib.ParticleSystem(upf_lib.derive_params(sc.params), capacity=sc.n, derive=False) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        assert L.upf_wait_frames(s.handle) == 0  # nothing issued yet
        s.step(2)
        n = s.n_dynamic
        pos = torch.zeros((n, 4), dtype=torch.float32, pin_memory=True)
        cnt = C.c_uint32()
        assert L.upf_get_particles_async(s.handle, _ptr(pos, C.c_float), None, None, None, None, None,
                                         C.byref(cnt)) == 0
        assert L.upf_wait_frames(s.handle) == 0
        assert cnt.value == n
        assert np.array_equal(pos.numpy(), s.particles()["pos"])


def test_batch_pipelined_frames_equal_synchronous_frames(upf_lib):
    """upf_batch_upload_state_async / upf_batch_download_state_async against
    upf_batch_upload_state / upf_batch_download_state, four frames."""
    torch = pytest.importorskip("torch")
    L = upf_lib.lib()
    fp = C.POINTER(C.c_float)
    scs = scenes.batch_scenes(num=6, seed=21, counts=(2048, 6000))
    frames = 4
    inputs, want = [], []
    with upf_lib.ParticleBatch.from_scenes(scs) as a:
        a.step(1)
        n = int(a.offsets[-1])
        pos = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        upf_lib.check(L.upf_batch_download_state(a.handle, pos.ctypes.data_as(fp), vel.ctypes.data_as(fp)), "dl")
        for k in range(frames):
            vel = (vel * np.float32(0.99)).astype(np.float32)
            inputs.append((pos.copy(), vel.copy()))
            upf_lib.check(L.upf_batch_upload_state(a.handle, pos.ctypes.data_as(fp), vel.ctypes.data_as(fp)), "ul")
            a.step(1)
            upf_lib.check(L.upf_batch_download_state(a.handle, pos.ctypes.data_as(fp), vel.ctypes.data_as(fp)), "dl")
            want.append((pos.copy(), vel.copy()))
    with upf_lib.ParticleBatch.from_scenes(scs) as b:
        b.step(1)
        ins = [(torch.from_numpy(p).pin_memory(), torch.from_numpy(v).pin_memory()) for p, v in inputs]
        outs = [(torch.zeros((n, 4), dtype=torch.float32, pin_memory=True),
                 torch.zeros((n, 4), dtype=torch.float32, pin_memory=True)) for _ in range(frames)]
        for k in range(frames):
            upf_lib.check(L.upf_batch_upload_state_async(b.handle, _ptr(ins[k][0], C.c_float),
                                                         _ptr(ins[k][1], C.c_float)), "ul async")
            b.step(1)
            upf_lib.check(L.upf_batch_download_state_async(b.handle, _ptr(outs[k][0], C.c_float),
                                                           _ptr(outs[k][1], C.c_float)), "dl async")
        upf_lib.check(L.upf_batch_wait_frames(b.handle), "upf_batch_wait_frames")
        b.synchronize()
    for k in range(frames):
        assert np.array_equal(outs[k][0].numpy().view(np.uint32), want[k][0].view(np.uint32)), k
        assert np.array_equal(outs[k][1].numpy().view(np.uint32), want[k][1].view(np.uint32)), k


@pytest.mark.parametrize("chunks", [1, 3, 16])
def test_exchange_round_trip_equals_readback_then_upload(upf_lib, chunks):
    """upf_exchange_frame_async (the readback and the upload of the same host
    arrays, chunk by chunk, the two copy directions overlapping) against the
    synchronous round trip: readback, wait, upload of what arrived. Every
    frame's host arrays and the states after each step are bit-identical,
    and the pieces cover the particles whatever the chunk count."""
    torch = pytest.importorskip("torch")
    L = upf_lib.lib()
    sc = scenes.small_coupling()
    p = upf_lib.derive_params(sc.params)
    frames = 3

    def system():
        s = upf_lib.ParticleSystem(p, capacity=sc.n, derive=False)
        s.set_particles(sc.pos, sc.vel, sc.type)
        s.set_rigid_bodies(sc.body, sc.num_bodies)
        s.step(1)
        return s

    want = []
    with system() as a:
        for _ in range(frames):
            st = a.particles()
            want.append(st)
            upf_lib.check(L.upf_upload_state(a.handle, st["pos"].ctypes.data_as(C.POINTER(C.c_float)),
                                             st["vel"].ctypes.data_as(C.POINTER(C.c_float)), len(st["pos"])),
                          "upload")
            a.step(1)
        final_want = a.particles()
    with system() as b:
        n = b.n_dynamic
        h = _host(torch, n)
        cnt = C.c_uint32()
        for k in range(frames):
            upf_lib.check(L.upf_exchange_frame_async(
                b.handle, _ptr(h["pos"], C.c_float), _ptr(h["vel"], C.c_float), _ptr(h["density"], C.c_float),
                _ptr(h["pressure"], C.c_float), _ptr(h["type"], C.c_int32), _ptr(h["id"], C.c_uint32), chunks,
                C.byref(cnt)), "upf_exchange_frame_async")
            upf_lib.check(L.upf_wait_frames(b.handle), "upf_wait_frames")
            assert cnt.value == n
            for f in FIELDS:
                got = h[f].numpy()
                assert np.array_equal(got.view(np.uint8), np.ascontiguousarray(want[k][f]).view(np.uint8)), (k, f)
            b.step(1)
        final_got = b.particles()
    for f in FIELDS:
        assert np.array_equal(final_got[f], final_want[f]), f
