"""The reference's own entry points (include/upf_compat.h, libupf_compat.so):
a host program shaped like the reference's facade (tests/compat/
facade_physics.cpp: InitDptr, InitCudaVariables, CudaParticlePhysics,
CopyGPUParticles, FreeDeviceArrays of src/cpu/UnifiedPhysics.cpp) compiles
against the header, links, and runs. Without a GPU the calls report the
missing device; on a GPU its steps are compared with the oracle."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import FROZEN, LIQUID, STATUS, UpfParams, scenes

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "unifiedparticleframeworkcuda_b200")
COMPAT = os.path.join(os.path.dirname(__file__), "compat")
CODE = {name: code for code, name in STATUS.items()}
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


@pytest.fixture(scope="module")
def facade(upf_lib, tmp_path_factory):
    exe = tmp_path_factory.mktemp("compat") / "facade_physics"
    subprocess.run([CXX, "-O1", "-std=c++17", "-I" + COMPAT, "-I" + INCLUDE, "-I/usr/local/cuda/include",
                    os.path.join(COMPAT, "facade_physics.cpp"),
                    os.path.join(LIBDIR, "compat", "upf_compat_particles.cpp"), "-o", str(exe),
                    "-L" + LIBDIR, "-lupf_compat", "-lupf", "-Wl,-rpath," + LIBDIR], check=True)
    return str(exe)


def _run(exe, tmp_path, params, sc, steps, entry, body=None):
    n = sc.n
    body = np.full(n, -1, np.int32) if body is None else np.asarray(body, np.int32)
    inp = tmp_path / ("in_%s.bin" % entry)
    out = tmp_path / ("out_%s.bin" % entry)
    with open(inp, "wb") as f:
        f.write(b"UPFC")
        f.write(bytes(params))
        f.write(np.array([n, steps], np.uint32).tobytes())
        f.write(entry.encode().ljust(64, b"\0"))
        f.write(np.ascontiguousarray(sc.pos, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.vel, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.type, np.int32).tobytes())
        f.write(body.tobytes())
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, (r.stdout, r.stderr)
    raw = out.read_bytes()
    status, count, rounded = np.frombuffer(raw[:12], np.int32)
    o = 12
    def take(dtype, k):
        nonlocal o
        a = np.frombuffer(raw[o:o + 4 * k], dtype)
        o += 4 * k
        return a
    res = dict(status=int(status), count=int(count), rounded=int(rounded))
    res["pos"] = take(np.float32, 4 * rounded).reshape(-1, 4)
    res["vel"] = take(np.float32, 4 * rounded).reshape(-1, 4)
    res["pressure"] = take(np.float32, rounded)
    res["density"] = take(np.float32, rounded)
    res["type"] = take(np.int32, rounded)
    res["active"] = take(np.int32, rounded)
    used = UpfParams.from_buffer_copy(raw[o:o + C.sizeof(UpfParams)])
    o += C.sizeof(UpfParams)
    res["params"] = used
    res["message"] = raw[o:o + 256].split(b"\0")[0].decode()
    res["stderr"] = r.stderr
    return res


def test_header_names_are_exported(upf_lib):
    """Every function upf_compat.h declares is exported by libupf_compat.so,
    except CopyParticleDataHostToDevice, which the caller compiles from
    compat/upf_compat_particles.cpp (it reads the caller's particle class)."""
    text = open(os.path.join(INCLUDE, "upf_compat.h")).read()
    body = text[text.index('extern "C" {'):]
    names = set(re.findall(r"^(?:void\*?|uint|upf_status|upf_system\*|const char\*)\s+\**(\w+)\(", body, re.M))
    assert len(names) > 90
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(LIBDIR, "libupf_compat.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = names - exported - {"CopyParticleDataHostToDevice"}
    assert not missing, sorted(missing)


def test_particle_upload_compiles_against_the_reference_class():
    """compat/upf_compat_particles.cpp reads the members of the reference's
    own UnifiedParticle.h (compiled where it lies, when the tree is here)."""
    from oracle import pyoracle
    if not pyoracle.reference_present():
        pytest.skip("reference tree not present")
    src = os.path.join(pyoracle.reference_dir(), "src")
    inc = ["-I" + os.path.join(src, d) for d in ("", "cpu", "sceneConfigure", "system", "vmmlib")]
    subprocess.run([CXX, "-std=c++17", "-fsyntax-only", "-fpermissive", "-w", "-include", "cstring", "-I" + INCLUDE,
                    "-I/usr/local/cuda/include"] + inc +
                   [os.path.join(LIBDIR, "compat", "upf_compat_particles.cpp")], check=True)


def test_facade_without_a_gpu_reports_no_device(facade, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    sc = scenes.small_pcisph(n_side=6)
    from unifiedparticleframeworkcuda_b200 import derive_params
    p = derive_params(sc.params)
    r = _run(facade, tmp_path, p, sc, 2, "ParticlePhysicsOnDeviceFluidStaticBoundariesPCISPH")
    assert r["status"] == CODE["UPF_ERR_NO_DEVICE"], r
    assert "device" in r["message"] and "upf_compat:" in r["stderr"]
    assert r["rounded"] % 64 == 0 and r["rounded"] >= sc.n


def _oracle_run(p, sc, steps):
    from oracle import pyoracle
    o = pyoracle.OracleSim(p, sc.pos, sc.vel, sc.type, keep_fields=False)
    infos = [o.step() for _ in range(steps)]
    st = o.state()
    o.close()
    order = np.argsort(st["id"])
    return {k: v[order] for k, v in st.items()}, infos


@pytest.mark.gpu
@pytest.mark.parametrize("entry,scene", [
    ("ParticlePhysicsOnDeviceFluidStaticBoundariesPCISPH", "small_pcisph"),
    ("ParticlePhysicsOnDevicePCISPH", "small_pcisph_no_boundary_pressure"),
    ("ParticlePhysicsOnDeviceSPH", "small_wcsph"),
])
def test_facade_steps_match_the_oracle(facade, tmp_path, entry, scene):
    """Three steps through the reference's entry points, read back with
    CopyParticlesCUDA in upload order (boundary particles included), against
    the oracle run with the parameters the layer derived from dataPointers:
    those equal the scene's own, and every field agrees within 1e-5."""
    from unifiedparticleframeworkcuda_b200 import FLAG_BOUNDARY_PRESSURE, derive_params
    if scene == "small_pcisph_no_boundary_pressure":
        sc = scenes.small_pcisph(n_side=10)
        sc.params.flags &= ~FLAG_BOUNDARY_PRESSURE
    else:
        sc = getattr(scenes, scene)()
    p = derive_params(sc.params)
    steps = 3
    r = _run(facade, tmp_path, p, sc, steps, entry)
    assert r["status"] == 0, r["message"]
    used = r["params"]
    # the optional GPU terms follow the entry point (upf_compat.h): surface
    # tension always, penalty walls with addBoundaryForce, the Akinci
    # boundary pressure in the static-boundary and coupling pipelines
    from unifiedparticleframeworkcuda_b200 import FLAG_PENALTY_WALLS, FLAG_SURFACE_TENSION
    want_flags = FLAG_SURFACE_TENSION | (p.flags & FLAG_PENALTY_WALLS)
    if "StaticBoundaries" in entry or "RigidCoupling" in entry:
        want_flags |= FLAG_BOUNDARY_PRESSURE
    assert used.flags == want_flags
    # the round trip through dataPointers keeps every other parameter
    for name, _ in UpfParams._fields_:
        if name in ("reserved", "density_error_fudge", "flags"):
            continue
        a, b = getattr(p, name), getattr(used, name)
        a = list(a) if hasattr(a, "__len__") else [a]
        b = list(b) if hasattr(b, "__len__") else [b]
        assert np.array_equal(np.float32(a), np.float32(b)), (name, a, b)
    n = sc.n
    assert r["count"] == n
    want, infos = _oracle_run(used, sc, steps)
    liq = sc.type != FROZEN
    scale = np.abs(want["pos"][:, :3]).max()
    assert np.abs(r["pos"][:n, :3] - want["pos"][:, :3]).max() <= 1e-5 * scale
    vs = max(np.abs(want["vel"][:, :3]).max(), 1e-6)
    assert np.abs(r["vel"][:n, :3] - want["vel"][:, :3]).max() <= 1e-5 * vs
    assert np.array_equal(r["type"][:n], sc.type)
    # the padding of the rounded arrays, as the reference fills it
    assert np.all(r["type"][n:] == 100) and np.all(r["active"] == 100)
    # boundary particles at their fixed positions, Morton key in pos.w
    fz = sc.type == FROZEN
    assert np.array_equal(r["pos"][:n][fz, :3], np.float32(sc.pos)[fz, :3])
    assert np.all(r["pos"][:n, 3] >= 0) and np.all(r["pos"][:n, 3] < 2.0 ** 30)
    if used.method == 2:  # PCISPH: correction pressure and predicted density of the last step
        ds = max(np.abs(want["density"][liq]).max(), 1.0)
        assert np.abs(r["density"][:n][liq] - want["density"][liq]).max() <= 1e-5 * ds
        ps = max(np.abs(want["pressure"][liq]).max(), 1.0)
        assert np.abs(r["pressure"][:n][liq] - want["pressure"][liq]).max() <= 1e-5 * ps


@pytest.mark.gpu
@pytest.mark.parametrize("n,bits", [(1, 8), (3072, 16), (100_003, 30), (262_144, 32)])
def test_legacy_radix_sort_on_interleaved_pairs(upf_lib, n, bits):
    """RadixSort(pData0, pData1, elements, bits) on the reference's
    interleaved (key, value) pairs: a stable sort by the low bits, whole
    8-bit digits as the reference's passes, the result in pData0."""
    torch = pytest.importorskip("torch")
    lib = C.CDLL(os.path.join(LIBDIR, "libupf_compat.so"))
    lib.RadixSort.argtypes = [C.c_void_p, C.c_void_p, C.c_uint, C.c_uint]
    lib.RadixSort.restype = None
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    keys[: n // 5] = keys[0]
    pairs = np.empty((n, 2), np.uint32)
    pairs[:, 0] = keys
    pairs[:, 1] = np.arange(n, dtype=np.uint32)
    d0 = torch.from_numpy(pairs.view(np.int32).copy()).cuda()
    d1 = torch.zeros_like(d0)
    lib.RadixSort(C.c_void_p(d0.data_ptr()), C.c_void_p(d1.data_ptr()), n, bits)
    torch.cuda.synchronize()
    got = d0.cpu().numpy().view(np.uint32)
    digits = (bits + 7) // 8
    mask = np.uint64((1 << (8 * digits)) - 1)
    order = np.argsort((keys.astype(np.uint64) & mask), kind="stable")
    assert np.array_equal(got[:, 1], order.astype(np.uint32))
    assert np.array_equal(got[:, 0], keys[order])
