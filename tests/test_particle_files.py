"""Particle files in the reference's text formats (src/cpu/UnifiedIO.cpp,
src/sceneConfigure/Scene.cpp), written and read by the library on the host.

Bars: the writers' output is byte-identical to the reference's writers (the
golden fixture holds the bytes the reference wrote, from
tests/golden/make_golden.py; at larger sizes the compiled reference is run
directly when oracle/_ref is built); the readers return bit-identical values
to the reference's reader on the same file."""
import ctypes as C
import os

import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import STATUS, UpfError
from unifiedparticleframeworkcuda_b200 import particle_files as pf

HERE = os.path.dirname(os.path.abspath(__file__))
CODE = {name: code for code, name in STATUS.items()}


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "reference_io.npz"))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_liquid_rigid_and_position_dumps_are_the_reference_bytes(upf_lib, gold, tmp_path):
    pos, t = gold["pos"], gold["type"]
    pf.save_liquid_info_full(tmp_path / "liquid.txt", pos, t, int(gold["num_liquid"]))
    pf.save_rigid_info_full(tmp_path / "rigid.txt", pos, t, int(gold["num_rigid"]))
    pf.save_particle_positions(tmp_path / "positions.txt", pos)
    assert (tmp_path / "liquid.txt").read_bytes() == bytes(gold["liquid_txt"])
    assert (tmp_path / "rigid.txt").read_bytes() == bytes(gold["rigid_txt"])
    assert (tmp_path / "positions.txt").read_bytes() == bytes(gold["positions_txt"])


def test_pcisph_reader_matches_the_reference_reader(upf_lib, gold, tmp_path):
    path = tmp_path / "fluid_in.txt"
    path.write_bytes(bytes(gold["reader_txt"]))
    assert pf.read_fluid_particle_num(path) == len(gold["read_type"])
    got = pf.read_fluid_particles_pcisph(path)
    for k in ("pos", "vel", "corr_pressure", "predicted_density"):
        assert np.array_equal(bits(got[k]), bits(gold["read_" + k])), k
    assert np.array_equal(got["type"], gold["read_type"])


def test_pcisph_file_round_trips_exactly(upf_lib, tmp_path):
    rng = np.random.default_rng(7)
    n = 5000
    pos = (rng.normal(size=(n, 4)) * 10.0 ** rng.integers(-6, 6, (n, 4))).astype(np.float32)
    vel = rng.normal(size=(n, 4)).astype(np.float32)
    t = rng.integers(0, 7, n).astype(np.int32)
    p = rng.uniform(0, 1e4, n).astype(np.float32)
    rho = rng.uniform(900, 1100, n).astype(np.float32)
    path = tmp_path / "fluid.txt"
    pf.save_fluid_particles_pcisph(path, pos, vel, t, p, rho)
    got = pf.read_fluid_particles_pcisph(path)
    assert np.array_equal(bits(got["pos"]), bits(pos[:, :3]))
    assert np.array_equal(bits(got["vel"]), bits(vel[:, :3]))
    assert np.array_equal(got["type"], t)
    assert np.array_equal(bits(got["corr_pressure"]), bits(p))
    assert np.array_equal(bits(got["predicted_density"]), bits(rho))


def test_scene_particle_file_round_trip_skips_granular(upf_lib, tmp_path):
    """Scene::saveParticles / readInParticles (Scene.cpp:218-279; not
    compilable here, so restated): 6 significant digits, type as a float,
    a trailing empty line; granular records are skipped on reading."""
    rng = np.random.default_rng(3)
    n = 1000
    pos = rng.uniform(-2, 2, (n, 4)).astype(np.float32)
    t = rng.choice(np.array([0, 2, 3, 6], np.int32), n)
    mass = rng.uniform(0.1, 2, n).astype(np.float32)
    path = tmp_path / "scene.txt"
    pf.save_scene_particles(path, pos, t, rest_density=1000.0, mass=mass)
    text = path.read_text()
    assert text.endswith(" \n\n")
    first = text.splitlines()[0].split()
    assert first == ["%g" % float(pos[0, 0]), "%g" % float(pos[0, 1]), "%g" % float(pos[0, 2]), "1000",
                     "%g" % float(mass[0]), "%g" % float(t[0])]
    got = pf.read_scene_particles(path)
    keep = t != 3
    six = np.vectorize(lambda v: np.float32(float("%g" % float(v))))
    assert np.array_equal(got["type"], t[keep])
    assert np.array_equal(bits(got["pos"][:, :3]), bits(six(pos[keep, :3])))
    assert np.array_equal(bits(got["mass"]), bits(six(mass[keep])))
    assert np.all(got["density"] == 1000.0)


def test_stream_extraction_rules(upf_lib, tmp_path):
    """The reader takes what operator>> takes: an int field stops at the
    first non-digit ("2.0" is 2, and ".0" is the next field), floats accept
    "1.", ".5", "+3e2", exponents need a mantissa digit before them."""
    path = tmp_path / "edge.txt"
    path.write_text("2\n1. .5 +3e2 2.0 -0 1e-45 7 8 9\n4 5 6 +6 -1e+2 0.25\t\t3\n0 1e5\n")
    got = pf.read_fluid_particles_pcisph(path)
    assert got["pos"][0].tolist() == [1.0, 0.5, 300.0]
    assert got["type"][0] == 2
    assert got["vel"][0, 0] == 0.0 and got["vel"][0, 1] == 0.0 and np.signbit(got["vel"][0, 1])
    assert bits(got["vel"][0, 2]) == 1  # 1e-45 is the smallest denormal
    assert got["corr_pressure"][0] == 7 and got["predicted_density"][0] == 8
    assert got["pos"][1].tolist() == [9.0, 4.0, 5.0]
    assert got["type"][1] == 6 and got["vel"][1].tolist() == [6.0, -100.0, 0.25]
    assert got["corr_pressure"][1] == 3 and got["predicted_density"][1] == 0


def test_reader_errors_are_reported(upf_lib, tmp_path):
    with pytest.raises(UpfError) as e:
        pf.read_fluid_particle_num(tmp_path / "missing.txt")
    assert e.value.status == CODE["UPF_ERR_IO"]
    bad = tmp_path / "truncated.txt"
    bad.write_text("3\n1 2 3 2 0 0 0 0 1000\n1 2 3 2 0 0\n")
    L = upf_lib.lib()
    n = 3
    pos = np.zeros((n, 3), np.float32)
    vel = np.zeros((n, 3), np.float32)
    t = np.zeros(n, np.int32)
    p = np.zeros(n, np.float32)
    r = np.zeros(n, np.float32)
    got = C.c_int32()
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    rc = L.upf_io_read_fluid_particles_pcisph(os.fsencode(bad), fp(pos), fp(vel),
                                              t.ctypes.data_as(C.POINTER(C.c_int32)), fp(p), fp(r), n,
                                              C.byref(got))
    assert rc == CODE["UPF_ERR_IO"] and got.value == 1 and r[0] == 1000
    assert b"record 1" in L.upf_last_error()
    rc = L.upf_io_read_fluid_particles_pcisph(os.fsencode(bad), fp(pos), fp(vel),
                                              t.ctypes.data_as(C.POINTER(C.c_int32)), fp(p), fp(r), 2,
                                              C.byref(got))
    assert rc == CODE["UPF_ERR_INVALID_ARG"]  # 3 records, capacity 2
    scene = tmp_path / "scene_bad.txt"
    scene.write_text("0 0 0 1000 1 2 \n0 0 zero 1000 1 2\n")
    with pytest.raises(UpfError) as e:
        pf.read_scene_particles(scene)
    assert e.value.status == CODE["UPF_ERR_IO"]
    with pytest.raises(UpfError) as e:
        pf.save_particle_positions(tmp_path / "no_such_dir" / "x.txt", np.zeros((2, 4), np.float32))
    assert e.value.status == CODE["UPF_ERR_IO"]


def test_empty_inputs(upf_lib, tmp_path):
    z4 = np.zeros((0, 4), np.float32)
    z = np.zeros(0, np.int32)
    pf.save_liquid_info_full(tmp_path / "l.txt", z4, z, 0)
    assert (tmp_path / "l.txt").read_bytes() == b"0\n"
    pf.save_particle_positions(tmp_path / "p.txt", z4)
    assert (tmp_path / "p.txt").read_bytes() == b"0\n"
    pf.save_fluid_particles_pcisph(tmp_path / "f.txt", z4, z4, z)
    assert pf.read_fluid_particles_pcisph(tmp_path / "f.txt")["type"].size == 0
    pf.save_scene_particles(tmp_path / "s.txt", z4, z)
    assert pf.read_scene_particles(tmp_path / "s.txt")["type"].size == 0


needs_ref = pytest.mark.skipif(
    not os.path.exists(os.path.join(HERE, "..", "oracle", "_ref", "libupfref.so")),
    reason="reference pin library (oracle/_ref) not built")


@needs_ref
def test_writers_match_the_compiled_reference_at_scale(upf_lib, tmp_path):
    """300k particles: formatted on several threads here, one stream in the
    reference; the bytes must agree."""
    from oracle import pyoracle
    from tests.golden.make_golden import io_positions
    rng = np.random.default_rng(11)
    n = 300_000
    pos = io_positions(rng, n)
    t = rng.choice(np.array([0, 2, 3, 6], np.int32), n).astype(np.int32)
    work = tmp_path / "ref"
    work.mkdir()
    nl = int(np.count_nonzero(t == 2))
    pf.save_liquid_info_full(tmp_path / "l.txt", pos, t, nl)
    assert (tmp_path / "l.txt").read_bytes() == pyoracle.ref_io_write("liquid", str(work), pos, t, nl)
    pf.save_rigid_info_full(tmp_path / "r.txt", pos, t, 17)
    assert (tmp_path / "r.txt").read_bytes() == pyoracle.ref_io_write("rigid", str(work), pos, t, 17)
    pf.save_particle_positions(tmp_path / "p.txt", pos[:50_000])
    assert (tmp_path / "p.txt").read_bytes() == pyoracle.ref_io_write("positions", str(work), pos[:50_000])


@needs_ref
def test_reference_reader_reads_the_library_pcisph_file(upf_lib, tmp_path):
    from oracle import pyoracle
    rng = np.random.default_rng(5)
    n = 20_000
    pos = rng.normal(size=(n, 4)).astype(np.float32)
    vel = rng.normal(size=(n, 4)).astype(np.float32)
    t = rng.integers(0, 7, n).astype(np.int32)
    p = rng.uniform(0, 1e4, n).astype(np.float32)
    rho = rng.uniform(900, 1100, n).astype(np.float32)
    path = tmp_path / "fluid.txt"
    pf.save_fluid_particles_pcisph(path, pos, vel, t, p, rho)
    ref = pyoracle.ref_io_read_pcisph(str(path))
    ours = pf.read_fluid_particles_pcisph(path)
    for k in ("pos", "vel", "corr_pressure", "predicted_density"):
        assert np.array_equal(bits(ref[k]), bits(ours[k])), k
    assert np.array_equal(ref["type"], ours["type"])
    assert np.array_equal(bits(ours["pos"]), bits(pos[:, :3]))


@needs_ref
def test_stream_extraction_rules_match_the_reference_reader(upf_lib, tmp_path):
    from oracle import pyoracle
    path = tmp_path / "edge.txt"
    # record 2: position 1e5, 12, -2.5e-4; type -7; velocity 50, FLT_MAX,
    # -FLT_MIN; pressure a denormal; density 100; the trailing ".0" is unread
    path.write_text("3\n1. .5 +3e2 2.0 -0 1e-45 7 8 9\n4 5 6 +6 -1e+2 0.25\t\t3\n0 1e5\n"
                    "0012 -.25e-3 -7 5E+1 3.4028235e38 -1.17549435e-38 2e-39\n1e2 .0\n")
    ref = pyoracle.ref_io_read_pcisph(str(path))
    ours = pf.read_fluid_particles_pcisph(path)
    for k in ("pos", "vel", "corr_pressure", "predicted_density"):
        assert np.array_equal(bits(ref[k]), bits(ours[k])), k
    assert np.array_equal(ref["type"], ours["type"])
