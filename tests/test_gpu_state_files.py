"""Snapshot files (upf_state_write_file / upf_state_read_file): a run stopped
after k steps and resumed from the file in a fresh system continues bit for
bit like the run that never stopped, rigid bodies included; a file from
another system or a damaged file is refused with the context intact; and the
reference-format text dumps of a device state equal those of its readback."""
import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import LIQUID, STATUS, UpfError, scenes
from unifiedparticleframeworkcuda_b200 import particle_files as pf

pytestmark = pytest.mark.gpu
CODE = {name: code for code, name in STATUS.items()}


def _system(upf, sc, params=None, bodies=True):
    p = params if params is not None else upf.derive_params(sc.params)
    s = upf.ParticleSystem(p, capacity=sc.n, derive=False)
    s.set_particles(sc.pos, sc.vel, sc.type)
    if bodies and getattr(sc, "num_bodies", 0):
        s.set_rigid_bodies(sc.body, sc.num_bodies)
    return s


@pytest.mark.parametrize("scene", ["small_pcisph", "small_coupling"])
def test_resume_from_a_state_file_is_bit_exact(upf_lib, tmp_path, scene):
    sc = getattr(scenes, scene)()
    path = tmp_path / "run.upfstate"
    with _system(upf_lib, sc) as a:
        a.step(3)
        a.write_state_file(path)
        a.step(4)
        ref = a.particles()
        ref_bodies = a.rigid_bodies() if getattr(sc, "num_bodies", 0) else None
    info = pf.state_file_info(path)
    assert info["n_dynamic"] == len(ref["id"]) and info["num_bodies"] == getattr(sc, "num_bodies", 0)
    with _system(upf_lib, sc, params=info["params"]) as b:
        b.read_state_file(path)
        b.step(4)
        got = b.particles()
        got_bodies = b.rigid_bodies() if ref_bodies is not None else None
    for k in ("pos", "vel", "density", "pressure", "id", "type"):
        assert np.array_equal(ref[k], got[k]), k
    if ref_bodies is not None:
        for k, (x, y) in enumerate(zip(ref_bodies, got_bodies)):
            assert np.array_equal(x, y), k


def test_foreign_or_damaged_state_files_are_refused(upf_lib, tmp_path):
    sc = scenes.small_pcisph()
    path = tmp_path / "run.upfstate"
    with _system(upf_lib, sc) as a:
        a.step(1)
        a.write_state_file(path)
        before = a.particles()
        raw = bytearray(path.read_bytes())
        raw[-100] ^= 0x40
        bad = tmp_path / "damaged.upfstate"
        bad.write_bytes(bytes(raw))
        with pytest.raises(UpfError) as e:
            a.read_state_file(bad)
        assert e.value.status == CODE["UPF_ERR_IO"] and "checksum" in str(e.value)
        short = tmp_path / "short.upfstate"
        short.write_bytes(bytes(raw[: len(raw) // 2]))
        with pytest.raises(UpfError) as e:
            a.read_state_file(short)
        assert e.value.status == CODE["UPF_ERR_IO"]
        (tmp_path / "text.txt").write_text("not a state file\n" * 10)
        with pytest.raises(UpfError) as e:
            a.read_state_file(tmp_path / "text.txt")
        assert e.value.status == CODE["UPF_ERR_IO"]
        # nothing above changed the state: the system steps on as before
        assert np.array_equal(a.particles()["pos"], before["pos"])
        a.step(1)
        a.synchronize()
    other = scenes.small_wcsph()
    with _system(upf_lib, other) as c:
        with pytest.raises(UpfError) as e:
            c.read_state_file(path)
        assert e.value.status == CODE["UPF_ERR_INVALID_ARG"]
    # the same scene under another time step: the snapshot would resume
    # under the wrong physics, so it is refused and the field is named
    changed = scenes.small_pcisph()
    changed.params.dt = sc.params.dt * 0.5
    with _system(upf_lib, changed) as d:
        with pytest.raises(UpfError) as e:
            d.read_state_file(path)
        assert e.value.status == CODE["UPF_ERR_INVALID_ARG"] and "dt" in str(e.value)


def test_text_dumps_of_a_device_state(upf_lib, tmp_path):
    """The reference writes its dumps from the device copies it reads back
    (UnifiedPhysics.cpp:6176-6178): the liquid dump holds the liquid
    particles' positions, the PCISPH-format file reads back to the state."""
    sc = scenes.small_coupling()
    with _system(upf_lib, sc) as s:
        s.step(2)
        st = s.particles()
    pf.save_liquid_info_full(tmp_path / "liquid.txt", st["pos"], st["type"])
    lines = (tmp_path / "liquid.txt").read_text().splitlines()
    liquid = st["type"] == LIQUID
    assert int(lines[0]) == int(liquid.sum()) == len(lines) - 1
    assert np.allclose(np.array([[float(v) for v in ln.split()[:3]] for ln in lines[1:]]),
                       st["pos"][liquid, :3], rtol=1e-7, atol=0)
    pf.save_fluid_particles_pcisph(tmp_path / "fluid.txt", st["pos"], st["vel"], st["type"], st["pressure"],
                                   st["density"])
    back = pf.read_fluid_particles_pcisph(tmp_path / "fluid.txt")
    assert np.array_equal(back["pos"], st["pos"][:, :3]) and np.array_equal(back["vel"], st["vel"][:, :3])
    assert np.array_equal(back["type"], st["type"])
