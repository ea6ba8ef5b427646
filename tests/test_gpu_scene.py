"""The device mesh voxeliser (upf_mesh_particles) against the reference's
ObjectLoader::LoadParticles: on every golden mesh the particles, their
positions and their order are bit-identical to what the compiled reference
produced (tests/golden/reference_mesh.npz, from tests/golden/make_golden.py),
reading the mesh through upf_obj_read_triangles as the reference reads it."""
import ctypes as C
import os

import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import STATUS, UpfError, scenes

pytestmark = pytest.mark.gpu
CODE = {name: code for code, name in STATUS.items()}
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "reference_mesh.npz"))
CASES = sorted({k[: -len("_tri")] for k in GOLD.files if k.endswith("_tri")})


@pytest.mark.parametrize("name", CASES)
def test_mesh_particles_match_the_reference_voxeliser(upf_lib, tmp_path, name):
    path = tmp_path / (name + ".obj")
    scenes.write_obj(path, GOLD[name + "_tri"])
    tri = upf_lib.obj_triangles(path)
    got = upf_lib.mesh_particles(tri, float(GOLD[name + "_spacing"]), GOLD[name + "_scale"])
    want = GOLD[name + "_pos"]
    assert got.shape[0] == want.shape[0]
    assert np.array_equal(got[:, :3].view(np.uint32), want.view(np.uint32))
    assert np.all(got[:, 3] == 0)


def _read_as_obj(upf, tmp_path, name):
    path = tmp_path / (name + ".obj")
    scenes.write_obj(path, GOLD[name + "_tri"])
    return np.ascontiguousarray(upf.obj_triangles(path))


def test_count_capacity_and_bad_arguments(upf_lib, tmp_path):
    L = upf_lib.lib()
    tri = _read_as_obj(upf_lib, tmp_path, "icosphere")
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    n = C.c_uint32()
    assert L.upf_mesh_particles(0, fp(tri), len(tri), 1.0, 1.0, 1.0, 0.012, None, 0, C.byref(n)) == 0
    assert n.value == len(GOLD["icosphere_pos"])
    small = np.zeros((10, 4), np.float32)
    rc = L.upf_mesh_particles(0, fp(tri), len(tri), 1.0, 1.0, 1.0, 0.012, fp(small), 10, C.byref(n))
    assert rc == CODE["UPF_ERR_INVALID_ARG"] and n.value == len(GOLD["icosphere_pos"])
    assert L.upf_mesh_particles(0, fp(tri), len(tri), 1.0, 1.0, 1.0, 0.0, None, 0, C.byref(n)) == 1
    # a lattice beyond the 2^31-point limit is refused before any device work
    rc = L.upf_mesh_particles(0, fp(tri), len(tri), 1.0, 1.0, 1.0, 1e-5, None, 0, C.byref(n))
    assert rc == CODE["UPF_ERR_INVALID_ARG"] and "limit" in L.upf_last_error().decode()
    # an empty mesh fills nothing, as in the reference
    assert L.upf_mesh_particles(0, None, 0, 1.0, 1.0, 1.0, 0.01, None, 0, C.byref(n)) == 0 and n.value == 0


def test_injected_allocation_failure_is_reported(upf_lib, tmp_path):
    L = upf_lib.lib()
    tri = _read_as_obj(upf_lib, tmp_path, "torus")
    try:
        L.upf_test_fail_allocation(2)
        with pytest.raises(UpfError) as e:
            upf_lib.mesh_particles(tri, 0.015, (1.5, 2.0, 1.0))
        assert e.value.status == CODE["UPF_ERR_ALLOC"] and "injected" in str(e.value)
    finally:
        L.upf_test_fail_allocation(-1)
    assert len(upf_lib.mesh_particles(tri, 0.015, (1.5, 2.0, 1.0))) == len(GOLD["torus_pos"])


FLUID_CASES = [
    ((0.0, 0.0, 0.0), (0.13, 0.1, 0.07), 0.01, 0.0, (0.04, 0.035, 0.04)),
    ((-0.5, 0.2, -0.1), (-0.41, 0.27, 0.0), 0.0125, 0.003, (0.1, -0.2, 0.3)),
    ((0.02, 0.02, 0.02), (1.30, 1.30, 0.66), 0.01, 0.001, (0.03, 0.025, 0.03)),  # 128 x 128 x 64
]


@pytest.mark.parametrize("case", range(len(FLUID_CASES)))
def test_fluid_block_matches_the_restated_reference(upf_lib, case):
    from oracle import pyoracle
    args = FLUID_CASES[case]
    got = upf_lib.scene_fluid_block(*args)
    want = pyoracle.scene_fluid_block(*args)
    assert got.shape == want.shape and len(got) > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("layers", [1, 2, 3])
@pytest.mark.parametrize("h", [0.02, 0.04])
def test_box_boundary_matches_the_restated_reference(upf_lib, layers, h):
    from oracle import pyoracle
    args = ((0.0, 0.0, 0.0), (2.0, 1.3, 1.3), (-0.05, -0.05, -0.05), 0.01, h, 0.005)
    want = pyoracle.scene_box_boundary(*args, layers)
    if want is None:  # an inner layer reaches the z-index origin: the reference aborts
        with pytest.raises(UpfError) as e:
            upf_lib.scene_box_boundary(*args, layers=layers)
        assert e.value.status == CODE["UPF_ERR_INVALID_ARG"]
        return
    wpos, wnrm = want
    pos, nrm = upf_lib.scene_box_boundary(*args, layers=layers)
    assert pos.shape == wpos.shape
    assert np.array_equal(pos.view(np.uint32), wpos.view(np.uint32))
    assert np.array_equal(nrm, wnrm)


def test_box_boundary_refuses_walls_at_the_origin(upf_lib):
    with pytest.raises(UpfError) as e:
        upf_lib.scene_box_boundary((0.0, 0.0, 0.0), (0.3, 0.2, 0.25), (0.0, 0.0, 0.0), 0.01, 0.005, 0.005, 1)
    assert e.value.status == CODE["UPF_ERR_INVALID_ARG"] and "origin" in str(e.value)


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_rigid_surface_on_gpu_equals_the_host_sampler(upf_lib, shape):
    """upf_scene_rigid_surface against the host samplers of the coupling
    scenes (scenes.sample_sphere / sample_box / sample_torus, rotated and
    moved in double): the same count, and every point within 1e-6 m (the two
    evaluate cos, sin and acos in different double libraries before rounding
    to float)."""
    rng = np.random.default_rng(shape)
    for r, n in ((0.05, 2000), (0.13, 7777)):
        R = scenes._random_rotation(rng.uniform(size=3))
        c = rng.uniform(0.2, 1.0, 3)
        want = (scenes.sample_sphere, scenes.sample_box, scenes.sample_torus)[shape](r, n) @ R.T + c
        got = upf_lib.scene_rigid_surface(shape, r, n, R.astype(np.float32), c.astype(np.float32))
        assert got.shape[0] == want.shape[0]
        # the host sampler works from the double radius and rotation; the
        # device takes them as float, so compare at float input precision
        want32 = (scenes.sample_sphere, scenes.sample_box, scenes.sample_torus)[shape](
            float(np.float32(r)), n) @ R.astype(np.float32).astype(np.float64).T + c.astype(np.float32)
        assert np.abs(got[:, :3] - want32).max() <= 1e-6
        assert np.abs(got[:, :3] - want).max() <= 1e-5 and np.all(got[:, 3] == 0)
