"""OBJ triangle reading (upf_obj_read_triangles, the reference's
ObjLoader::Load) and the procedural closed meshes the voxeliser fills; the
voxeliser itself runs on the GPU (tests/test_gpu_scene.py)."""
import os

import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import STATUS, UpfError, scenes

CODE = {name: code for code, name in STATUS.items()}
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("mesh", ["ico", "torus", "box"])
def test_written_obj_reads_back_exactly(upf_lib, tmp_path, mesh):
    tri = {"ico": scenes.mesh_icosphere(0.1, 2, (0.3, -0.2, 0.25)),
           "torus": scenes.mesh_torus(center=(0.2, 0.1, 0.3)),
           "box": scenes.mesh_box(rotation_seed=3)}[mesh]
    path = tmp_path / "m.obj"
    scenes.write_obj(path, tri)
    got = upf_lib.obj_triangles(path)
    # the file ends with a newline-terminated face line: listed twice, as the
    # reference's read loop lists it
    want = np.concatenate([tri, tri[-1:]])
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_last_line_is_read_twice_like_the_reference(upf_lib, tmp_path):
    """ObjLoader::Load loops `while (!feof(fp)) { fgets(...); ... }`: after
    a newline-terminated last line, one more pass reads nothing and handles
    the same buffer again. A last face line therefore appears twice; without
    the final newline, or after a trailing comment, it appears once."""
    head = "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 2 3\nf 1 2 4"
    cases = {head + "\n": 3, head: 2, head + "\n# end\n": 2, head + "\nv 5 5 5\n": 2}
    for k, (text, faces) in enumerate(cases.items()):
        path = tmp_path / ("c%d.obj" % k)
        path.write_text(text)
        assert len(upf_lib.obj_triangles(path)) == faces, repr(text)


def test_procedural_meshes_are_closed_and_outward(upf_lib):
    for tri in (scenes.mesh_icosphere(0.1, 2), scenes.mesh_torus(), scenes.mesh_box(rotation_seed=1)):
        t = tri.astype(np.float64).reshape(-1, 3, 3)
        # every edge is shared by exactly two faces, once in each direction
        edges = {}
        for f in t:
            for a in range(3):
                e = (tuple(f[a]), tuple(f[(a + 1) % 3]))
                edges[e] = edges.get(e, 0) + 1
        assert all(edges.get((b, a), 0) == 1 for (a, b) in edges)
        # signed volume > 0: counter-clockwise seen from outside
        vol = np.einsum("ij,ij->i", t[:, 0], np.cross(t[:, 1], t[:, 2])).sum() / 6.0
        assert vol > 0


def test_face_spellings_and_errors(upf_lib, tmp_path):
    path = tmp_path / "f.obj"
    path.write_text("# test\ng g0\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nvt 0 0\nvn 0 0 1\n"
                    "f 1/1/1 2/1/1 3/1/1\nf 1 2 4\nf 1//1 3//1 4//1\nf 2/1 3/1 4/1 1/1\nusemtl x\n")
    t = upf_lib.obj_triangles(path).reshape(-1, 3, 3)
    assert t.shape == (4, 3, 3)
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    assert np.array_equal(t[0], v[[0, 1, 2]]) and np.array_equal(t[1], v[[0, 1, 3]])
    assert np.array_equal(t[2], v[[0, 2, 3]]) and np.array_equal(t[3], v[[1, 2, 3]])
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nf 1/1/1 2/1/1 3/1/1\n")
    with pytest.raises(UpfError) as e:
        upf_lib.obj_triangles(bad)
    assert e.value.status == CODE["UPF_ERR_IO"] and "vertex 3 of 2" in str(e.value)
    bad.write_text("v 0 0\n")
    with pytest.raises(UpfError) as e:
        upf_lib.obj_triangles(bad)
    assert e.value.status == CODE["UPF_ERR_IO"]
    with pytest.raises(UpfError) as e:
        upf_lib.obj_triangles(tmp_path / "missing.obj")
    assert e.value.status == CODE["UPF_ERR_IO"]


def test_golden_meshes_are_the_library_meshes(upf_lib):
    """The fixture's meshes are the procedural meshes (so the GPU test fills
    exactly what the reference filled)."""
    from tests.golden.make_golden import mesh_cases
    gold = np.load(os.path.join(HERE, "golden", "reference_mesh.npz"))
    for name, tri, scale, spacing in mesh_cases():
        assert np.array_equal(gold[name + "_tri"], tri), name
        assert np.array_equal(gold[name + "_scale"], np.array(scale, np.float32)), name


needs_ref = pytest.mark.skipif(
    not os.path.exists(os.path.join(HERE, "..", "oracle", "_ref", "libupfref.so")),
    reason="reference pin library (oracle/_ref) not built")


@needs_ref
def test_reference_voxeliser_reproduces_the_fixture(upf_lib, tmp_path):
    from oracle import pyoracle
    from tests.golden.make_golden import mesh_cases
    gold = np.load(os.path.join(HERE, "golden", "reference_mesh.npz"))
    for name, tri, scale, spacing in mesh_cases()[:3]:
        path = tmp_path / (name + ".obj")
        scenes.write_obj(path, tri)
        assert np.array_equal(pyoracle.ref_obj_particles(str(path), scale, spacing), gold[name + "_pos"]), name


# ---------------------------------------------------------------- scene generators
# The reference's Scene.cpp does not compile here, so the generators are
# restated in the oracle (oracle/scene_oracle.cpp); the restatement is
# checked here against an independent numpy reading of the same loops, and
# the device generators against the restatement (tests/test_gpu_scene.py).

def _numpy_fluid_block(box_min, box_max, spacing, jitter, offset):
    f = np.float32
    box_min, box_max, offset = (np.asarray(v, f) for v in (box_min, box_max, offset))
    num = [int(f(f(box_max[a] - box_min[a]) / f(spacing))) for a in range(3)]
    out = []
    for iy in range(num[1]):
        y = f(f(jitter) + f(f(iy) * f(spacing)))
        for ix in range(num[0]):
            x = f(f(jitter) + f(f(ix) * f(spacing)))
            for iz in range(num[2]):
                z = f(f(jitter) + f(f(iz) * f(spacing)))
                sh = -0.5 * float(f(jitter))
                out.append([f(float(c) + sh + float(o)) for c, o in zip((x, y, z), offset)] + [0.0])
    return np.array(out, f).reshape(-1, 4)


def test_fluid_block_restatement(upf_lib):
    from oracle import pyoracle
    for args in [((0.0, 0.0, 0.0), (0.13, 0.1, 0.07), 0.01, 0.0, (0.04, 0.035, 0.04)),
                 ((-0.5, 0.2, -0.1), (-0.41, 0.27, 0.0), 0.0125, 0.003, (0.1, -0.2, 0.3))]:
        got = pyoracle.scene_fluid_block(*args)
        want = _numpy_fluid_block(*args)
        assert got.shape == want.shape and np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_box_boundary_restatement_counts_and_order(upf_lib):
    from oracle import pyoracle
    cmin, cmax, zs = (0.0, 0.0, 0.0), (0.3, 0.2, 0.25), (-0.06, -0.06, -0.06)
    sp, h, d = 0.01, 0.04, 0.005
    for layers in (1, 2, 3):
        pos, nrm = pyoracle.scene_box_boundary(cmin, cmax, zs, sp, h, d, layers)
        num = [int(np.float32(np.float32(np.float32(cmax[a]) + np.float32(d)) -
                              np.float32(np.float32(cmin[a]) - np.float32(d))) / np.float32(sp)) for a in range(3)]
        nx, ny, nz = num
        assert len(pos) == 2 * layers * ((nx + 2) * (nz + 2) + (nx + 2) * ny + ny * nz)
        # the first pair: ground then ceiling at the first lattice column
        assert nrm[0, 1] == 1 and nrm[1, 1] == -1 and pos[0, 0] == pos[1, 0] and pos[0, 2] == pos[1, 2]
        f = np.float32
        base = f(f(zs[0]) + f(f(h) - f(d)))
        assert pos[0, 0] == base and pos[0, 1] == f(f(zs[1]) + f(f(h) - f(d)))
        # every normal points into the box along one axis
        assert np.all(np.abs(nrm[:, :3]).sum(1) == 1)
    # a wall at the z-index origin: where the reference aborts
    assert pyoracle.scene_box_boundary(cmin, cmax, (0.0, 0.0, 0.0), sp, 0.005, 0.005, 1) is None
