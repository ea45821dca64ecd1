"""PLY files (autoquantizer_b200.mesh_io): the particle dump layout of
mpm_exps/engine/mesh_io.py:49-80 byte for byte, and the reader on ascii,
little- and big-endian files with list properties (meshes)."""
import numpy as np
import pytest

from autoquantizer_b200 import mesh_io as M


def test_packed_dump_layout(tmp_path):
    fn = str(tmp_path / "data_000000.ply")
    pos = np.array([[0.1, 0.2, 0.3], [1.5, -2.0, 4.25]], dtype=np.float32)
    M.write_point_cloud_packed(fn, pos, 2)
    raw = open(fn, "rb").read()
    head = (b"ply\nformat binary_little_endian 1.0\ncomment Created by taichi\nelement vertex 2\n"
            b"property float x\nproperty float y\nproperty float z\nend_header\n")
    assert raw == head + pos.astype("<f4").tobytes()
    assert np.array_equal(M.load_particles_only(fn), pos)


def test_point_cloud_with_velocities(tmp_path):
    fn = str(tmp_path / "pv.ply")
    a = np.arange(18, dtype=np.float32).reshape(3, 6)
    M.write_point_cloud(fn, a)
    el = M.read_ply(fn)["vertex"]
    assert list(el) == ["x", "y", "z", "vel_x", "vel_y", "vel_z"]
    assert np.array_equal(np.stack(list(el.values()), 1), a)


def test_writer_rejects_bad_shapes(tmp_path):
    with pytest.raises(ValueError):
        M.write_point_cloud_packed(str(tmp_path / "a.ply"), np.zeros((4, 2)), 4)
    with pytest.raises(ValueError):
        M.write_point_cloud_packed(str(tmp_path / "a.ply"), np.zeros((4, 3)), 5)


def _cube():
    v = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], dtype=np.float64)
    f = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                  [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]])
    return v, f


def _write_mesh(fn, v, f, fmt):
    head = ["ply", "format %s 1.0" % fmt, "element vertex %d" % len(v), "property double x", "property double y",
            "property double z", "element face %d" % len(f), "property list uchar int vertex_indices", "end_header"]
    with open(fn, "wb") as out:
        out.write(("\n".join(head) + "\n").encode())
        if fmt == "ascii":
            for p in v:
                out.write(("%.17g %.17g %.17g\n" % tuple(p)).encode())
            for t in f:
                out.write(("3 %d %d %d\n" % tuple(t)).encode())
            return
        e = "<" if fmt == "binary_little_endian" else ">"
        out.write(v.astype(e + "f8").tobytes())
        for t in f:
            out.write(np.uint8(3).tobytes() + t.astype(e + "i4").tobytes())


@pytest.mark.parametrize("fmt", ["ascii", "binary_little_endian", "binary_big_endian"])
def test_mesh_reader(tmp_path, fmt):
    v, f = _cube()
    fn = str(tmp_path / "cube.ply")
    _write_mesh(fn, v, f, fmt)
    tri = M.load_mesh(fn, scale=(2.0, 3.0, 4.0), offset=(0.5, 0.0, -1.0))
    want = (v * [2.0, 3.0, 4.0] + [0.5, 0.0, -1.0])[f].reshape(-1, 9).astype(np.float32)
    assert tri.dtype == np.float32 and np.array_equal(tri, want)
    verts, idx = M.load_mesh_vertices_and_indices(fn)
    assert np.array_equal(idx, f.ravel())
    assert np.array_equal(verts, np.stack([v[:, 0], v[:, 2], -v[:, 1]], 1))


def test_not_a_ply(tmp_path):
    fn = str(tmp_path / "x.ply")
    open(fn, "wb").write(b"solid cube\n")
    with pytest.raises(ValueError):
        M.read_ply(fn)


def test_ragged_faces_and_large_meshes(tmp_path):
    fn = str(tmp_path / "mixed.ply")
    v = np.arange(15, dtype="<f4").reshape(5, 3)
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex 5\nproperty float x\nproperty float y\n"
            "property float z\nelement face 2\nproperty list uchar int vertex_indices\nend_header\n").encode()
    body = v.tobytes() + np.uint8(3).tobytes() + np.array([0, 1, 2], "<i4").tobytes() + \
        np.uint8(4).tobytes() + np.array([1, 2, 3, 4], "<i4").tobytes()
    open(fn, "wb").write(head + body)
    faces = M.read_ply(fn)["face"]["vertex_indices"]
    assert [f.tolist() for f in faces] == [[0, 1, 2], [1, 2, 3, 4]]
    with pytest.raises(ValueError):
        M.load_mesh(fn)
    # 200k triangles read through the vectorized path
    n = 200000
    rng = np.random.default_rng(1)
    f = rng.integers(0, 5, (n, 3)).astype("<i4")
    rec = np.zeros(n, dtype=[("n", "u1"), ("i", "<i4", (3,))])
    rec["n"], rec["i"] = 3, f
    head = head.replace(b"element face 2", b"element face %d" % n)
    open(fn, "wb").write(head + v.tobytes() + rec.tobytes())
    tri = M.load_mesh(fn)
    assert tri.shape == (n, 9) and np.array_equal(tri.reshape(n, 3, 3), v[f])
