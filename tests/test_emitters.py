"""Particle emitters on the host and the voxelizer's CPU restatement
(oracle/aq_oracle_emit.c, voxelizer.py:53-105) on meshes whose voxels are
known in closed form."""
import numpy as np
import pytest

import oracle as O
from autoquantizer_b200 import scenes
from autoquantizer_b200.mpm_solver import MPMSolver
from helpers import box_mesh, sphere_mesh

PAD = 3


def _box_voxels(lo, hi, res, dx):
    """Voxels inside [lo, hi]: columns whose centres the box covers, from
    int(lo_z / dx + 0.5) to int(hi_z / dx + 0.5) (the column heights of the
    bottom and top faces), within the padding."""
    want = np.zeros(res, dtype=np.int32)
    c = (np.arange(res[0]) + 0.5) * dx
    cols = [(c >= lo[k]) & (c <= hi[k]) for k in range(2)]
    cols = [m & (np.arange(res[0]) >= PAD) & (np.arange(res[0]) < res[0] - PAD) for m in cols]
    z0 = max(PAD, int(lo[2] / dx + 0.5))
    z1 = min(res[1] - PAD, int(hi[2] / dx + 0.5))
    want[np.ix_(cols[0], cols[1], np.arange(z0, z1))] = 1
    return want


@pytest.mark.parametrize("lo,hi", [((0.13, 0.21, 0.17), (0.61, 0.44, 0.72)),
                                   ((0.0013, 0.3, 0.011), (0.99, 0.71, 0.998))])
def test_box_voxels_known_answer(lo, hi):
    res, dx = (64, 64, 64), 1 / 64
    got = O.voxelize(box_mesh(lo, hi), res, dx, PAD)
    assert np.array_equal(got, _box_voxels(lo, hi, res, dx))


def test_overlapping_boxes_add_and_reversed_mesh_subtracts():
    res, dx = (32, 32, 32), 1 / 32
    a, b = box_mesh((0.2, 0.2, 0.2), (0.6, 0.6, 0.6)), box_mesh((0.4, 0.3, 0.35), (0.8, 0.7, 0.7))
    both = O.voxelize(np.concatenate([a, b]), res, dx, PAD)
    assert np.array_equal(both, O.voxelize(a, res, dx, PAD) + O.voxelize(b, res, dx, PAD))
    assert both.max() == 2
    inv = a[:, [0, 1, 2, 6, 7, 8, 3, 4, 5]]  # b and c swapped: normals inward
    assert np.array_equal(O.voxelize(inv, res, dx, PAD), -O.voxelize(a, res, dx, PAD))


def test_sphere_volume():
    res, dx = (64, 64, 64), 1 / 64
    r = 0.3
    v = O.voxelize(sphere_mesh((0.5, 0.5, 0.5), r, 24, 32), res, dx, PAD)
    assert set(np.unique(v)) <= {0, 1}
    vol = v.sum() * dx ** 3
    assert vol == pytest.approx(4 / 3 * np.pi * r ** 3, rel=0.03)


def test_empty_and_flat_meshes():
    res = (16, 16, 16)
    assert not O.voxelize(np.zeros((0, 9)), res, 1 / 16).any()
    flat = np.array([[0.1, 0.1, 0.5, 0.9, 0.1, 0.5, 0.1, 0.9, 0.5],   # normal along z: counted
                     [0.1, 0.5, 0.1, 0.9, 0.5, 0.1, 0.1, 0.5, 0.9]])  # vertical: skipped
    v = O.voxelize(flat, res, 1 / 16)
    assert v.min() == 0 and v.max() == 1


def _solver(dim=3, n=4000):
    cfg, _ = (scenes.falling_block_3d if dim == 3 else scenes.dam_break_2d)(n=n, n_grid=32)
    return MPMSolver(cfg)


def test_add_ball_points_lie_in_the_ball():
    s = _solver()
    s.initialize()
    assert s.add_ball((0.5, 0.5, 0.5), 0.1, 500) == 500
    x = s._staging()[:500, :3]
    assert np.all(np.linalg.norm(x - 0.5, axis=1) <= 0.1 + 1e-12)
    assert s.current_idx == 500
    # the reference adds nothing unless current_idx + num < n_particles
    assert s.add_ball((0.5, 0.5, 0.5), 0.1, s.n_particles - 500) == 0 and s.current_idx == 500


def test_emit_water_disc_and_velocity():
    s = _solver()
    s.initialize()
    s.emit_water((0.5, 0.6, 0.4), 0.05, (0.0, -3.0, 1.0), 300)
    h = s._staging()[:300]
    x, v = h[:, 0:3], h[:, 3:6]
    assert np.all(np.hypot(x[:, 0] - 0.5, x[:, 1] - 0.6) <= 0.05 + 1e-12)
    assert np.all(x[:, 2] == 0.4) and np.all(v == [0.0, -3.0, 1.0])
    F = h[:, 15:24]
    assert np.all(F == np.eye(3).ravel())


def test_letters_emitter_appends_the_emit_data():
    s = _solver()
    s.initialize()
    data = np.random.default_rng(0).random((50, 3))
    s.set_emit_data(data)
    s.emit_letters_one_frame()
    s.emit_letters_one_frame()
    h = s._staging()
    assert s.current_idx == 100
    assert np.array_equal(h[50:100, 0:3], data) and np.all(h[:100, 3:6] == [0.0, -2.0, 0.0])


def test_emitters_refuse_overflow():
    s = _solver(n=100)
    s.initialize()
    with pytest.raises(ValueError):
        s.add_cube((0.1, 0.1, 0.1), (0.1, 0.1, 0.1), 101)


@pytest.mark.parametrize("theta", [0.0, np.pi / 2])
def test_add_cube_pushes_particles_out_of_the_rotated_collider(theta):
    """fill_in_box with the collider (mpm_solver.py:1582-1588) on the host:
    a bar along x (cells y 8..11, z 28..35) rotated by theta about
    (32, ., 32); particles whose cell the rotated bar covers move up by 2..5
    cells along the stored normal, the others stay."""
    import torch

    cfg, _ = scenes.falling_block_3d(n=20000, n_grid=32)
    cfg.grid_res, cfg.ub = [64, 32, 64], [61, 29, 61]
    s = MPMSolver(cfg)
    s.initialize()
    sdf = np.full((64, 32, 64), 0.02, dtype=np.float32)
    sdf[:, 8:12, 28:36] = -0.01
    normal = np.zeros((64, 32, 64, 3), dtype=np.float32)
    normal[..., 1] = 1.0
    # the collider's volumes as host tensors: add_cube reads them on the host
    s._col = {"sdf": torch.from_numpy(sdf), "normal": torch.from_numpy(normal), "offset": [0, 0, 0],
              "theta": theta, "height": 0.0, "omega": 5.0, "rate": 0.1}
    s.add_cube((0.3, 0.2, 0.3), (1.4, 0.3, 1.4), 20000)
    free = MPMSolver(cfg)
    free.initialize()
    free.add_cube((0.3, 0.2, 0.3), (1.4, 0.3, 1.4), 20000)
    x, x0 = s._staging()[:20000, :3], free._staging()[:20000, :3]
    cell = (x0 / s.dx + 0.5).astype(int)
    across = cell[:, 2] if theta == 0.0 else cell[:, 0]  # the bar's cross-section axis
    inside = (cell[:, 1] >= 8) & (cell[:, 1] < 12) & (across >= 28) & (across < 36)
    moved = np.any(x != x0, axis=1)
    assert inside.any() and np.array_equal(moved, inside)
    dy = (x[moved, 1] - x0[moved, 1]) / s.dx
    assert np.all((dy >= 2) & (dy <= 5)) and np.all(x[moved][:, [0, 2]] == x0[moved][:, [0, 2]])


def _letters():
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "letters_voxels.npz"))
    res = tuple(int(r) for r in g["res"])
    mask = np.unpackbits(g["mask_bits"])[: np.prod(res)].reshape(res).astype(bool)
    return g, mask


def test_voxelizer_reproduces_the_reference_letters():
    """The reference's own emitted letters (mpm_exps/inputs/
    letters_emit_one_frame.npy: 63,856 particles from auto_quant.ply at a
    128^3 grid, 2 per inside voxel) occupy exactly the voxels the oracle's
    voxelizer finds inside the mesh (tests/golden/make_letters_golden.py)."""
    g, mask = _letters()
    v = O.voxelize(g["triangles"].astype(np.float64), mask.shape, 1 / 256, 3, 1e-8)
    assert set(np.unique(v)) <= {0, 1}
    assert int(mask.sum()) == 31928 and np.array_equal(v > 0, mask)
    assert int(g["n_particles"]) == 2 * int(mask.sum()) and g["per_voxel"].tolist() == [2]


def test_voxelizer_geometry():
    """voxelizer.py:17-40: every axis rounded up to a power of two, times
    the super-sampling; spacing dx / super_sample; jitter by precision."""
    from autoquantizer_b200.voxelizer import Voxelizer

    v = Voxelizer(res=(48, 100, 128), dx=1 / 48, super_sample=2)
    assert v.res == (128, 256, 256) and v.dx == 1 / 96 and v.inv_dx == 96 and v.padding == 3
    assert v.jitter_scale == 1e-8 and Voxelizer((8, 8, 8), 0.1, 1, precision="f32").jitter_scale == 1e-4
    with pytest.raises(ValueError):
        Voxelizer((8, 8), 0.1)
    with pytest.raises(ValueError):
        Voxelizer((8, 8, 8), 0.1, precision="f16")
