"""Emitters and on-disk formats on the GPU: the CUDA voxelizer
(aq_voxelize) bit-exact against the oracle's restatement, add_mesh
seeding, the collider push-out of add_cube, the grid mass, and the
dump / checkpoint / load round trip."""
import os

import numpy as np
import pytest

import oracle as O
from autoquantizer_b200 import scenes
from autoquantizer_b200.mpm_solver import MPMSolver
from autoquantizer_b200.voxelizer import Voxelizer
from helpers import box_mesh, sphere_mesh, quant_steps

pytestmark = pytest.mark.gpu


def _soup(n, seed=0):
    """Random triangles, many of them large and overlapping."""
    rng = np.random.default_rng(seed)
    c = rng.random((n, 1, 3)) * 0.8 + 0.1
    return (c + (rng.random((n, 3, 3)) - 0.5) * rng.random((n, 1, 1)) * 0.6).reshape(n, 9)


@pytest.mark.parametrize("mesh", ["box", "sphere", "soup", "empty"])
def test_voxelizer_matches_oracle(mesh):
    tris = {"box": lambda: box_mesh((0.13, 0.21, 0.17), (0.61, 0.44, 0.72)),
            "sphere": lambda: sphere_mesh((0.45, 0.5, 0.55), 0.3, 20, 28),
            "soup": lambda: _soup(3000),
            "empty": lambda: np.zeros((0, 9))}[mesh]()
    vox = Voxelizer(res=(48, 48, 48), dx=1 / 48, super_sample=2)
    assert vox.res == (128, 128, 128) and vox.dx == 1 / 96
    got = vox.voxelize(tris).cpu().numpy()
    want = O.voxelize(tris, vox.res, vox.dx, vox.padding, vox.jitter_scale)
    assert np.array_equal(got, want)
    if mesh == "box":
        assert got.sum() > 0 and got.max() == 1


def _solver(n=200000, n_grid=32):
    cfg, _ = scenes.falling_block_3d(n=n, n_grid=n_grid)
    s = MPMSolver(cfg)
    s.initialize()
    return s


def test_add_mesh_seeds_every_inside_voxel():
    s = _solver()
    tris = box_mesh((0.1, 0.12, 0.14), (0.2, 0.25, 0.22))
    cnt = s.cnt_mesh_particles_num(tris, sample_density=3)
    n = s.add_mesh(tris, sample_density=3, velocity=(0.0, -4.0, 0.0), translation=(0.3, 0.2, 0.1))
    assert n == cnt == s.current_idx > 0
    vox = s.voxelizer.voxels.cpu().numpy()
    h = s._staging()[:n]
    idx = np.floor((h[:, :3] - [0.3, 0.2, 0.1]) / s.dx + 1e-9).astype(int)
    assert np.all(vox[idx[:, 0], idx[:, 1], idx[:, 2]] > 0)
    # every inside voxel got sample_density + 1 particles
    _, per = np.unique(idx, axis=0, return_counts=True)
    assert len(per) == int((vox > 0).sum()) and np.all(per == 4)
    assert np.all(h[:, 3:6] == [0.0, -4.0, 0.0])
    s.substeps(4)
    assert s.status()[0] == 0


def test_add_cube_moves_particles_out_of_the_collider():
    from test_gpu_collider import bar_sdf

    cfg, _ = scenes.falling_block_3d(n=20000, n_grid=32)
    cfg.grid_res = [64, 32, 64]
    cfg.ub = [61, 29, 61]
    s = MPMSolver(cfg)
    s.initialize()
    sdf, normal = bar_sdf()
    s.init_sdf_value(sdf, normal, theta=0.0)
    s.add_cube((0.3, 0.2, 0.9), (1.4, 0.3, 0.2), 20000)
    x = s._staging()[:20000, :3]
    free = MPMSolver(cfg)
    free.initialize()
    free.add_cube((0.3, 0.2, 0.9), (1.4, 0.3, 0.2), 20000)
    x0 = free._staging()[:20000, :3]
    moved = np.any(x != x0, axis=1)
    # the bar occupies y cells 8..11 over z cells 28..35: particles whose
    # cell int(x / dx + 0.5) is there moved up by 2..5 cells
    cell = (x0 / s.dx + 0.5).astype(int)
    inside = (cell[:, 1] >= 8) & (cell[:, 1] < 12) & (cell[:, 2] >= 28) & (cell[:, 2] < 36)
    assert inside.any() and np.array_equal(moved, inside)
    dy = (x[moved, 1] - x0[moved, 1]) / s.dx
    assert np.all((dy >= 2) & (dy <= 5)) and np.all(x[moved][:, [0, 2]] == x0[moved][:, [0, 2]])


def test_grid_mass_conserves_particle_mass():
    s = _solver(n=20000)
    s.add_cube((0.3, 0.3, 0.3), (0.3, 0.3, 0.3), 20000)
    assert float(s.grid_mass().abs().sum()) == 0.0  # before the first substep
    s.substeps(3)
    m = s.grid_mass()
    assert tuple(m.shape) == (32, 32, 32)
    assert float(m.double().sum()) == pytest.approx(20000 * s.p_mass, rel=1e-5)


def test_dump_checkpoint_load_round_trip(tmp_path):
    s = _solver(n=20000)
    s.param.pos_output_folder = str(tmp_path)
    s.add_cube((0.3, 0.3, 0.3), (0.3, 0.3, 0.3), 20000)
    s.substeps(10)
    fn = s.dump_states(7)
    assert os.path.basename(fn) == "data_000007.ply"
    s.checkpoint_states(7)
    assert sorted(os.listdir(tmp_path)) == ["C.npy", "F.npy", "data_000007.ply", "v.npy"]
    g = s.dump_grid(7)
    assert np.load(g)["m"].dtype == np.float16
    before = s.state_values()
    t = _solver(n=20000)
    t.load_states(str(tmp_path), 7)
    assert t.current_idx == 20000
    after = t.state_values()
    # float32 files, re-encoded: within one quantization step (plus f32 rounding)
    tol = np.maximum(np.nan_to_num(quant_steps(s)), 1e-6 * np.abs(before).max(0))
    assert np.all(np.abs(after - before) <= tol[None, :] + 1e-7)


def test_run_forward_only_dumps_every_frame(tmp_path):
    s = _solver(n=5000)
    s.param.pos_output_folder = str(tmp_path)
    s.n_timestep, s.param.steps = 11, 4
    s.add_cube((0.3, 0.3, 0.3), (0.2, 0.2, 0.2), 5000)
    s.run_forward_only(save_states=True)
    assert sorted(os.listdir(tmp_path)) == ["data_000000.ply", "data_000001.ply", "data_000002.ply"]
    assert s.launches() > 0


def test_reference_letters_on_the_gpu():
    """The CUDA voxelizer and add_mesh on the reference's letters mesh
    reproduce the voxels of the reference's shipped emission
    (tests/golden/letters_voxels.npz, made by make_letters_golden.py)."""
    from test_emitters import _letters

    g, mask = _letters()
    tri = g["triangles"]
    vox = Voxelizer(res=(128, 128, 128), dx=1 / 128, super_sample=2)
    assert vox.res == mask.shape
    assert np.array_equal(vox.voxelize(tri).cpu().numpy() > 0, mask)
    cfg, _ = scenes.falling_block_3d(n=64000, n_grid=128)
    s = MPMSolver(cfg)
    s.initialize()
    t = [float(x) for x in g["translation"]]
    n = s.add_mesh(tri, sample_density=1, velocity=(0.0, -2.0, 0.0), translation=t)
    assert n == int(g["n_particles"]) == 63856
    idx = np.floor((s._staging()[:n, :3] - t) * 128 + 1e-9).astype(int)
    got = np.zeros_like(mask)
    got[idx[:, 0], idx[:, 1], idx[:, 2]] = True
    assert np.array_equal(got, mask)


def test_emission_into_a_running_simulator_leaves_stored_records_alone():
    """Particles emitted while a simulator runs are encoded on the device
    behind the stored records (aq_sim_append), as the reference's emitters
    write only the new particles' fields: the stored records keep their
    bits (re-encoding them, with dithering on, could move codes), the
    simulator is not rebuilt, and the new particles hold the emitted values
    to within a quantization step."""
    cfg, vals = scenes.dam_break_2d(n=8192, n_grid=128)
    cfg.n_particles = 12000
    s = MPMSolver(cfg)
    s.set_particles(vals)
    s.substeps(5)
    sim = s._sim.value
    before = s.words()
    assert s.emit_water([0.5, 0.5], 0.04, [0.0, -1.0], 1000) == 1000
    s.add_cube((0.6, 0.6), (0.1, 0.1), 1500)  # 2D: a 38 x 38 lattice
    m = s.current_idx - 8192 - 1000
    assert m == 38 * 38
    assert s._sim.value == sim
    after = s.words()
    assert after.shape == (8192 + 1000 + m, before.shape[1])
    assert np.array_equal(after[:8192], before)
    new = s.state_values()[8192:]
    q = np.nan_to_num(quant_steps(s))
    assert np.all(np.abs(new[:1000, 2:4] - [0.0, -1.0]) <= q[2:4] * 2 + 1e-6 * 2 ** 12)
    d = np.hypot(new[:1000, 0] - 0.5, new[:1000, 1] - 0.5)
    assert np.all(d <= 0.04 + q[0])
    assert np.all((new[1000:, 0] >= 0.6 - q[0]) & (new[1000:, 0] <= 0.7 + q[0]))
    s.substeps(5)
    assert s.status()[0] == 0


def test_appended_particles_run_like_particles_set_at_once():
    """A run whose second half of particles was appended to the running
    simulator matches, over 4 substeps, a run that set all of them at once
    (f64 compute, FP32-state layout: the only difference is the order of the
    grid sums)."""
    cfg, vals = scenes.mixed_boxes_3d(n=20000, n_grid=32, quantized=False, precision="f64")
    a = MPMSolver(cfg)
    a.set_particles(vals)
    a.substeps(4)
    b = MPMSolver(cfg)
    b.set_particles(vals[:12000])
    b.substeps(0)  # starts the simulator
    sim = b._sim.value
    b._append(vals[12000:, :3], v=vals[12000:, 3:6], material=vals[12000:, -1])
    b.substeps(4)
    assert b._sim.value == sim
    x, y = a.state_values(), b.state_values()
    assert x.shape == y.shape == (20000, 25)
    np.testing.assert_allclose(y, x, rtol=0, atol=1e-9 * max(1.0, np.abs(x).max()))
