"""Regenerate tests/golden/letters_voxels.npz from the AutoQuantizer
reference checkout (read-only), given as the one argument:

    python tests/golden/make_letters_golden.py <reference checkout>

The reference's 3D letters experiment emits particles from the mesh
mpm_exps/inputs/auto_quant.ply, loaded with load_mesh(..., scale=(0.1, 0.1,
2), offset=(0.02, 0.02, 0.5)) (run_mpm_elastic_3d.py:249), voxelized at
twice the resolution of a 128^3 grid (mpm_solver.py:115-116) and seeded
with sample_density + 1 = 2 particles per inside voxel at translation (1.5,
0.8, 0.1) (add_letters_ad, run_mpm_elastic_3d.py:65-75).  The reference
shipped the emitted positions of that set-up as
mpm_exps/inputs/letters_emit_one_frame.npy (63,856 particles).  The fixture
keeps the mesh's triangles (after load_mesh's scale and offset) and the
voxel indices those particles occupy, floor((x - translation) * 128), as a
bit mask; the tests voxelize the triangles and compare with the mask.
Nothing at test time reads the reference checkout.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from autoquantizer_b200.mesh_io import load_mesh  # noqa: E402

RES = 256
TRANSLATION = (1.5, 0.8, 0.1)


def main(ref):
    inputs = os.path.join(ref, "mpm_exps", "inputs")
    tri = load_mesh(os.path.join(inputs, "auto_quant.ply"), scale=(0.1, 0.1, 2), offset=(0.02, 0.02, 0.5))
    pos = np.load(os.path.join(inputs, "letters_emit_one_frame.npy")).astype(np.float64)
    idx = np.floor((pos - np.array(TRANSLATION)) * 128.0).astype(np.int64)
    assert idx.min() >= 0 and idx.max() < RES
    mask = np.zeros((RES, RES, RES), dtype=bool)
    mask[idx[:, 0], idx[:, 1], idx[:, 2]] = True
    per_voxel = np.unique(idx, axis=0, return_counts=True)[1]
    out = os.path.join(HERE, "letters_voxels.npz")
    np.savez_compressed(out, triangles=tri.astype(np.float32), mask_bits=np.packbits(mask.ravel()),
                        res=np.array([RES] * 3), translation=np.array(TRANSLATION),
                        n_particles=np.array(len(pos)), per_voxel=np.array(sorted(set(per_voxel.tolist()))))
    print(out, "triangles", tri.shape, "voxels", int(mask.sum()), "particles", len(pos))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path of the AutoQuantizer reference checkout>" % sys.argv[0])
    main(sys.argv[1])
