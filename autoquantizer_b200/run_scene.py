"""Run one of the seeded scenes for a number of substeps and print timing.

    python -m autoquantizer_b200.run_scene --scene mixed_boxes_3d --substeps 8 [--fp32] [--sparse] [--n N] [--grid G]
    python -m autoquantizer_b200.run_scene --device-gen --n 300000000 --grid 640 --substeps 50

A small fixed workload for profiler captures of single kernel launches.
"""
import argparse
import json
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="mixed_boxes_3d",
                    choices=["mixed_boxes_3d", "dam_break_2d", "elastic_block_2d", "falling_block_3d"])
    ap.add_argument("--substeps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--grid", type=int, default=None)
    ap.add_argument("--fp32", action="store_true", help="FP32 particle state instead of the quantized record")
    ap.add_argument("--sort-interval", type=int, default=None)
    ap.add_argument("--device-gen", action="store_true",
                    help="mixed_boxes_3d generated on the GPU (large particle counts)")
    ap.add_argument("--sparse", action="store_true", help="sparse grid (block table and node pools)")
    args = ap.parse_args()

    import torch

    from . import scenes
    from .mpm_solver import MPMSolver

    kw = {}
    if args.n:
        kw["n"] = args.n
    if args.grid:
        kw["n_grid"] = args.grid
    if args.fp32 and args.scene in ("mixed_boxes_3d", "dam_break_2d"):
        kw["quantized"] = False
    if args.device_gen:
        if args.scene != "mixed_boxes_3d" or args.fp32:
            ap.error("--device-gen builds the quantized mixed_boxes_3d scene only")
        cfg, vals = scenes.mixed_boxes_3d_device(n=kw.get("n", 2097152), n_grid=kw.get("n_grid", 128))
    else:
        cfg, vals = getattr(scenes, args.scene)(**kw)
    if args.sort_interval:
        cfg.sort_interval = args.sort_interval
    cfg.sparse_grid = bool(args.sparse)
    s = MPMSolver(cfg)
    s.set_particles(vals)
    s.substeps(args.warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.substeps(args.substeps)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    fl, fb = s.status()
    print(json.dumps({"scene": args.scene, "particles": int(cfg.n_particles), "substeps": args.substeps,
                      "ms_per_substep": 1e3 * dt / args.substeps,
                      "particle_substeps_per_s": cfg.n_particles * args.substeps / dt,
                      "bytes_per_particle": s.bytes_per_particle(),
                      "status": fl, "tile_fallbacks": fb,
                      "sparse_blocks": s.sparse_blocks() if args.sparse else None}))


if __name__ == "__main__":
    main()
