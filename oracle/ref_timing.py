"""Time the REFERENCE's own PatchMatch kernels on a B200 (test infrastructure).

Runs the first reference view of bench.py's workload — the seeded 11-view
1600x1200 heightfield scene, 10 source views, window radius 5 step 1, 6
iterations — through oracle/_ref/libref_pm.so: the reference's
kernel_functions.cu launched in PatchMatchACMMCuda::Run's order
(patch_match_cuda.cu:748-1057) with its launch shapes, its 8-bit layered
source texture and a device sync after every launch. One photometric pass
(random initialisation) and one geometric pass (initialised from, and checked
against, noisy ground-truth maps) are timed; a depth map is one of each.
Prints one JSON line. Needs a GPU and the built reference library.

    python oracle/ref_timing.py [--repeats 2]
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from oracle import ref_oracle as R  # noqa: E402
from sensemap_b200 import synthetic as syn  # noqa: E402
from sensemap_b200.patch_match import PatchMatchOptions, Problem, View  # noqa: E402


def options(scene, geometric):
    return PatchMatchOptions(depth_min=scene.depth_min, depth_max=scene.depth_max, window_radius=5, window_step=1,
                             sigma_spatial=5, num_iterations=6, geom_consistency=geometric,
                             init_depth_random=not geometric, geom_consistency_regularizer=0.1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--width", type=int, default=1600)
    ap.add_argument("--height", type=int, default=1200)
    ap.add_argument("--views", type=int, default=11)
    args = ap.parse_args()
    import torch
    scene = syn.heightfield_scene(seed=0, width=args.width, height=args.height, num_src=args.views - 1,
                                  device="cuda")
    maps = syn.noisy_maps(scene, seed=100)
    V = len(scene.views)
    fviews = [O.FilterView(v.K, v.R, v.T, d, n) for v, (d, n) in zip(scene.views, maps)]
    _, _, poses = O.cross_filter_poses(fviews, (0, list(range(1, V))))  # 43-float records, scale 1
    photo = Problem(0, list(range(1, V)), [View(v.image, v.K, v.R, v.T) for v in scene.views])
    geo = Problem(0, list(range(1, V)), [View(v.image, v.K, v.R, v.T, depth=d, normal=n)
                                         for v, (d, n) in zip(scene.views, maps)])
    out = {}
    for name, prob, opt in (("photometric", photo, options(scene, False)), ("geometric", geo, options(scene, True))):
        R.run(opt, prob, poses)  # warm-up (module load, first allocations)
        torch.cuda.synchronize()
        times = []
        for _ in range(args.repeats):
            t = time.perf_counter()
            res = R.run(opt, prob, poses)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t)
        out[name] = {"seconds": min(times), "all": times,
                     "within_1pct_gt": syn.depth_accuracy(res["depth"], scene.views[0].depth_gt)}
    per_map = out["photometric"]["seconds"] + out["geometric"]["seconds"]
    print(json.dumps({"reference_gpu": {
        "what": "reference kernels (kernel_functions.cu, --use_fast_math) on this GPU, launch order and syncs of "
                "PatchMatchACMMCuda::Run, 8-bit layered source texture",
        "workload": f"view 0 of the {V}-view {args.width}x{args.height} heightfield scene, N={V - 1}, R=5, S=1, "
                    f"6 iterations",
        "passes": out, "seconds_per_depth_map": per_map, "depth_maps_per_s": 1.0 / per_map}}), flush=True)


if __name__ == "__main__":
    main()
