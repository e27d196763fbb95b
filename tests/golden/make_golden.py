"""Generate the golden fixtures from the REFERENCE's own kernels.

Run on a GPU box with oracle/_ref/libref_pm.so built (oracle/ref_build.py):

    python tests/golden/make_golden.py [out_dir]

Each fixture is self-contained (images, cameras, hypotheses, options, and the
reference's outputs), so tests replay it on the CPU oracle without rendering:
  ref_initconf_planes.npz  InitConfMapKernel costs/conf/view_sel for given
                           (perturbed ground-truth) hypotheses, 96x72, N=4
  ref_filter_planes.npz    FilterDepthMapsKernel decisions on perturbed maps
  ref_run_planes.npz       a full photometric run (6 iterations) of the
                           reference (cuRAND draws; compared statistically)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle.oracle as orc  # noqa: E402
import oracle.ref_oracle as ref  # noqa: E402
from sensemap_b200 import synthetic as syn  # noqa: E402
from tests.helpers import perturbed_gt, photometric_options, problem_from_scene  # noqa: E402


def pack_scene(scene, prob, opt, poses):
    d = {"ref_index": prob.ref_image_idx, "src_indices": np.array(prob.src_image_idxs),
         "images": np.stack([v.image.astype(np.uint8) for v in scene.views]),
         "K": np.stack([v.K for v in scene.views]), "R": np.stack([v.R for v in scene.views]),
         "T": np.stack([v.T for v in scene.views]), "poses": poses,
         "depth_gt": scene.views[prob.ref_image_idx].depth_gt,
         "opt": np.array([repr(vars(opt))])}
    return d


def main(out_dir: Path):
    out_dir.mkdir(parents=True, exist_ok=True)
    scene = syn.planes_scene(seed=11, width=96, height=72, focal=75.0, num_src=4)
    base_opt = photometric_options(scene, iters=0, init_depth_random=False)
    # Case A: InitConfMapKernel on given hypotheses.
    init = perturbed_gt(scene, seed=4)
    prob = problem_from_scene(scene, init=init)
    poses = orc.run(base_opt, prob)["poses"]
    r = ref.run(base_opt, prob, poses)
    np.savez_compressed(out_dir / "ref_initconf_planes.npz", **pack_scene(scene, prob, base_opt, poses),
                        init_depth=init[0], init_normal=init[1], cost=r["cost"], conf=r["conf"],
                        view_sel=r["view_sel"], depth=r["depth"])
    # Case B: FilterDepthMapsKernel on perturbed ground-truth maps of every view.
    rng = np.random.default_rng(5)
    maps = []
    for v in scene.views:
        d = v.depth_gt * (1 + rng.normal(0, 0.01, v.depth_gt.shape)).astype(np.float32)
        d[rng.random(d.shape) < 0.1] = 0
        maps.append(d.astype(np.float32))
    fprob = problem_from_scene(scene, depth_maps=maps)
    fopt = photometric_options(scene, filter_min_num_consistent=2)
    fr = ref.run_filter(fopt, fprob, poses)
    np.savez_compressed(out_dir / "ref_filter_planes.npz", **pack_scene(scene, fprob, fopt, poses),
                        depth_maps=np.stack(maps), filtered=fr,
                        filter_min_num_consistent=2, filter_max_cost=fopt.filter_geom_consistency_max_cost,
                        geom_max=fopt.geom_consistency_max_cost)
    # Case C: a full photometric run.
    scene_c = syn.planes_scene(seed=12, width=160, height=120, focal=125.0, num_src=4)
    copt = photometric_options(scene_c, iters=6)
    cprob = problem_from_scene(scene_c)
    cposes = orc.run(photometric_options(scene_c, iters=0), cprob)["poses"]
    rc = ref.run(copt, cprob, cposes)
    np.savez_compressed(out_dir / "ref_run_planes.npz", **pack_scene(scene_c, cprob, copt, cposes),
                        depth=rc["depth"], normal=rc["normal"].astype(np.float16),
                        gt_accuracy=syn.depth_accuracy(rc["depth"], scene_c.views[cprob.ref_image_idx].depth_gt))
    print("written to", out_dir)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
