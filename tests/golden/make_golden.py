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
  ref_crossfilter_planes.npz  CrossFilterKernel refined maps and
                           DeduplicFilterKernel visibility/delta maps of a
                           6-view set (CrossFilterCuda::Run + DedupRun)

    python tests/golden/make_golden.py [out_dir] --only crossfilter
regenerates the last fixture alone.
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


def cross_filter_case(out_dir: Path):
    from sensemap_b200.patch_match import PatchMatchOptions
    from tests.helpers import filter_set
    scene, views, problems = filter_set(seed=21, w=96, h=72, f=75.0, n_views=6,
                                        ref_flags=[True, True, True, True, True, False])
    problems = [(r, s) for r, s in problems if r != 5]  # view 5 is a source only
    opt = PatchMatchOptions(filter_min_num_consistent=2)
    refined = ref.cross_filter(opt, views, problems)
    vis, delta = ref.dedup(opt, views, problems, refined)
    refs = sorted(refined)
    src = np.full((len(problems), max(len(s) for _, s in problems)), -1, np.int32)
    for k, (_, s_) in enumerate(problems):
        src[k, :len(s_)] = s_
    np.savez_compressed(out_dir / "ref_crossfilter_planes.npz",
                        K=np.stack([v.K for v in views]), R=np.stack([v.R for v in views]),
                        T=np.stack([v.T for v in views]), depth=np.stack([v.depth for v in views]),
                        normal=np.stack([v.normal for v in views]),
                        ref_flag=np.array([v.ref_flag for v in views]),
                        problem_ref=np.array([r for r, _ in problems], np.int32), problem_src=src,
                        filter_min_num_consistent=opt.filter_min_num_consistent,
                        refined_views=np.array(refs, np.int32), refined=np.stack([refined[r] for r in refs]),
                        vis=np.stack(vis), delta=np.stack([delta[r] for r in refs]))


def main(out_dir: Path, only: str = ""):
    out_dir.mkdir(parents=True, exist_ok=True)
    if only == "crossfilter":
        cross_filter_case(out_dir)
        print("written to", out_dir)
        return
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
    cross_filter_case(out_dir)
    print("written to", out_dir)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else ""
    args = [a for a in args if a != only]
    main(Path(args[0]) if args else Path(__file__).resolve().parent, only)
