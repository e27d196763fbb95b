"""The CUDA engine against the REFERENCE's own kernels (oracle/_ref), run
side by side on the same GPU and inputs."""
import numpy as np
import pytest

import oracle.oracle as orc
import oracle.ref_oracle as ref
from sensemap_b200 import synthetic as syn
from sensemap_b200.patch_match import PatchMatchACMMCuda
from tests.helpers import frac_close, perturbed_gt, photometric_options, problem_from_scene, small_planes

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")]


def engine(opt, prob):
    with PatchMatchACMMCuda(opt, prob) as pm:
        pm.Run()
        return {"depth": pm.GetDepthMap(), "normal": pm.GetNormalMap(), "conf": pm.GetConfMap(),
                "cost": pm.GetCostMap(), "view_sel": pm.GetViewSelMap()}


@pytest.mark.parametrize("nsrc", [4, 10])
def test_costs_match_reference_kernels(nsrc):
    sc = small_planes(seed=21, n_src=nsrc)
    init = perturbed_gt(sc, seed=3)
    prob = problem_from_scene(sc, init=init)
    opt = photometric_options(sc, iters=0, init_depth_random=False)
    poses = orc.run(opt, prob)["poses"]
    r = ref.run(opt, prob, poses)
    g = engine(opt, prob)
    err = np.abs(g["cost"] - r["cost"])
    assert np.median(err) < 1e-4 and np.quantile(err, 0.999) < 1e-2
    assert np.mean(g["view_sel"] == r["view_sel"]) > 0.99


def test_full_run_matches_reference_statistically():
    sc = small_planes(seed=22)
    prob = problem_from_scene(sc)
    opt = photometric_options(sc, iters=6)
    poses = orc.run(photometric_options(sc, iters=0), prob)["poses"]
    r = ref.run(opt, prob, poses)
    g = engine(opt, prob)
    gt = sc.views[sc.ref_index].depth_gt
    acc_r, acc_g = syn.depth_accuracy(r["depth"], gt), syn.depth_accuracy(g["depth"], gt)
    assert abs(acc_g - acc_r) < 0.03, (acc_g, acc_r)
    assert frac_close(g["depth"], r["depth"], 0.01) > 0.8
    assert syn.normal_accuracy(g["normal"], r["normal"], 10.0) > 0.7


def test_geometric_pass_matches_reference_statistically():
    sc = small_planes(seed=23)
    n = len(sc.views)
    photo = [engine(photometric_options(sc, iters=4, random_seed=i), problem_from_scene(sc, ref=i)) for i in range(n)]
    prob = problem_from_scene(sc, depth_maps=[p["depth"] for p in photo], normal_maps=[p["normal"] for p in photo])
    opt = photometric_options(sc, iters=3, geom_consistency=True, init_depth_random=False,
                              geom_consistency_regularizer=0.1)
    poses = orc.run(photometric_options(sc, iters=0), problem_from_scene(sc))["poses"]
    r = ref.run(opt, prob, poses)
    g = engine(opt, prob)
    gt = sc.views[sc.ref_index].depth_gt
    assert abs(syn.depth_accuracy(g["depth"], gt) - syn.depth_accuracy(r["depth"], gt)) < 0.03
    assert frac_close(g["depth"], r["depth"], 0.01) > 0.85
