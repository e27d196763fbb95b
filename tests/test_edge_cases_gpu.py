"""Edge cases through the C ABI, each against the CPU oracle: images smaller
than the window, a single source view, the 32-view maximum, sources of other
sizes than the reference, scaled source intrinsics, and masks."""
import numpy as np
import pytest

import oracle.oracle as orc
from sensemap_b200 import synthetic as syn
from sensemap_b200 import _native as N
from sensemap_b200.patch_match import PatchMatchACMMCuda, Problem, View
from tests.helpers import frac_close, perturbed_gt, photometric_options, problem_from_scene

pytestmark = pytest.mark.gpu


def engine(opt, prob):
    with PatchMatchACMMCuda(opt, prob) as pm:
        pm.Run()
        return {"depth": pm.GetDepthMap(), "cost": pm.GetCostMap(), "view_sel": pm.GetViewSelMap(),
                "conf": pm.GetConfMap()}


def costs_close(a, b):
    err = np.abs(a - b)
    return np.median(err) < 2e-3 and np.quantile(err, 0.99) < 5e-2


def test_image_smaller_than_window():
    sc = syn.planes_scene(seed=51, width=7, height=5, focal=6.0, num_src=2)
    init = perturbed_gt(sc, seed=1)
    prob = problem_from_scene(sc, init=init)
    opt = photometric_options(sc, iters=0, init_depth_random=False)
    g, o = engine(opt, prob), orc.run(opt, prob)
    assert costs_close(g["cost"], o["cost"])
    opt = photometric_options(sc, iters=3)
    g, o = engine(opt, prob), orc.run(opt, prob)
    assert np.isfinite(g["depth"]).all()


def test_single_source_view():
    sc = syn.planes_scene(seed=52, width=96, height=72, focal=75.0, num_src=1)
    prob = problem_from_scene(sc)
    opt = photometric_options(sc, iters=4)
    g, o = engine(opt, prob), orc.run(opt, prob)
    assert frac_close(g["depth"], o["depth"], 0.01) > 0.85
    assert set(np.unique(g["view_sel"])) <= {0, 1}


def test_thirty_two_source_views():
    sc = syn.heightfield_scene(seed=53, width=64, height=48, focal=50.0, num_src=32, ring_radius=0.6)
    init = perturbed_gt(sc, seed=2, ref=0)
    prob = problem_from_scene(sc, init=init)
    opt = photometric_options(sc, iters=0, init_depth_random=False)
    g, o = engine(opt, prob), orc.run(opt, prob)
    assert g["cost"].shape[0] == 32
    assert costs_close(g["cost"], o["cost"])
    assert np.mean(g["view_sel"] == o["view_sel"]) > 0.98
    opt = photometric_options(sc, iters=2)
    g, o = engine(opt, prob), orc.run(opt, prob)
    assert frac_close(g["depth"], o["depth"], 0.01) > 0.9


def test_more_than_thirty_two_sources_rejected():
    sc = syn.planes_scene(seed=54, width=32, height=24, focal=25.0, num_src=1)
    v = [View(x.image, x.K, x.R, x.T) for x in sc.views]
    prob = Problem(0, [1] * 33, v)
    with pytest.raises(N.SmvsError) as ei:
        PatchMatchACMMCuda(photometric_options(sc), prob)
    assert ei.value.status == N.SMVS_EINVAL


def test_sources_of_other_sizes_and_scaled_intrinsics():
    sc = syn.planes_scene(seed=55, width=128, height=96, focal=100.0, num_src=4)
    # Source 1 at half resolution: its image resampled by the caller, its K scaled by the engine.
    views = [View(v.image, v.K, v.R, v.T) for v in sc.views]
    src = 1 if sc.ref_index != 1 else 0
    half = sc.views[src].image.reshape(48, 2, 64, 2).mean(axis=(1, 3)).round().astype(np.float32)
    views[src] = View(half, sc.views[src].K, sc.views[src].R, sc.views[src].T)
    srcs = [i for i in range(len(views)) if i != sc.ref_index]
    scales = [0.5 if i == src else 1.0 for i in srcs]
    init = perturbed_gt(sc, seed=3)
    views[sc.ref_index].depth, views[sc.ref_index].normal = init
    prob = Problem(sc.ref_index, srcs, views, src_image_scales=scales)
    opt = photometric_options(sc, iters=0, init_depth_random=False)
    g, o = engine(opt, prob), orc.run(opt, prob)
    assert costs_close(g["cost"], o["cost"])
    # The half-resolution view still sees the true surface: its costs at the GT hypothesis are low.
    k = srcs.index(src)
    assert np.median(g["cost"][k]) < 0.6


def test_mask_zeroes_depth():
    sc = syn.planes_scene(seed=56, width=96, height=72, focal=75.0, num_src=3)
    prob = problem_from_scene(sc)
    prob.mask = np.ones((72, 96), np.uint8)
    prob.mask[10:30, 20:50] = 0
    opt = photometric_options(sc, iters=2)
    g, o = engine(opt, prob), orc.run(opt, prob)
    assert (g["depth"][10:30, 20:50] == 0).all()
    np.testing.assert_array_equal(g["depth"] == 0, o["depth"] == 0)
