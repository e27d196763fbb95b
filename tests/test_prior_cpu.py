"""Prior-depth and propagate-depth paths of the CPU oracle (no GPU).

The propagate-depth initial maps (InitWorkspace, patch_match_cuda.cu:603-659)
are checked against the scene's analytic depth and normals: the sources'
exact depth maps projected into the reference view must land within 1 % of
the reference's own depth almost everywhere, and the fitted normals within
10 degrees. The full runs check that a prior (has_prior_depth) or the
propagated start (propagate_depth) does not lose accuracy against the plain
photometric pass on the same scene, and the option rules of both modes.
"""
import numpy as np
import pytest

import oracle.oracle as orc
from sensemap_b200 import synthetic as syn
from tests.helpers import perturbed_gt, photometric_options, problem_from_scene, small_planes


def _propagate_problem(sc, drop=()):
    ref = sc.ref_index
    H, W = sc.views[ref].depth_gt.shape
    depths = [None if i in drop else v.depth_gt for i, v in enumerate(sc.views)]
    zero = (np.zeros((H, W), np.float32), np.zeros((3, H, W), np.float32))
    return problem_from_scene(sc, depth_maps=depths, init=zero)


def test_propagate_init_lands_on_the_analytic_depth():
    sc = small_planes(seed=31)
    out = orc.propagate_init(_propagate_problem(sc))
    ref = sc.views[sc.ref_index]
    d, prior = out["depth"], out["prior"]
    filled = d > 0
    assert filled.mean() > 0.95
    assert np.mean(np.abs(d[filled] - ref.depth_gt[filled]) <= 0.01 * ref.depth_gt[filled]) > 0.9
    # A prior is set only where more than two projections agree within 1 %;
    # it is one of the projected depths, so it equals the initial depth there.
    has_prior = prior > 0
    assert has_prior.mean() > 0.5
    assert np.array_equal(prior[has_prior], d[has_prior])
    fitted = np.linalg.norm(out["normal"], axis=0) > 0.5
    assert fitted.mean() > 0.9
    assert syn.normal_accuracy(out["normal"], ref.normal_gt, 10.0, mask=fitted) > 0.95


def test_propagate_init_keeps_given_depths_and_skips_sources_without_maps():
    sc = small_planes(seed=32)
    prob = _propagate_problem(sc)
    ref = prob.images[prob.ref_image_idx]
    given = np.zeros_like(ref.depth)
    given[:, : given.shape[1] // 2] = 7.5  # the left half has a depth already
    ref.depth = given
    out = orc.propagate_init(prob)
    left = np.s_[:, : given.shape[1] // 2]
    assert np.all(out["depth"][left] == 7.5) and np.all(out["prior"][left] == 0)
    # With only two sources carrying a map no pixel gets more than two
    # projections: depths are filled, but no prior is set.
    sc2 = small_planes(seed=32)
    keep = [i for i in range(len(sc2.views)) if i != sc2.ref_index][:2]
    drop = [i for i in range(len(sc2.views)) if i not in keep]
    out2 = orc.propagate_init(_propagate_problem(sc2, drop=drop))
    assert (out2["depth"] > 0).mean() > 0.5
    assert not np.any(out2["prior"] > 0)


def test_prior_and_propagate_runs_keep_accuracy():
    sc = small_planes(seed=31)
    gt = sc.views[sc.ref_index].depth_gt
    plain = syn.depth_accuracy(orc.run(photometric_options(sc, iters=6), problem_from_scene(sc))["depth"], gt)
    prop = orc.run(photometric_options(sc, iters=6, init_depth_random=False, propagate_depth=True),
                   _propagate_problem(sc))
    prior = orc.run(photometric_options(sc, iters=6, has_prior_depth=True),
                    problem_from_scene(sc, init=perturbed_gt(sc, seed=3, rel=0.02)))
    assert syn.depth_accuracy(prop["depth"], gt) >= plain - 0.02
    assert syn.depth_accuracy(prior["depth"], gt) >= plain + 0.02


def test_prior_weights_change_the_run():
    sc = small_planes(seed=33)
    prob = problem_from_scene(sc, init=perturbed_gt(sc, seed=4, rel=0.02))
    opt = photometric_options(sc, iters=3, has_prior_depth=True)
    a = orc.run(opt, prob)["depth"]
    prob.prior_wgt = np.full(a.shape, 0.5, np.float32)
    b = orc.run(opt, prob)["depth"]
    assert not np.array_equal(a, b)


def test_prior_option_rules():
    sc = small_planes(seed=34)
    both = photometric_options(sc, iters=1, has_prior_depth=True, propagate_depth=True)
    with pytest.raises(RuntimeError):
        orc.run(both, problem_from_scene(sc, init=perturbed_gt(sc)))
    # propagate_depth starts from given maps and excludes the geometric pass.
    with pytest.raises(RuntimeError):
        orc.run(photometric_options(sc, iters=1, propagate_depth=True), _propagate_problem(sc))
    with pytest.raises(RuntimeError):
        orc.run(photometric_options(sc, iters=1, has_prior_depth=True), problem_from_scene(sc))
