"""The coarse-to-fine pyramid: level sizes, the device image rescale and map
resampling bit for bit against the oracle's restatements, and a small
three-level run whose accuracy stays within 0.5 points of the single-level
pass at full resolution."""
import numpy as np
import pytest

import oracle.oracle as orc
from sensemap_b200 import STORE_F32
from sensemap_b200 import synthetic as syn
from sensemap_b200.patch_match import PatchMatchACMMCuda, PatchMatchOptions, Problem, View
from sensemap_b200.pyramid import PyramidPatchMatch, level_size, rescale_image, resample_maps

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,new", [((120, 160), (60, 80)), ((97, 131), (24, 33)), ((64, 64), (100, 90)),
                                       ((400, 600), (100, 150))])
def test_rescale_image_matches_oracle(shape, new):
    import torch
    rng = np.random.default_rng(3)
    img = np.round(rng.uniform(0, 255, shape)).astype(np.float32)
    out, _ = rescale_image(torch.from_numpy(img).cuda(), new[1], new[0])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), orc.rescale_image(img, *new))


@pytest.mark.parametrize("shape,new", [((30, 40), (60, 80)), ((61, 83), (122, 165)), ((50, 50), (25, 25))])
def test_resample_maps_match_oracle(shape, new):
    import torch
    rng = np.random.default_rng(4)
    d = rng.uniform(1, 10, shape).astype(np.float32)
    d[rng.random(shape) < 0.1] = 0
    n = rng.normal(0, 1, (3,) + shape).astype(np.float32)
    n /= np.linalg.norm(n, axis=0, keepdims=True)
    od, on = resample_maps(torch.from_numpy(d).cuda(), torch.from_numpy(n).cuda(), new[1], new[0])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(od.cpu().numpy(), orc.resample_maps(d[None], *new, False)[0])
    np.testing.assert_array_equal(on.cpu().numpy(), orc.resample_maps(n, *new, True))


def test_level_sizes():
    assert level_size(6000, 4000, 0)[:2] == (6000, 4000)
    assert level_size(6000, 4000, 1)[:2] == (3000, 2000)
    assert level_size(6000, 4000, 2)[:2] == (1500, 1000)
    # Never below 320 pixels on the longer side (patch_match_controller.cc:4407-4410).
    assert level_size(640, 480, 2)[:2] == (320, 240)
    assert level_size(200, 100, 3)[:2] == (200, 100)


def test_three_level_pyramid_keeps_accuracy():
    import torch
    sc = syn.heightfield_scene(seed=5, width=640, height=480, focal=480.0, num_src=6, device="cuda")
    V = len(sc.views)
    views = [View(torch.from_numpy(v.image).cuda(), v.K, v.R, v.T) for v in sc.views]
    opt = PatchMatchOptions(depth_min=sc.depth_min, depth_max=sc.depth_max, window_radius=5, window_step=1,
                            num_iterations=6, geom_consistency_regularizer=0.1, image_storage=STORE_F32)
    problems = [(r, [i for i in range(V) if i != r]) for r in range(V)]
    res = PyramidPatchMatch(opt, views, problems, levels=3, refine=[0]).Run()
    d = res.depth[0].cpu().numpy()
    assert d.shape == sc.views[0].depth_gt.shape
    acc_pyr = syn.depth_accuracy(d, sc.views[0].depth_gt)
    # Single level at full resolution: photometric, then geometric.
    from dataclasses import replace
    photo = []
    for r in range(V):
        with PatchMatchACMMCuda(replace(opt, geom_consistency=False, init_depth_random=True, random_seed=r),
                                Problem(r, problems[r][1], views)) as pm:
            pm.Run()
            photo.append((torch.from_numpy(pm.GetDepthMap()).cuda(), torch.from_numpy(pm.GetNormalMap()).cuda()))
    gv = [View(v.image, v.K, v.R, v.T, depth=photo[i][0], normal=photo[i][1]) for i, v in enumerate(views)]
    with PatchMatchACMMCuda(replace(opt, geom_consistency=True, init_depth_random=False, random_seed=1000),
                            Problem(0, problems[0][1], gv)) as pm:
        pm.Run()
        acc_one = syn.depth_accuracy(pm.GetDepthMap(), sc.views[0].depth_gt)
    print(f"pyramid {acc_pyr:.4f} single level {acc_one:.4f}; level seconds {res.level_seconds}")
    assert acc_pyr >= acc_one - 0.005
    assert res.passes == 2 * V + 2
