"""The no-allocation geometric-consistency filter (smvs_filter_depth_map_noalloc).

It exists for callers that cannot allocate device memory — a process working
inside a device-memory budget it reserved at start-up, or work issued on a
stream that is being captured into a CUDA graph — so it takes every input and
output as a caller-owned device buffer and keeps its scratch in a fixed device
array. This checks it through the C ABI against the allocating entry point
(smvs_run_filter) on the same inputs, for two calls in a row (the second call
reuses the scratch the first one left behind), and that it rejects more source
views than its scratch holds. Collected last so a failure here cannot stop the
other tests from running.
"""
import ctypes as C

import numpy as np
import pytest

from sensemap_b200 import _native as N
from sensemap_b200.patch_match import PatchMatchACMMCuda
from tests.helpers import photometric_options, problem_from_scene, small_planes

pytestmark = pytest.mark.gpu


def _device_problem(scene, depth_tensors):
    """smvs_problem over device depth maps (pixels are not read by the filter)."""
    prob = N.smvs_problem()
    views = []
    for i, v in enumerate(scene.views):
        cv = N.smvs_view()
        cv.width, cv.height, cv.pixel_format = v.image.shape[1], v.image.shape[0], N.PIX_F32
        cv.pixels = None
        cv.K[:] = list(np.asarray(v.K, np.float64).reshape(9))
        cv.R[:] = list(np.asarray(v.R, np.float64).reshape(9))
        cv.T[:] = list(np.asarray(v.T, np.float64).reshape(3))
        cv.scale = 1.0
        cv.depth = depth_tensors[i].data_ptr()
        views.append(cv)
    ref = scene.ref_index
    prob.ref = views[ref]
    srcs = (N.smvs_view * (len(views) - 1))(*[v for i, v in enumerate(views) if i != ref])
    prob.src = srcs
    prob.num_src = len(views) - 1
    prob.memory = N.MEM_DEVICE
    return prob, srcs


def test_noalloc_filter_matches_allocating_entry_point():
    import torch
    scene = small_planes(seed=31)
    rng = np.random.default_rng(7)
    maps = []
    for v in scene.views:
        d = v.depth_gt * (1 + rng.normal(0, 0.01, v.depth_gt.shape)).astype(np.float32)
        d[rng.random(d.shape) < 0.1] = 0
        maps.append(d.astype(np.float32))
    opt = photometric_options(scene, filter_min_num_consistent=2)

    # Existing (allocating) entry point.
    with PatchMatchACMMCuda(opt, problem_from_scene(scene, depth_maps=maps)) as pm:
        pm.RunFilter(False)
        expected = pm.GetDepthMap()

    dev = [torch.from_numpy(m).cuda() for m in maps]
    prob, keep = _device_problem(scene, dev)
    copt = opt.to_c()
    for call in range(2):
        out = torch.full_like(dev[scene.ref_index], -1.0)
        N.check(N.lib().smvs_filter_depth_map_noalloc(C.byref(copt), C.byref(prob), C.c_void_p(out.data_ptr()), 0,
                                                      None))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.mean((got > 0) == (expected > 0)) > 0.999, f"call {call}"
        both = (got > 0) & (expected > 0)
        np.testing.assert_array_equal(got[both], expected[both])
        assert (got >= 0).all()  # every pixel written


def test_noalloc_filter_rejects_too_many_views():
    import torch
    scene = small_planes(seed=32)
    d = torch.ones((scene.views[0].image.shape[0], scene.views[0].image.shape[1]), device="cuda")
    prob, _ = _device_problem(scene, [d] * len(scene.views))
    many = (N.smvs_view * (N.SMVS_MAX_SRC + 1))(*([prob.src[0]] * (N.SMVS_MAX_SRC + 1)))
    prob.src = many
    prob.num_src = N.SMVS_MAX_SRC + 1
    out = torch.zeros_like(d)
    st = N.lib().smvs_filter_depth_map_noalloc(C.byref(photometric_options(scene).to_c()), C.byref(prob),
                                               C.c_void_p(out.data_ptr()), 0, None)
    assert st == N.SMVS_EINVAL
    assert "32" in N.last_error()
