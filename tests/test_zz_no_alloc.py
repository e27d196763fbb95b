"""The no-allocation geometric-consistency filter (smvs_filter_depth_map_noalloc).

Some callers of this library cannot allocate device memory: a serving process
that reserved its whole device budget at start-up and may not grow it per
request, or a host whose framework owns every device allocation. For them the
filter takes every input and output as a caller-owned device buffer and keeps
its only scratch (the source views' pose records) in a fixed device array.

These tests call it through the C ABI and compare it with the allocating entry
point (smvs_create + smvs_run_filter) on the same inputs, for two calls in a
row whose problems differ (another reference view and fewer source views), so
that a second call reading the first call's leftover scratch would fail. They
also check that it rejects more source views than its scratch holds and options
the engine rejects. Collected last, so a failure here cannot stop the other
tests from running.
"""
import ctypes as C

import numpy as np
import pytest

from sensemap_b200 import _native as N
from sensemap_b200.patch_match import PatchMatchACMMCuda, Problem, View
from tests.helpers import photometric_options, small_planes

pytestmark = pytest.mark.gpu

# Keep/drop decisions may differ where a reprojection error lies within the
# texture unit's 1/256 position grid of the limit: the allocating filter samples
# through hardware textures, this one with the same 8-bit weights in software.
MAX_DECISION_MISMATCH = 1e-3


def _device_problem(scene, ref, srcs, depth_tensors):
    """smvs_problem over device depth maps (pixels are not read by the filter)."""
    def view(i):
        v = scene.views[i]
        cv = N.smvs_view()
        cv.width, cv.height, cv.pixel_format = v.image.shape[1], v.image.shape[0], N.PIX_F32
        cv.pixels = None
        cv.K[:] = list(np.asarray(v.K, np.float64).reshape(9))
        cv.R[:] = list(np.asarray(v.R, np.float64).reshape(9))
        cv.T[:] = list(np.asarray(v.T, np.float64).reshape(3))
        cv.scale = 1.0
        cv.depth = depth_tensors[i].data_ptr()
        return cv

    prob = N.smvs_problem()
    prob.ref = view(ref)
    arr = (N.smvs_view * len(srcs))(*[view(i) for i in srcs])
    prob.src = arr
    prob.num_src = len(srcs)
    prob.memory = N.MEM_DEVICE
    return prob, arr


def _noisy_maps(scene, seed):
    rng = np.random.default_rng(seed)
    maps = []
    for v in scene.views:
        d = v.depth_gt * (1 + rng.normal(0, 0.01, v.depth_gt.shape)).astype(np.float32)
        d[rng.random(d.shape) < 0.1] = 0
        maps.append(d.astype(np.float32))
    return maps


def _allocating_filter(scene, opt, ref, srcs, maps):
    views = [View(v.image, v.K, v.R, v.T, depth=maps[i]) for i, v in enumerate(scene.views)]
    with PatchMatchACMMCuda(opt, Problem(ref, list(srcs), views)) as pm:
        pm.RunFilter(False)
        return pm.GetDepthMap()


def test_noalloc_filter_matches_allocating_entry_point():
    import torch
    N.lib().smvs_test_take_cuda_error()  # start from a clean thread state
    scene = small_planes(seed=31)
    maps = _noisy_maps(scene, 7)
    opt = photometric_options(scene, filter_min_num_consistent=2)
    copt = opt.to_c()
    dev = [torch.from_numpy(m).cuda() for m in maps]
    # Two calls in a row on the same stream; the second one filters another
    # reference view against fewer source views.
    calls = [(0, [1, 2, 3, 4]), (2, [0, 3])]
    for k, (ref, srcs) in enumerate(calls):
        expected = _allocating_filter(scene, opt, ref, srcs, maps)
        prob, keep = _device_problem(scene, ref, srcs, dev)
        out = torch.full_like(dev[ref], -1.0)
        N.check(N.lib().smvs_filter_depth_map_noalloc(C.byref(copt), C.byref(prob), C.c_void_p(out.data_ptr()), 0,
                                                      None))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        d_in = maps[ref]
        # Every pixel is written, with the input depth or with 0.
        assert ((got == d_in) | (got == 0)).all(), f"call {k}"
        mismatch = float(np.mean((got > 0) != (expected > 0)))
        assert mismatch <= MAX_DECISION_MISMATCH, f"call {k}: keep/drop decisions differ on {mismatch:.5f}"
        # The problem is not trivial: the filter drops some pixels and keeps most.
        assert 0.05 < float(np.mean(expected > 0)) < 0.99


def test_noalloc_filter_rejects_too_many_views_and_bad_options():
    import torch
    scene = small_planes(seed=32)
    d = torch.ones((scene.views[0].image.shape[0], scene.views[0].image.shape[1]), device="cuda")
    prob, _ = _device_problem(scene, 0, [1, 2, 3, 4], [d] * len(scene.views))
    many = (N.smvs_view * (N.SMVS_MAX_SRC + 1))(*([prob.src[0]] * (N.SMVS_MAX_SRC + 1)))
    prob.src = many
    prob.num_src = N.SMVS_MAX_SRC + 1
    out = torch.zeros_like(d)
    opt = photometric_options(scene)
    st = N.lib().smvs_filter_depth_map_noalloc(C.byref(opt.to_c()), C.byref(prob), C.c_void_p(out.data_ptr()), 0,
                                               None)
    assert st == N.SMVS_EINVAL
    assert "32" in N.last_error()
    prob2, _ = _device_problem(scene, 0, [1, 2], [d] * len(scene.views))
    bad = photometric_options(scene, filter_min_num_consistent=-1)
    st = N.lib().smvs_filter_depth_map_noalloc(C.byref(bad.to_c()), C.byref(prob2), C.c_void_p(out.data_ptr()), 0,
                                               None)
    assert st == N.SMVS_EINVAL
