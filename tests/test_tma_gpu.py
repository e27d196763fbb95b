"""Launch shapes of the checkerboard kernels. Each block's reference tile is
staged with one TMA load (cp.async.bulk.tensor) where the image qualifies, else
with plain loads; both fill the same shared-memory tile. A pixel's NCC windows
are split over 1, 2 or 4 threads whose partial moments are always combined in
the same order. Every map must be bit-identical whatever the launch shape."""
import numpy as np
import pytest

from sensemap_b200.patch_match import PatchMatchACMMCuda
from tests.helpers import photometric_options, problem_from_scene, small_planes

pytestmark = pytest.mark.gpu


def _run(scene, tma, block_x=32, iters=4, tpp=2, problem=None, **kw):
    opt = photometric_options(scene, iters=iters, **kw)
    pm = PatchMatchACMMCuda(opt, problem if problem is not None else problem_from_scene(scene))
    pm.SetTuning(block_x, ref_tile_tma=tma, threads_per_pixel=tpp)
    pm.Run()
    out = (pm.GetDepthMap(), pm.GetNormalMap(), pm.GetCostMap(), pm.GetViewSelMap(), pm.Tuning())
    pm.close()
    return out


@pytest.mark.parametrize("block_x", [8, 32, 64])
def test_tma_tiles_match_plain_loads(block_x):
    scene = small_planes(seed=2, w=200, h=120)  # rows of 800 bytes: TMA qualifies
    a = _run(scene, True, block_x)
    b = _run(scene, False, block_x)
    assert a[4]["ref_tile_tma"] and not b[4]["ref_tile_tma"]
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)


def test_tma_falls_back_for_unaligned_rows():
    scene = small_planes(seed=3, w=162, h=100)  # 648-byte rows: not a multiple of 16
    a = _run(scene, True)
    b = _run(scene, False)
    assert not a[4]["ref_tile_tma"]
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)


def test_tma_small_image_falls_back():
    scene = small_planes(seed=4, w=64, h=16)  # smaller than one tile box
    a = _run(scene, True, iters=2)
    b = _run(scene, False, iters=2)
    assert not a[4]["ref_tile_tma"]
    assert np.array_equal(a[0], b[0])


@pytest.mark.parametrize("tpp,block_x", [(1, 32), (2, 8), (2, 64), (4, 16), (4, 64)])
def test_threads_per_pixel_do_not_change_maps(tpp, block_x):
    scene = small_planes(seed=6, w=200, h=120)
    a = _run(scene, True, block_x, iters=4, tpp=tpp)
    b = _run(scene, True, 32, iters=4, tpp=2)
    assert a[4]["threads_per_pixel"] == tpp
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)


def test_threads_per_pixel_geometric_pass_and_step_two():
    """A geometric pass with a (5, 2) window through every threads-per-pixel."""
    from tests.helpers import perturbed_gt
    scene = small_planes(seed=7, w=200, h=120)
    depth = [v.depth_gt for v in scene.views]
    normal = [v.normal_gt for v in scene.views]
    prob = problem_from_scene(scene, depth_maps=depth, normal_maps=normal, init=perturbed_gt(scene))
    outs = [_run(scene, True, 32, iters=4, tpp=t, problem=prob, window_step=2, geom_consistency=True,
                 init_depth_random=False) for t in (1, 2, 4)]
    for o in outs[1:]:
        for x, y in zip(o[:4], outs[0][:4]):
            assert np.array_equal(x, y)


def test_autotune_picks_a_candidate_and_maps_do_not_change():
    from sensemap_b200.patch_match import autotune
    scene = small_planes(seed=5, w=200, h=120)
    opt = photometric_options(scene, iters=3)
    res = autotune(opt, problem_from_scene(scene), repeats=2)
    shapes = {(c["sweep_block_x"], c["threads_per_pixel"]) for c in res["candidates"]}
    assert (res["sweep_block_x"], res["threads_per_pixel"]) in shapes
    assert {8, 16, 32, 64} <= {c["sweep_block_x"] for c in res["candidates"]}
    assert {1, 2, 4} <= {c["threads_per_pixel"] for c in res["candidates"]}
    assert all(c["ms_per_sweep"] > 0 for c in res["candidates"])
    a = _run(scene, res["ref_tile_tma"], res["sweep_block_x"], iters=3, tpp=res["threads_per_pixel"])
    b = _run(scene, False, 32, iters=3)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("tma,block_x,cap", [(True, 32, 0), (True, 32, 7), (False, 32, 7), (True, 8, 5),
                                             (True, 64, 3)])
def test_persistent_launch_does_not_change_maps(tma, block_x, cap):
    """Thread-per-pixel kernels as a persistent grid: with a cap of a few blocks
    each block loops over many tiles (one TMA barrier, one phase per tile)."""
    from sensemap_b200 import _native as N
    scene = small_planes(seed=6, w=200, h=120)
    opt = photometric_options(scene, iters=4)
    pm = PatchMatchACMMCuda(opt, problem_from_scene(scene))
    pm.SetTuning(block_x, ref_tile_tma=tma, threads_per_pixel=1, persistent=True)
    N.check(N.lib().smvs_test_persistent_grid(cap))
    try:
        pm.Run()
        a = (pm.GetDepthMap(), pm.GetNormalMap(), pm.GetCostMap(), pm.GetViewSelMap(), pm.Tuning())
    finally:
        N.check(N.lib().smvs_test_persistent_grid(0))
        pm.close()
    b = _run(scene, True, 32, iters=4, tpp=2)
    assert a[4]["persistent"] and a[4]["threads_per_pixel"] == 1 and a[4]["ref_tile_tma"] == tma
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)
