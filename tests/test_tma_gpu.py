"""The checkerboard kernels stage each block's reference tile with one TMA
load (cp.async.bulk.tensor) where the image qualifies, else with plain loads;
both fill the same shared-memory tile, so every map must be bit-identical."""
import numpy as np
import pytest

from sensemap_b200.patch_match import PatchMatchACMMCuda
from tests.helpers import photometric_options, problem_from_scene, small_planes

pytestmark = pytest.mark.gpu


def _run(scene, tma, block_x=32, iters=4):
    opt = photometric_options(scene, iters=iters)
    pm = PatchMatchACMMCuda(opt, problem_from_scene(scene))
    pm.SetTuning(block_x, ref_tile_tma=tma)
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


def test_autotune_picks_a_candidate_and_maps_do_not_change():
    from sensemap_b200.patch_match import autotune
    scene = small_planes(seed=5, w=200, h=120)
    opt = photometric_options(scene, iters=3)
    res = autotune(opt, problem_from_scene(scene), repeats=2)
    shapes = {(c["sweep_block_x"], c["ref_tile_tma"]) for c in res["candidates"]}
    assert (res["sweep_block_x"], res["ref_tile_tma"]) in shapes
    assert {8, 16, 32, 64} <= {c["sweep_block_x"] for c in res["candidates"]}
    assert all(c["ms_per_sweep"] > 0 for c in res["candidates"])
    a = _run(scene, res["ref_tile_tma"], res["sweep_block_x"], iters=3)
    b = _run(scene, False, 32, iters=3)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
