"""GPU parity of the Delaunay initial map (smvs_init_depth_from_delaunay)
against the C oracle (oracle/smvs_oracle_init.c), bit for bit.

The oracle rasterises the same triangulation (the library's host
triangulation, itself pinned against scipy's Qhull in the CPU tests) with the
same float and double operations; depth, normals and the depth range must be
identical, for host and device inputs, and the map must follow the surface.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sensemap_b200 import init_maps as IM
from sensemap_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return syn.planes_scene(seed=11, width=200, height=150, focal=160.0, num_src=3)


@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("count", [40, 3000])
def test_delaunay_bit_exact(scene, device, count):
    for view in range(len(scene.views)):
        v = scene.views[view]
        H, W = v.depth_gt.shape
        pts = syn.sparse_points(scene, (view + 1) % len(scene.views), count, seed=view)
        uv, _, _ = O.delaunay_points(W, H, v.K, v.R, v.T, pts)
        tris = IM.delaunay_triangles(uv)
        ref = O.init_from_delaunay(W, H, v.K, v.R, v.T, pts, tris)
        x = torch.from_numpy(pts).cuda() if device else pts
        got = IM.init_depth_from_delaunay(W, H, v.K, v.R, v.T, x)
        gd, gn = (got[0].cpu().numpy(), got[1].cpu().numpy()) if device else (got[0], got[1])
        assert np.array_equal(gd.view(np.uint32), ref[0].view(np.uint32))
        assert np.array_equal(gn.view(np.uint32), ref[1].view(np.uint32))
        assert got[2] == ref[2]
        if count == 3000:
            covered = gd > 0
            assert covered.mean() > 0.5
            gt = v.depth_gt
            ok = covered & (gt > 0)
            assert np.mean(np.abs(gd[ok] - gt[ok]) <= 0.05 * gt[ok]) > 0.8


def test_delaunay_empty_and_collinear(scene):
    v = scene.views[0]
    H, W = v.depth_gt.shape
    d, n, r = IM.init_depth_from_delaunay(W, H, v.K, v.R, v.T, np.zeros((0, 3), np.float32))
    assert not d.any() and not n.any() and r[1] == pytest.approx(110.0)
    pts = syn.sparse_points(scene, 0, 2, seed=1)
    d, n, _ = IM.init_depth_from_delaunay(W, H, v.K, v.R, v.T, pts)
    assert not d.any()
