"""GPU parity of the initial maps from the model (smvs_init_depth_from_*).

The CUDA unit (sensemap_b200/csrc/smvs_init_maps.cu) rebuilds the reference's
sequential depth tests from order-independent atomics; the CPU oracle
(oracle/smvs_oracle_init.c) runs them one candidate after another in the
reference's order with the same arithmetic. Depth, normal and depth range
must match bit for bit, including repeated faces and points (ties), for host
and device inputs, and for any order of the candidates.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sensemap_b200 import init_maps as IM
from sensemap_b200 import synthetic as syn
from sensemap_b200._native import SmvsError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return syn.planes_scene(seed=5, width=200, height=150, num_src=3)


def _same(got, ref):
    gd, gn, gr = got
    rd, rn, rr = ref
    if torch.is_tensor(gd):
        gd, gn = gd.cpu().numpy(), gn.cpu().numpy()
    assert np.array_equal(gd, rd), f"depth differs at {np.count_nonzero(gd != rd)} pixels"
    assert np.array_equal(gn, rn), f"normal differs at {np.count_nonzero(gn != rn)} entries"
    assert gr == rr


@pytest.mark.parametrize("device", [False, True])
def test_sparse_points_bit_exact(scene, device):
    for view in range(len(scene.views)):
        v = scene.views[view]
        H, W = v.depth_gt.shape
        pts = syn.sparse_points(scene, (view + 1) % len(scene.views), 3000, seed=view)  # seen from another view
        x = torch.from_numpy(pts).cuda() if device else pts
        _same(IM.init_depth_from_sparse_points(W, H, v.K, v.R, v.T, x), O.init_from_sparse_points(W, H, v.K, v.R,
                                                                                                   v.T, pts))


@pytest.mark.parametrize("device", [False, True])
def test_mesh_bit_exact(scene, device):
    X, F, FN = syn.grid_mesh(scene, 0, step=5, duplicate_frac=0.3, seed=1)
    for view in range(len(scene.views)):
        v = scene.views[view]
        H, W = v.depth_gt.shape
        args = [torch.from_numpy(a).cuda() for a in (X, F, FN)] if device else (X, F, FN)
        ref = O.init_from_mesh(W, H, v.K, v.R, v.T, X, F, FN)
        assert (ref[0] > 0).mean() > 0.3
        _same(IM.init_depth_from_mesh(W, H, v.K, v.R, v.T, *args), ref)


def test_mesh_any_face_order(scene):
    """The reference's result depends on the face order only through ties; the
    GPU result follows whatever order it is given."""
    X, F, FN = syn.grid_mesh(scene, 1, step=4, duplicate_frac=0.5, seed=2)
    v = scene.views[2]
    H, W = v.depth_gt.shape
    for seed in range(3):
        order = np.random.default_rng(seed).permutation(len(F))
        f, fn = F[order], FN[order]
        _same(IM.init_depth_from_mesh(W, H, v.K, v.R, v.T, X, f, fn), O.init_from_mesh(W, H, v.K, v.R, v.T, X, f, fn))


@pytest.mark.parametrize("device", [False, True])
def test_dense_points_bit_exact(scene, device):
    P, PN = syn.dense_points(scene, 0, step=2, duplicate_frac=0.4, seed=3)
    for view in range(len(scene.views)):
        v = scene.views[view]
        H, W = v.depth_gt.shape
        args = [torch.from_numpy(a).cuda() for a in (P, PN)] if device else (P, PN)
        ref = O.init_from_dense_points(W, H, v.K, v.R, v.T, P, PN, 2)
        _same(IM.init_depth_from_dense_points(W, H, v.K, v.R, v.T, *args, level=2), ref)
    v = scene.views[0]
    H, W = v.depth_gt.shape
    for level in (0, 1, 3):
        _same(IM.init_depth_from_dense_points(W, H, v.K, v.R, v.T, P, PN, level=level),
              O.init_from_dense_points(W, H, v.K, v.R, v.T, P, PN, level))


def test_empty_inputs_and_errors(scene):
    v = scene.views[0]
    d, n, r = IM.init_depth_from_sparse_points(32, 24, v.K, v.R, v.T, np.zeros((0, 3), np.float32))
    assert not d.any() and not n.any() and r == (np.float32(1e-6), np.float32(110.0))
    d, n, r = IM.init_depth_from_mesh(32, 24, v.K, v.R, v.T, np.zeros((0, 3)), np.zeros((0, 3), np.int32),
                                      np.zeros((0, 3)))
    assert not d.any() and r == (np.float32(1e-6), np.float32(110.0))
    X, F, FN = syn.grid_mesh(scene, 0, step=20)
    F = F.copy()
    F[3, 1] = len(X) + 5
    with pytest.raises(SmvsError):
        IM.init_depth_from_mesh(200, 150, v.K, v.R, v.T, X, F, FN)


def test_heightfield_mesh_larger(scene):
    hs = syn.heightfield_scene(seed=4, width=400, height=300, focal=300.0, num_src=2, device="cuda")
    X, F, FN = syn.grid_mesh(hs, 0, step=3, duplicate_frac=0.1)
    for view in range(len(hs.views)):
        v = hs.views[view]
        H, W = v.depth_gt.shape
        ref = O.init_from_mesh(W, H, v.K, v.R, v.T, X, F, FN)
        _same(IM.init_depth_from_mesh(W, H, v.K, v.R, v.T, X, F, FN), ref)
        m = (ref[0] > 0) & (v.depth_gt > 0)
        assert np.median(np.abs(ref[0][m] - v.depth_gt[m]) / v.depth_gt[m]) < 0.01
