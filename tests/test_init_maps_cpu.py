"""CPU checks of the initial-map oracle (oracle/smvs_oracle_init.c), which
restates InitDepthMap / InitDepthMapFromSparsePoint / Model2Depth / Ply2Depth
(patch_match_controller.cc:483-750, 1205-1307) sequentially."""
import numpy as np
import pytest

from oracle import oracle as O
from sensemap_b200 import _native as N
from sensemap_b200 import synthetic as syn


@pytest.fixture(scope="module")
def scene():
    return syn.planes_scene(seed=3, width=160, height=120, num_src=2)


def test_sparse_splat_is_windowed_minimum(scene):
    v = scene.views[1]
    H, W = v.depth_gt.shape
    pts = syn.sparse_points(scene, 1, 400, seed=2)
    d, n, rng = O.init_from_sparse_points(W, H, v.K, v.R, v.T, pts)
    # brute force: project in float like the reference, minimum over 7x7 windows
    K, R, T = (np.asarray(a, np.float32) for a in (v.K, v.R, v.T))
    Y = (pts @ R.T + T).astype(np.float32)
    Xc = (Y @ K.T).astype(np.float32)
    ref = np.full((H, W), np.inf, np.float32)
    zs = []
    for (x, y, z) in Xc:
        if not z > 0:
            continue
        qu, qv = np.float32(x) / np.float32(z), np.float32(y) / np.float32(z)
        if not (-1 < qu < W and -1 < qv < H):
            continue
        fu, fv = int(qu), int(qv)
        zs.append(z)
        win = ref[max(fv - 3, 0):min(fv + 3, H - 1) + 1, max(fu - 3, 0):min(fu + 3, W - 1) + 1]
        np.minimum(win, z, out=win)
    ref[np.isinf(ref)] = 0
    # numpy's product sums in another order: the same pixels, depths within an ulp or two
    assert np.mean((d > 0) == (ref > 0)) > 0.999
    both = (d > 0) & (ref > 0)
    np.testing.assert_allclose(d[both], ref[both], rtol=1e-6)
    assert not n.any()
    assert rng[0] == np.float32(1e-6) and abs(rng[1] - max(zs) * np.float32(1.1)) <= 1e-6 * rng[1]


def test_sparse_empty_range(scene):
    v = scene.views[0]
    d, n, rng = O.init_from_sparse_points(16, 12, v.K, v.R, v.T, np.zeros((0, 3), np.float32))
    assert not d.any() and rng == (np.float32(1e-6), np.float32(110.0))


def test_mesh_draws_front_faces_at_true_depth(scene):
    X, F, FN = syn.grid_mesh(scene, 1, step=6)
    for view in range(3):
        v = scene.views[view]
        H, W = v.depth_gt.shape
        d, n, rng = O.init_from_mesh(W, H, v.K, v.R, v.T, X, F, FN)
        m = (d > 0) & (v.depth_gt > 0)
        assert m.mean() > 0.5
        assert np.median(np.abs(d[m] - v.depth_gt[m]) / v.depth_gt[m]) < 1e-4
        assert np.allclose(np.linalg.norm(n[:, d > 0], axis=0), 1, atol=1e-5)
    v = scene.views[1]
    H, W = v.depth_gt.shape
    assert not O.init_from_mesh(W, H, v.K, v.R, v.T, X, F[:, ::-1], FN)[0].any()  # other winding
    assert not O.init_from_mesh(W, H, v.K, v.R, v.T, X, F, -FN)[0].any()  # back faces culled
    with pytest.raises(RuntimeError):
        O.init_from_mesh(W, H, v.K, v.R, v.T, X, np.array([[0, 1, len(X)]]), FN[:1])


def test_mesh_tie_first_writer(scene):
    """Two copies of a face: the sequential test keeps the first copy unless
    the second copy's double depth is below the stored float."""
    X, F, FN = syn.grid_mesh(scene, 1, step=12)
    v = scene.views[1]
    H, W = v.depth_gt.shape
    d1, n1, _ = O.init_from_mesh(W, H, v.K, v.R, v.T, X, F, FN)
    d2, n2, _ = O.init_from_mesh(W, H, v.K, v.R, v.T, X, np.concatenate([F, F]), np.concatenate([FN, -FN * 0 + FN]))
    assert np.array_equal(d1, d2) and np.array_equal(n1, n2)


def test_dense_points_odd_pixels(scene):
    P, PN = syn.dense_points(scene, 1, step=3)
    v = scene.views[1]
    H, W = v.depth_gt.shape
    d, n, rng = O.init_from_dense_points(W, H, v.K, v.R, v.T, P, PN, level=2)
    ys, xs = np.nonzero(d)
    assert len(ys) and (ys % 2 == 1).all() and (xs % 2 == 1).all()
    assert rng[0] == np.float32(1e-6) and rng[1] > 0


def test_init_abi_rejects_bad_arguments():
    import ctypes as C
    lib = N.lib()
    v = N.smvs_view()
    v.width, v.height = 0, 10
    buf = np.zeros(30, np.float32)
    assert lib.smvs_init_depth_from_sparse_points(C.byref(v), None, 0, N.MEM_HOST, buf.ctypes.data,
                                                  buf.ctypes.data, None, None) == N.SMVS_EINVAL
    v.width = 10
    assert lib.smvs_init_depth_from_dense_points(C.byref(v), None, None, 0, 99, N.MEM_HOST, buf.ctypes.data,
                                                 buf.ctypes.data, None, None) == N.SMVS_EINVAL
