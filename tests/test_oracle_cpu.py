"""The CPU oracle on its own: generator, texture model, pose algebra, FP32 vs
FP64 costs, convergence on a seeded scene, and the synthetic scenes' ground
truth (multi-view consistent). No GPU."""
import numpy as np
import pytest

import oracle.oracle as orc
from sensemap_b200 import synthetic as syn
from tests.helpers import perturbed_gt, photometric_options, problem_from_scene, small_planes


def test_uniform_range_and_determinism():
    vals = np.array([orc.uniform(7, 3, p, d) for p in range(200) for d in range(5)])
    assert vals.min() > 0 and vals.max() <= 1
    assert abs(vals.mean() - 0.5) < 0.05
    assert orc.uniform(7, 3, 11, 2) == orc.uniform(7, 3, 11, 2)
    assert orc.uniform(7, 3, 11, 2) != orc.uniform(8, 3, 11, 2)


def test_texture_model_interpolates_and_borders():
    img = np.arange(12, dtype=np.float32).reshape(3, 4)
    f = lambda x, y: orc.lib().orc_tex_bilinear(img.ctypes.data, 4, 3, x, y)
    assert f(0.5, 0.5) == 0.0 and f(1.5, 0.5) == 1.0 and f(1.5, 2.5) == 9.0
    assert abs(f(1.0, 0.5) - 0.5) < 1e-6  # halfway between texels 0 and 1
    assert f(-5.0, 1.0) == 0.0 and f(1.0, 40.0) == 0.0
    assert abs(f(0.0, 0.5) - 0.0) < 1e-6  # blends with the zero border


@pytest.fixture(scope="module")
def scene():
    return small_planes(seed=3)


def test_pose_records_are_consistent(scene):
    out = orc.run(photometric_options(scene, iters=0), problem_from_scene(scene))
    for rec in out["poses"]:
        P = rec[19:31].reshape(3, 4).astype(np.float64)
        iP = rec[31:43].reshape(3, 4).astype(np.float64)
        P4 = np.vstack([P, [0, 0, 0, 1]])
        iP4 = np.vstack([iP, [0, 0, 0, 1]])
        np.testing.assert_allclose(P4 @ iP4, np.eye(4), atol=2e-4)
        R = rec[4:13].reshape(3, 3)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-5)


def test_fp32_cost_matches_fp64_evaluator(scene):
    d, n = perturbed_gt(scene, rel=0.0, ang_deg=0.0)
    rng = np.random.default_rng(0)
    H, W = d.shape
    rows = rng.integers(8, H - 8, 300)
    cols = rng.integers(8, W - 8, 300)
    c32, c64 = orc.eval_costs(photometric_options(scene), problem_from_scene(scene), rows, cols, d[rows, cols],
                              n[:, rows, cols].T)
    err = np.abs(c32 - c64)
    # Fixed-point texture weights and FP32 rounding: small per-cost error.
    assert np.median(err) < 2e-3 and np.quantile(err, 0.99) < 2e-2
    # At the true surface most views agree well.
    assert np.median(c64) < 0.5


def test_oracle_converges_on_planes(scene):
    out = orc.run(photometric_options(scene, iters=6), problem_from_scene(scene))
    gt = scene.views[scene.ref_index].depth_gt
    assert syn.depth_accuracy(out["depth"], gt) > 0.75
    assert out["view_sel"].max() < (1 << 4)


def test_synthetic_ground_truth_is_multiview_consistent():
    sc = syn.heightfield_scene(seed=0, width=96, height=72, focal=72.0, num_src=3)
    ref, src = sc.views[0], sc.views[1]
    H, W = ref.depth_gt.shape
    ys, xs = np.mgrid[0:H, 0:W]
    Ki = np.linalg.inv(ref.K)
    pc = np.stack([xs, ys, np.ones_like(xs)], -1) @ Ki.T * ref.depth_gt[..., None]
    Xw = (pc - ref.T) @ ref.R  # R^T (x - T)
    xs_cam = Xw @ src.R.T + src.T
    uv = xs_cam @ src.K.T
    u, v = uv[..., 0] / uv[..., 2], uv[..., 1] / uv[..., 2]
    ok = (u >= 1) & (u < W - 2) & (v >= 1) & (v < H - 2)
    ui, vi = np.round(u[ok]).astype(int), np.round(v[ok]).astype(int)
    rel = np.abs(src.depth_gt[vi, ui] - xs_cam[..., 2][ok]) / xs_cam[..., 2][ok]
    assert ok.mean() > 0.5 and np.median(rel) < 0.01
