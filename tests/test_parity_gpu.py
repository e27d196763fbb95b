"""Parity of the CUDA engine (through the C ABI) with the CPU oracle on seeded
inputs. Tolerances: per-view NCC costs within 2e-3 (median) for the same
hypothesis; depth within 1 % and normals within 10 degrees (the accuracy the
depth-map stage is held to) on the stated fraction of pixels for iterated runs."""
import numpy as np
import pytest

import oracle.oracle as orc
from sensemap_b200 import STORE_F16, STORE_F32, STORE_U8
from sensemap_b200 import _native as N
from sensemap_b200 import synthetic as syn
from sensemap_b200.patch_match import PatchMatchACMMCuda
from tests.helpers import frac_close, perturbed_gt, photometric_options, problem_from_scene, small_planes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return small_planes(seed=5)


def run_engine(opt, prob, filt=False):
    with PatchMatchACMMCuda(opt, prob) as pm:
        if filt:
            pm.RunFilter(False)
            return {"depth": pm.GetDepthMap()}
        pm.Run()
        return {"depth": pm.GetDepthMap(), "normal": pm.GetNormalMap(), "conf": pm.GetConfMap(),
                "cost": pm.GetCostMap(), "view_sel": pm.GetViewSelMap()}


@pytest.mark.parametrize("storage", [STORE_U8, STORE_F16, STORE_F32])
def test_texture_model_matches_hardware(storage):
    """The oracle's model of hardware bilinear filtering (8-bit positions,
    integer 1/256 weights with w11 = round(A*B/256)) against the texture unit."""
    rng = np.random.default_rng(storage)
    img = rng.integers(0, 256, (9, 13)).astype(np.float32)
    xy = np.stack([rng.uniform(-2, 15, 4000), rng.uniform(-2, 11, 4000)], 1).astype(np.float32)
    xy[:64] = np.round(xy[:64] * 256) / 256  # exact 8-bit fractions
    out = np.zeros(len(xy), np.float32)
    N.check(N.lib().smvs_test_sample_texture(img.ctypes.data, 13, 9, storage, xy.ctypes.data, len(xy),
                                             out.ctypes.data))
    if storage == STORE_U8:
        stored = img / 255.0
    elif storage == STORE_F16:
        stored = img.astype(np.float16).astype(np.float32)
    else:
        stored = img
    stored = np.ascontiguousarray(stored, np.float32)
    model = np.array([orc.lib().orc_tex_bilinear(stored.ctypes.data, 13, 9, float(x), float(y)) for x, y in xy],
                     np.float32)
    if storage == STORE_F16:  # the unit returns FP16-rounded results for FP16 texels
        model = model.astype(np.float16).astype(np.float32)
    err = np.abs(out - model) / (1.0 if storage == STORE_U8 else 255.0)
    if storage == STORE_F32:
        assert err.max() == 0.0, f"max {err.max():.3g} at {xy[np.argmax(err)]}"
    elif storage == STORE_U8:  # fixed-point filtering of 8-bit texels: < 0.01 grey levels
        assert err.max() < 4e-5, f"max {err.max():.3g} at {xy[np.argmax(err)]}"
    else:  # FP16 result rounding: within one FP16 ulp
        assert np.mean(err == 0) > 0.9 and err.max() < 1e-3, f"max {err.max():.3g}"


def test_init_conf_matches_oracle(scene):
    init = perturbed_gt(scene, seed=2)
    prob = problem_from_scene(scene, init=init)
    opt = photometric_options(scene, iters=0, init_depth_random=False)
    gpu = run_engine(opt, prob)
    ref = orc.run(opt, prob)
    np.testing.assert_allclose(gpu["depth"], ref["depth"], rtol=0, atol=0)
    err = np.abs(gpu["cost"] - ref["cost"])
    assert np.median(err) < 2e-3 and np.quantile(err, 0.999) < 5e-2
    assert np.quantile(np.abs(gpu["conf"] - ref["conf"]), 0.99) < 1e-2
    assert np.mean(gpu["view_sel"] == ref["view_sel"]) > 0.98


def test_one_iteration_matches_oracle(scene):
    init = perturbed_gt(scene, seed=3)
    prob = problem_from_scene(scene, init=init)
    opt = photometric_options(scene, iters=1, init_depth_random=False)
    gpu = run_engine(opt, prob)
    ref = orc.run(opt, prob)
    assert frac_close(gpu["depth"], ref["depth"], 0.01) > 0.97
    assert syn.normal_accuracy(gpu["normal"], ref["normal"], 10.0) > 0.95


def test_full_photometric_run_matches_oracle(scene):
    prob = problem_from_scene(scene)
    opt = photometric_options(scene, iters=6)
    gpu = run_engine(opt, prob)
    ref = orc.run(opt, prob)
    gt = scene.views[scene.ref_index].depth_gt
    acc_gpu, acc_ref = syn.depth_accuracy(gpu["depth"], gt), syn.depth_accuracy(ref["depth"], gt)
    assert acc_gpu > 0.7
    assert abs(acc_gpu - acc_ref) < 0.03
    assert frac_close(gpu["depth"], ref["depth"], 0.01) > 0.85


def test_geometric_pass_and_filter_match_oracle():
    sc = small_planes(seed=6)
    n = len(sc.views)
    # Photometric maps of every view first (each view against all others).
    photo = []
    for r in range(n):
        prob = problem_from_scene(sc, ref=r)
        photo.append(run_engine(photometric_options(sc, iters=4, random_seed=r), prob))
    depths = [p["depth"] for p in photo]
    normals = [p["normal"] for p in photo]
    r = sc.ref_index
    prob = problem_from_scene(sc, depth_maps=depths, normal_maps=normals)
    opt = photometric_options(sc, iters=3, geom_consistency=True, init_depth_random=False,
                              geom_consistency_regularizer=0.1)
    gpu = run_engine(opt, prob)
    ref = orc.run(opt, prob)
    gt = sc.views[r].depth_gt
    assert frac_close(gpu["depth"], ref["depth"], 0.01) > 0.85
    assert abs(syn.depth_accuracy(gpu["depth"], gt) - syn.depth_accuracy(ref["depth"], gt)) < 0.03
    # RunFilter on the oracle's geometric map: integer decisions must agree.
    views_maps = list(depths)
    views_maps[r] = ref["depth"]
    fprob = problem_from_scene(sc, depth_maps=views_maps)
    fopt = photometric_options(sc, filter_min_num_consistent=2)
    g = run_engine(fopt, fprob, filt=True)["depth"]
    o = orc.run_filter(fopt, fprob)
    assert np.mean((g > 0) == (o > 0)) > 0.995
    both = (g > 0) & (o > 0)
    np.testing.assert_array_equal(g[both], o[both])


def test_fp16_storage_keeps_accuracy(scene):
    prob = problem_from_scene(scene)
    gt = scene.views[scene.ref_index].depth_gt
    acc = {}
    for st in (STORE_F32, STORE_F16, STORE_U8):
        out = run_engine(photometric_options(scene, iters=6, image_storage=st), prob)
        acc[st] = syn.depth_accuracy(out["depth"], gt)
    assert abs(acc[STORE_F16] - acc[STORE_F32]) < 0.02
    assert abs(acc[STORE_U8] - acc[STORE_F32]) < 0.02


def test_errors_are_status_codes(scene):
    prob = problem_from_scene(scene)
    opt = photometric_options(scene)
    pm = PatchMatchACMMCuda(opt, prob)
    with pytest.raises(N.SmvsError) as ei:
        pm.GetConfMap()
    assert ei.value.status == N.SMVS_ESTATE
    with pytest.raises(N.SmvsError) as ei:
        pm.RunFilter()
    assert ei.value.status == N.SMVS_EINVAL
    pm.close()
    bad = photometric_options(scene, geom_consistency=True)
    with pytest.raises(N.SmvsError) as ei:
        PatchMatchACMMCuda(bad, prob)
    assert ei.value.status == N.SMVS_EINVAL


def test_results_are_deterministic(scene):
    prob = problem_from_scene(scene)
    opt = photometric_options(scene, iters=3)
    a = run_engine(opt, prob)
    b = run_engine(opt, prob)
    np.testing.assert_array_equal(a["depth"], b["depth"])
    np.testing.assert_array_equal(a["cost"], b["cost"])


def test_post_filters_match_oracle(scene):
    """Curvature, median and confidence filters on given maps (0 iterations),
    so both sides filter identical inputs."""
    init = perturbed_gt(scene, seed=9, rel=0.03, ang_deg=15.0)
    maps = [v.depth_gt for v in scene.views]
    prob = problem_from_scene(scene, depth_maps=maps, init=init)
    opt = photometric_options(scene, iters=0, init_depth_random=False, geom_consistency=True, est_curvature=True,
                              median_filter=True, filter=True, conf_filter=True, conf_threshold=0.6)
    with PatchMatchACMMCuda(opt, prob) as pm:
        pm.Run()
        g = {"depth": pm.GetDepthMap(), "normal": pm.GetNormalMap(), "curv": pm.GetCurvatureMap()}
    o = orc.run(opt, prob)
    assert np.mean((g["depth"] > 0) == (o["depth"] > 0)) > 0.995
    assert frac_close(g["depth"], o["depth"], 1e-5, mask=(o["depth"] > 0)) > 0.99
    # Curvature is computed before the filters; gradient slice exact, angle slice within rounding.
    assert np.mean(np.abs(g["curv"][0].astype(int) - o["curvature"][0].astype(int)) <= 2) > 0.999
    assert np.mean(np.abs(g["curv"][1].astype(int) - o["curvature"][1].astype(int)) <= 20) > 0.99
