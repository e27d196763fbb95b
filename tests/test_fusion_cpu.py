"""Depth-map fusion on the CPU: the C oracle (oracle/smvs_oracle_fusion.c)
pinned against the pure-Python restatement (oracle/fusion_oracle.py), the
image order, the float form of the depth-error test, and argument checks of
the C ABI (no GPU needed)."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import fusion_oracle as FP
from oracle import oracle as O
from sensemap_b200 import _native as N
from sensemap_b200 import synthetic as syn
from sensemap_b200.fusion import FusionImage, FusionOptions, fusion_structs


def _same(r, py):
    pts, vis, order, masks = py
    P = r["points"]
    assert r["order"] == order
    assert len(P) == len(pts)
    for k, p in enumerate(pts):
        for f in ("x", "y", "z", "nx", "ny", "nz", "score"):
            assert np.float32(p[f]).view(np.uint32) == P[f][k].view(np.uint32), (k, f, p[f], P[f][k])
        assert (p["r"], p["g"], p["b"]) == (P["r"][k], P["g"][k], P["b"][k])
        assert list(r["vis_images"][r["vis_offsets"][k]:r["vis_offsets"][k + 1]]) == vis[k]
    for a, b in zip(r["masks"], masks):
        assert np.array_equal(a, b)


@pytest.fixture(scope="module")
def tiny():
    scene = syn.planes_scene(seed=3, width=64, height=48, focal=52.0, num_src=2)
    return syn.fusion_inputs(scene, seed=1)


@pytest.mark.parametrize("opts", [
    FusionOptions(),
    FusionOptions(step_size=2, num_slices=3, min_num_visible_images=2, min_num_pixels=2),
    FusionOptions(with_normal=False, max_num_pixels=4, min_num_pixels=2, min_num_visible_images=1,
                  max_traversal_depth=2),
    FusionOptions(max_reproj_error=1.0, max_depth_error=0.005, max_normal_error=5.0, min_num_pixels=3),
])
def test_oracle_matches_python_restatement(tiny, opts):
    ims, ov = tiny
    _same(O.fusion_run(opts, ims, ov), FP.fuse(opts, ims, ov))


def test_oracle_rigs_unused_images_and_short_lists():
    scene = syn.planes_scene(seed=7, width=56, height=40, focal=46.0, num_src=3)
    ims, ov = syn.fusion_inputs(scene, seed=2, rig_every=2)
    ims[3] = FusionImage(K=ims[3].K, R=ims[3].R, T=ims[3].T)  # no depth map: not used
    ov[1] = ov[1][:1]
    opts = FusionOptions(min_num_visible_images=2)
    r = O.fusion_run(opts, ims, ov)
    _same(r, FP.fuse(opts, ims, ov))
    assert 3 not in r["order"] and not r["masks"][3].size
    assert r["order"][0] == 1  # the first image that is not a rig image


def test_oracle_find_next_image_order():
    """FindNextImage (fusion.cc:697-727): overlapping non-rig images first, then
    overlapping rig images, then the first unfused non-rig image, then any."""
    scene = syn.planes_scene(seed=1, width=40, height=32, focal=34.0, num_src=4)
    ims, _ = syn.fusion_inputs(scene, seed=0)
    for k, im in enumerate(ims):
        im.is_rig = k in (0, 2)
    ov = [[2, 4], [], [0], [4], [2]]
    r = O.fusion_run(FusionOptions(), ims, ov)
    # start 1 (first non-rig); its list is empty -> first non-rig 3; 3 -> 4; 4 -> rig 2; 2 -> rig 0.
    assert r["order"] == [1, 3, 4, 2, 0]
    assert FP.fuse(FusionOptions(), ims, ov)[2] == r["order"]


def _float_floor(d: float) -> np.float32:
    """The CUDA unit's threshold: the largest float <= d."""
    f = np.float32(d)
    if float(f) > d:
        f = np.nextafter(f, np.float32(-np.inf))
    return f


@pytest.mark.parametrize("d", [float(np.float32(0.01)), 0.01, 0.02, 1e-3, 0.3, 0.0])
def test_float_form_of_the_depth_error_test(d):
    """(double)x > max_depth_error (fusion.cc:1909) equals x > largest float <= it."""
    thr = _float_floor(d)
    lo = np.float32(max(d / 2, 1e-30)).view(np.int32)
    hi = np.float32(max(d * 2, 1e-29)).view(np.int32)
    xs = np.arange(lo, hi, max(1, (hi - lo) // 2000000), dtype=np.int32).view(np.float32)
    xs = np.concatenate([xs, [thr, np.nextafter(thr, np.float32(1)), np.float32(d), 0.0, np.inf, np.nan]]).astype(
        np.float32)
    assert np.array_equal(xs.astype(np.float64) > d, xs > thr)


def test_defaults_match_reference():
    o = N.smvs_fusion_options()
    N.check(N.lib().smvs_fusion_options_default(C.byref(o)))
    py = FusionOptions()
    # StereoFusion::Options (fusion.h:48-139)
    assert (o.step_size, o.min_num_pixels, o.max_num_pixels, o.min_num_visible_images, o.max_traversal_depth) == \
        (1, 5, 10000, 3, 100)
    assert o.max_reproj_error == 2.0 and o.max_depth_error == float(np.float32(0.01)) and o.max_normal_error == 10.0
    for name, _ in N.smvs_fusion_options._fields_:
        assert float(getattr(py, name)) == float(getattr(o, name)), name


@pytest.mark.parametrize("field,value", [("min_num_pixels", 1), ("max_num_pixels", 3), ("max_traversal_depth", 0),
                                         ("step_size", 0), ("num_slices", 0), ("max_depth_error", -1.0),
                                         ("min_num_visible_images", -1)])
def test_create_rejects_bad_options(tiny, field, value):
    ims, ov = tiny
    opts = FusionOptions()
    setattr(opts, field, value)
    views, off, flat, memory, keep = fusion_structs(ims, ov)
    h = C.c_void_p()
    st = N.lib().smvs_fusion_create(C.byref(opts.to_c()), views, len(ims), off.ctypes.data, flat.ctypes.data, memory,
                                    None, C.byref(h))
    assert st == N.SMVS_EINVAL and not h.value
    assert "fusion" in N.last_error()


def test_create_rejects_bad_overlaps(tiny):
    ims, ov = tiny
    views, off, flat, memory, keep = fusion_structs(ims, [[0, 9]] + ov[1:])
    h = C.c_void_p()
    st = N.lib().smvs_fusion_create(C.byref(FusionOptions().to_c()), views, len(ims), off.ctypes.data,
                                    flat.ctypes.data, memory, None, C.byref(h))
    assert st == N.SMVS_EINVAL


def test_oracle_on_a_larger_scene():
    scene = syn.planes_scene(seed=3, width=320, height=240, focal=256.0, num_src=4)
    ims, ov = syn.fusion_inputs(scene, seed=1)
    r = O.fusion_run(FusionOptions(), ims, ov)
    P = r["points"]
    assert len(P) > 10000
    nvis = np.diff(r["vis_offsets"].astype(np.int64))
    assert nvis.min() >= 3 and nvis.max() <= len(ims)
    for k in range(0, len(P), 97):
        v = r["vis_images"][r["vis_offsets"][k]:r["vis_offsets"][k + 1]]
        assert np.all(np.diff(v.astype(np.int64)) > 0)
    assert np.all(np.abs(np.sqrt(P["nx"] ** 2 + P["ny"] ** 2 + P["nz"] ** 2) - 1) < 1e-5)
    assert np.all((P["score"] >= 0) & (P["score"] <= 1))
    assert sum(int(m.sum()) for m in r["masks"]) >= 5 * len(P)


def test_oracle_concurrent_slices_timing_mode():
    """The timing baseline with the reference's concurrent row slices: its
    result depends on the timing, but it fuses the same scene into a similar
    cloud."""
    scene = syn.planes_scene(seed=3, width=320, height=240, focal=256.0, num_src=4)
    ims, ov = syn.fusion_inputs(scene, seed=1)
    one = O.fusion_run(FusionOptions(), ims, ov, masks=False)
    many = O.fusion_run(FusionOptions(), ims, ov, masks=False, threads=4)
    assert abs(len(many["points"]) - len(one["points"])) < 0.1 * len(one["points"])
    nvis = np.diff(many["vis_offsets"].astype(np.int64))
    assert nvis.min() >= 3 and many["order"] == one["order"]


def test_oracle_image_without_seed_pixels(tiny):
    """An image too narrow for a seed (6 pixels: all inside the blank border)
    is fused without points and never entered by a traversal."""
    ims, ov = tiny
    ims = list(ims)
    im = ims[1]
    ims[1] = FusionImage(K=im.K, R=im.R, T=im.T, depth=np.ascontiguousarray(im.depth[:, :6]),
                         normal=np.ascontiguousarray(im.normal[:, :, :6]),
                         color=np.ascontiguousarray(im.color[:, :6]))
    r = O.fusion_run(FusionOptions(), ims, ov)
    _same(r, FP.fuse(FusionOptions(), ims, ov))
    assert 1 in r["order"] and not r["masks"][1].any()
