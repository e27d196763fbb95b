"""GPU parity of the depth-map fusion (StereoFusion) against the C oracle.

The CUDA unit (sensemap_b200/csrc/smvs_fusion.cu) replays each seed's
traversal in dependency order; the oracle (oracle/smvs_oracle_fusion.c) runs
the reference's loop seed after seed. Points (every field, bit for bit), their
images, the image order and every fused-pixel mask must be identical.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sensemap_b200 import _native as N
from sensemap_b200 import synthetic as syn
from sensemap_b200.fusion import FusionImage, FusionOptions, StereoFusion

pytestmark = pytest.mark.gpu


def _run(opts, ims, ov):
    with StereoFusion(opts, ims, ov) as f:
        f.Run()
        pts = f.GetFusedPoints().copy()
        off, vis = f.VisibilityCSR()
        out = {"points": pts, "vis_offsets": off.copy(), "vis_images": vis.copy(), "order": f.ImageOrder(),
               "masks": [f.FusedPixelMask(k) for k in range(len(ims))], "launches": f.LaunchCount()}
    return out


def _same(got, ref):
    assert got["order"] == ref["order"]
    for k, (a, b) in enumerate(zip(got["masks"], ref["masks"])):
        assert np.array_equal(a, b), f"mask of image {k} differs at {np.count_nonzero(a != b)} pixels"
    gp, rp = got["points"], ref["points"]
    assert len(gp) == len(rp), (len(gp), len(rp))
    assert np.array_equal(gp.view(np.uint8), rp.view(np.uint8)), \
        f"{np.count_nonzero(np.any(gp.view(np.uint8).reshape(len(gp), -1) != rp.view(np.uint8).reshape(len(rp), -1), axis=1))} points differ"
    assert np.array_equal(got["vis_offsets"], ref["vis_offsets"])
    assert np.array_equal(got["vis_images"], ref["vis_images"])


@pytest.fixture(scope="module")
def planes():
    scene = syn.planes_scene(seed=3, width=200, height=150, focal=160.0, num_src=4)
    return syn.fusion_inputs(scene, seed=1)


@pytest.mark.parametrize("opts", [
    FusionOptions(),
    FusionOptions(step_size=2, num_slices=3),
    FusionOptions(with_normal=False, max_num_pixels=6, min_num_pixels=2, min_num_visible_images=1,
                  max_traversal_depth=3),
    FusionOptions(max_reproj_error=1.0, max_depth_error=0.005, max_normal_error=5.0, min_num_pixels=3),
])
def test_bit_exact_planes(planes, opts):
    ims, ov = planes
    got = _run(opts, ims, ov)
    assert got["launches"] > 0
    ref = O.fusion_run(opts, ims, ov)
    assert len(ref["points"]) > 100
    _same(got, ref)


def test_device_inputs(planes):
    ims, ov = planes
    dev = [FusionImage(K=i.K, R=i.R, T=i.T, depth=torch.from_numpy(i.depth).cuda(),
                       normal=torch.from_numpy(i.normal).cuda(), color=torch.from_numpy(i.color).cuda(),
                       is_rig=i.is_rig) for i in ims]
    _same(_run(FusionOptions(), dev, ov), O.fusion_run(FusionOptions(), ims, ov))


def test_rigs_unused_image_and_missing_color():
    scene = syn.planes_scene(seed=7, width=160, height=120, focal=128.0, num_src=4)
    ims, ov = syn.fusion_inputs(scene, seed=2, rig_every=2)
    ims[2] = FusionImage(K=ims[2].K, R=ims[2].R, T=ims[2].T)  # no depth map: not used
    ims[3].color = None
    ov[1] = ov[1][:2]
    opts = FusionOptions(min_num_visible_images=2)
    _same(_run(opts, ims, ov), O.fusion_run(opts, ims, ov))


@pytest.mark.parametrize("caps", [(8, 0, 0), (0, 8, 0), (0, 0, 16), (12, 10, 24)])
def test_overflow_paths(planes, caps):
    """Records over the closure capacity take the overflow pass; records over the
    shared-memory budget replay from global scratch; results do not change."""
    ims, ov = planes
    N.check(N.lib().smvs_test_fusion_caps(*caps))
    try:
        got = _run(FusionOptions(), ims, ov)
    finally:
        N.check(N.lib().smvs_test_fusion_caps(0, 0, 0))
    _same(got, O.fusion_run(FusionOptions(), ims, ov))


def test_heightfield_views():
    hs = syn.heightfield_scene(seed=4, width=480, height=360, focal=360.0, num_src=3, device="cuda")
    ims, ov = syn.fusion_inputs(hs, seed=5)
    opts = FusionOptions()
    got = _run(opts, ims, ov)
    ref = O.fusion_run(opts, ims, ov)
    _same(got, ref)
    assert len(ref["points"]) > 5000


def test_profile_and_errors(planes):
    ims, ov = planes
    with StereoFusion(FusionOptions(), ims, ov) as f:
        with pytest.raises(N.SmvsError):
            f.GetFusedPoints()
        f.SetProfiling(True)
        f.Run()
        prof = f.Profile()
        assert prof["closure"][0] >= 5 and prof["replay"][0] == 5
        assert all(ms >= 0 for _, ms in prof.values())
        chains = f.DependencyChains()
        assert len(chains) == 5 and all(c >= 1 for c in chains)
        pts = f.GetFusedPoints().copy()
    # Profiling adds the chain bookkeeping to the replay; results do not change.
    assert np.array_equal(pts.view(np.uint8), O.fusion_run(FusionOptions(), ims, ov)["points"].view(np.uint8))
    with StereoFusion(FusionOptions(), ims, ov) as f:
        f.Run()
        with pytest.raises(N.SmvsError):
            f.Run()  # Run may be called once
        with pytest.raises(N.SmvsError):
            f.DependencyChains()  # recorded only with profiling


@pytest.mark.parametrize("depth", [100, 6])
def test_many_views_large_records(depth):
    """Eleven mutually overlapping views: records of a hundred pixels and more,
    where the traversal-depth limit can bind."""
    hs = syn.heightfield_scene(seed=6, width=320, height=240, focal=240.0, num_src=10, device="cuda")
    ims, ov = syn.fusion_inputs(hs, seed=7)
    opts = FusionOptions(max_traversal_depth=depth)
    _same(_run(opts, ims, ov), O.fusion_run(opts, ims, ov))
