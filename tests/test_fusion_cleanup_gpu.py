"""GPU parity of the fusion clean-up passes against the C oracle.

The fused cloud of the GPU image loop is cleaned on the GPU
(smvs_fusion_remove_duplicate_points, smvs_fusion_remove_outliers) and, from
the same cloud, by the oracle (oracle/smvs_oracle_fusion.c: the greedy
duplicate loop of RemoveDuplicatePoints and RemoveOutliers with brute-force
neighbours). Kept points (every field, bit for bit, scores included), their
images and the counts dropped must be identical.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sensemap_b200 import synthetic as syn
from sensemap_b200.fusion import FusionOptions, StereoFusion

pytestmark = pytest.mark.gpu


def _cloud(f):
    pts = f.GetFusedPoints().copy()
    off, vis = f.VisibilityCSR()
    return pts, off.copy(), vis.copy()


def _same_cloud(a, b):
    assert len(a[0]) == len(b[0]), (len(a[0]), len(b[0]))
    assert np.array_equal(a[0].view(np.uint8), b[0].view(np.uint8))
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])


@pytest.mark.parametrize("scene_kind", ["planes", "heightfield"])
def test_cleanup_matches_oracle(scene_kind):
    if scene_kind == "planes":
        scene = syn.planes_scene(seed=3, width=200, height=150, focal=160.0, num_src=4)
    else:
        scene = syn.heightfield_scene(seed=2, width=320, height=240, focal=240.0, num_src=5)
    ims, ov = syn.fusion_inputs(scene, seed=1)
    with StereoFusion(FusionOptions(), ims, ov) as f:
        f.Run()
        fused = _cloud(f)
        dropped = f.RemoveDuplicatePoints()
        dedup = _cloud(f)
        kp, ko, kv, o_dropped = O.fusion_remove_duplicates(ims, *fused)
        assert dropped == o_dropped
        _same_cloud(dedup, (kp, ko, kv))
        removed = f.RemoveOutliers(nb_neighbors=6, max_spacing_factor=6.0)
        clean = _cloud(f)
        rp, ro, rv, o_removed, _ = O.fusion_remove_outliers(*dedup, nb_neighbors=6, max_spacing_factor=6.0)
        assert removed == o_removed
        _same_cloud(clean, (rp, ro, rv))
    assert len(fused[0]) > 500


def test_outlier_pass_with_far_points_and_other_neighbour_counts():
    scene = syn.planes_scene(seed=5, width=160, height=120, focal=128.0, num_src=4)
    ims, ov = syn.fusion_inputs(scene, seed=3)
    for nb in (1, 12):
        with StereoFusion(FusionOptions(), ims, ov) as f:
            f.Run()
            before = _cloud(f)
            removed = f.RemoveOutliers(nb_neighbors=nb, max_spacing_factor=3.0)
            after = _cloud(f)
        rp, ro, rv, o_removed, _ = O.fusion_remove_outliers(*before, nb_neighbors=nb, max_spacing_factor=3.0)
        assert removed == o_removed
        _same_cloud(after, (rp, ro, rv))
