"""Source-view selection and depth ranges (host code; no GPU) against the
pure-Python restatement in oracle/view_selection_oracle.py
(Model::GetMaxOverlappingImages / ComputeDepthRanges, src/mvs/model.cc)."""
import numpy as np
import pytest

from oracle import view_selection_oracle as VO
from sensemap_b200 import synthetic as syn
from sensemap_b200 import view_selection as VS


@pytest.fixture(scope="module")
def model():
    return syn.ring_model(num_cameras=24, num_points=1500, seed=1)


@pytest.mark.parametrize("max_num, min_angle", [(10, 1.0), (5, 3.0), (20, 0.0), (3, 30.0)])
def test_select_views_matches_oracle(model, max_num, min_angle):
    Rs, Ts, K, P, tracks, rig = model
    got = VS.get_max_overlapping_images(Rs, Ts, P, tracks, max_num, min_angle, is_rig=rig)
    ref = VO.get_max_overlapping_images(Rs, Ts, P, tracks, max_num, min_angle, is_rig=rig)
    assert got == ref
    assert all(len(g) <= max_num for g in got)
    assert any(len(g) for g in got)


def test_select_views_candidates_and_spatial_fallback(model):
    Rs, Ts, K, P, tracks, rig = model
    # images 0..3 observe nothing: they fall back to spatial neighbours
    tracks2 = [[c for c in t if c > 3] for t in tracks]
    unique = list(range(0, 24, 2))
    got = VS.get_max_overlapping_images(Rs, Ts, P, tracks2, 6, 1.0, unique_image_idxs=unique, is_rig=rig)
    ref = VO.get_max_overlapping_images(Rs, Ts, P, tracks2, 6, 1.0, unique_image_idxs=unique, is_rig=rig)
    assert got == ref
    assert all(got[i] == [] for i in range(24) if i not in unique)
    assert got[0] and got[2]  # spatial neighbours of images without points
    # shared-point neighbours only come from the candidate set
    for i in unique:
        if i > 3:
            assert set(got[i]) <= set(unique)


def test_select_views_ties_keep_image_order():
    """Two sources sharing the same number of points with the reference: the
    lower image index comes first."""
    Rs, Ts, K, P, tracks, rig = syn.ring_model(num_cameras=6, num_points=0, seed=2)
    pts = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], np.float32)
    tracks = [[0, 4, 2], [0, 2, 4], [0, 4, 2, 1]]
    got = VS.get_max_overlapping_images(Rs, Ts, pts, tracks, 10, 0.0)
    assert got == VO.get_max_overlapping_images(Rs, Ts, pts, tracks, 10, 0.0)
    assert got[0][:2] == [2, 4]


def test_depth_ranges_match_oracle(model):
    Rs, Ts, K, P, tracks, rig = model
    lt, rb = P.min(0) - 1, P.max(0) + 1
    got = VS.compute_depth_ranges(Rs, Ts, lt, rb)
    assert np.array_equal(got, VO.compute_depth_ranges(Rs, Ts, lt, rb))
    assert (got[:, 0] >= np.float32(1e-6)).all() and (got[:, 1] > got[:, 0]).all()


def test_select_views_rejects_bad_tracks(model):
    Rs, Ts, K, P, tracks, rig = model
    bad = [list(t) for t in tracks]
    bad[0] = [99]
    with pytest.raises(Exception):
        VS.get_max_overlapping_images(Rs, Ts, P, bad, 5, 1.0)
