"""GPU parity of the cross-view filter (smvs_cross_filter_* through the C ABI).

The CUDA unit (sensemap_b200/csrc/smvs_cross_filter.cu) and the CPU oracle
(oracle/smvs_oracle_filter.c) perform the same IEEE single-precision
operations in the same order, so refined maps, visibility layers, delta maps
and deduplicated maps must match bit for bit. The reference's own kernels
(CrossFilterKernel / DeduplicFilterKernel, built into oracle/_ref) are built
with --use_fast_math and read maps through textures: against them the test
asks for the same decision on nearly every pixel.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sensemap_b200 import _native as N
from sensemap_b200.cross_filter import CrossFilterCuda
from sensemap_b200.patch_match import PatchMatchOptions
from tests.helpers import filter_api_inputs, filter_set

pytestmark = pytest.mark.gpu


def _gpu_run(opt, views, problems, device=False, dedup=True):
    probs, ids, flags = filter_api_inputs(views, problems, device=device)
    cf = CrossFilterCuda(opt, probs, ids, flags)
    cf.Run()
    out = {"refined": {r: cf.GetRefineDepthMap(r) for r, s in problems if s}}
    if dedup:
        cf.DedupRun()
        out["vis"] = [cf.GetVisibilyMap(k) for k in range(len(views))]
        out["delta"] = {r: cf.GetDeltDepthMap(r) for r, s in problems if s}
        out["dedup"] = [cf.GetDeduplicDepthMap(k) for k in range(len(views))]
        out["levels"] = cf.DedupLevels()
    out["launches"] = cf.LaunchCount()
    cf.close()
    return out


def _oracle(opt, views, problems):
    refined = O.cross_filter_run(opt, views, problems)
    vis, delta = O.cross_filter_dedup(opt, views, problems, refined)
    dd = [O.cross_filter_dedup_depth(v, refined.get(k), vis[k]) for k, v in enumerate(views)]
    return refined, vis, delta, dd


def _assert_same(got, views, refined, vis, delta, dd):
    for r, m in refined.items():
        assert np.array_equal(got["refined"][r], m), f"refined map of view {r} differs"
    for k in range(len(views)):
        assert np.array_equal(got["vis"][k], vis[k]), f"visibility of view {k} differs"
        assert np.array_equal(got["dedup"][k], dd[k]), f"dedup depth of view {k} differs"
    for r, m in delta.items():
        assert np.array_equal(got["delta"][r], m), f"delta map of view {r} differs"


@pytest.mark.parametrize("seed", [0, 7])
def test_cross_filter_bit_exact_vs_oracle(seed):
    scene, views, problems = filter_set(seed=seed, w=200, h=150, n_views=7)
    opt = PatchMatchOptions()
    got = _gpu_run(opt, views, problems)
    _assert_same(got, views, *_oracle(opt, views, problems))
    assert all((got["refined"][r] > 0).mean() > 0.5 for r in got["refined"])


def test_cross_filter_options_bit_exact():
    scene, views, problems = filter_set(seed=2, n_views=6, outlier_frac=0.1, normal_noise_deg=8.0)
    opt = PatchMatchOptions(filter_min_num_consistent=3, filter_geom_consistency_max_cost=0.5, max_normal_error=8.0,
                            depth_diff_threshold=0.01)
    got = _gpu_run(opt, views, problems)
    _assert_same(got, views, *_oracle(opt, views, problems))


def test_cross_filter_device_inputs_match_host():
    scene, views, problems = filter_set(seed=11, n_views=5)
    opt = PatchMatchOptions()
    host = _gpu_run(opt, views, problems)
    dev = _gpu_run(opt, views, problems, device=True)
    for r in host["refined"]:
        assert np.array_equal(host["refined"][r], dev["refined"][r])
    for k in range(len(views)):
        assert np.array_equal(host["vis"][k], dev["vis"][k])


def test_cross_filter_ragged_set():
    """Views of different sizes, a problem without sources, a view that is in
    no problem, and a ref_flag view that nothing refined (its dedup input is
    all zero)."""
    from oracle.oracle import FilterView
    from sensemap_b200 import synthetic as syn
    scene = syn.planes_scene(seed=9, width=150, height=110, focal=120.0, num_src=5)
    maps = syn.noisy_maps(scene, seed=1)
    views = []
    for k, (v, (d, n)) in enumerate(zip(scene.views, maps)):
        if k == 2:  # a smaller view with its own intrinsics: crop the top-left corner
            d, n = d[:80, :120], n[:, :80, :120]
        views.append(FilterView(v.K, v.R, v.T, d, n, ref_flag=k != 4))
    problems = [(0, [1, 2, 3]), (1, [0, 2, 3, 4]), (2, []), (3, [2, 4]), (5, [0, 1, 3, 4])]
    # view 4 is a source only (ref_flag False); view 2's problem has no source and is
    # skipped, so view 2 (ref_flag True) has no refined map and its dedup input is zero
    opt = PatchMatchOptions()
    got = _gpu_run(opt, views, problems)
    refined, vis, delta, dd = _oracle(opt, views, problems)
    assert sorted(got["refined"]) == sorted(refined) == [0, 1, 3, 5]
    _assert_same(got, views, refined, vis, delta, dd)
    assert not dd[2].any()


def test_cross_filter_max_sources():
    scene, views, problems = filter_set(seed=6, w=64, h=48, f=50.0, n_views=32, hole_frac=0.0)
    opt = PatchMatchOptions()
    # view 0 against all 31 others; the rest against three neighbours each
    problems = [(0, list(range(1, 32)))] + [(r, [(r + 1) % 32, (r + 2) % 32, (r + 3) % 32]) for r in range(1, 32)]
    got = _gpu_run(opt, views, problems)
    _assert_same(got, views, *_oracle(opt, views, problems))
    probs, ids, flags = filter_api_inputs(views, [(0, list(range(1, 32)))])
    probs[0].src_image_extend_idxs = list(range(1, 32)) + [1]  # 32 sources
    with pytest.raises(N.SmvsError):
        CrossFilterCuda(opt, probs, ids, flags)


def test_dedup_levels_keep_problem_order():
    """Problems that touch a common visibility layer run in the reference's
    order, in separate passes; the others share a pass."""
    scene, views, problems = filter_set(seed=8, n_views=6)
    opt = PatchMatchOptions()
    independent = [(0, [3]), (1, [4]), (2, [5])]  # no reference is another problem's source
    got = _gpu_run(opt, views, independent)
    _assert_same(got, views, *_oracle(opt, views, independent))
    assert got["levels"] == 1
    chain = [(r, [r + 1]) for r in range(5)]  # problem r reads layer r+1 before problem r+1 writes it
    got = _gpu_run(opt, views, chain)
    _assert_same(got, views, *_oracle(opt, views, chain))
    assert got["levels"] == 5
    back = [(r, [r - 1]) for r in range(1, 6)]  # each reads the layer the previous problem wrote
    got = _gpu_run(opt, views, back)
    _assert_same(got, views, *_oracle(opt, views, back))
    assert got["levels"] == 5
    pairs = [(0, [1]), (2, [3]), (4, [5]), (1, [0]), (3, [2]), (5, [4])]
    got = _gpu_run(opt, views, pairs)
    _assert_same(got, views, *_oracle(opt, views, pairs))
    assert got["levels"] == 2


def test_cross_filter_state_errors():
    scene, views, problems = filter_set(seed=1, n_views=3)
    opt = PatchMatchOptions()
    probs, ids, flags = filter_api_inputs(views, problems)
    cf = CrossFilterCuda(opt, probs, ids, flags)
    with pytest.raises(N.SmvsError):
        cf.GetRefineDepthMap(0)  # before Run
    with pytest.raises(N.SmvsError):
        cf.GetVisibilyMap(0)  # before DedupRun
    cf.Run()
    cf.GetRefineDepthMap(0)
    with pytest.raises(N.SmvsError):
        cf.GetDeltDepthMap(0)
    cf.close()
    opt0 = PatchMatchOptions(filter_min_num_consistent=0)
    cf = CrossFilterCuda(opt0, probs, ids, flags)
    cf.Run()
    with pytest.raises(N.SmvsError):
        cf.DedupRun()
    cf.close()


def test_cross_filter_vs_reference_kernels():
    """Same decisions as the reference's CrossFilterKernel / DeduplicFilterKernel
    on nearly every pixel (the reference uses fast-math and texture fetches)."""
    from oracle import ref_oracle as R
    if not R.available():
        pytest.skip("reference kernels not built (oracle/ref_build.py)")
    scene, views, problems = filter_set(seed=12, w=200, h=150, n_views=6)
    opt = PatchMatchOptions()
    got = _gpu_run(opt, views, problems)
    ref_refined = R.cross_filter(opt, views, problems)
    for r, m in ref_refined.items():
        g = got["refined"][r]
        same_decision = np.mean((g > 0) == (m > 0))
        both = (g > 0) & (m > 0)
        close = np.mean(np.abs(g[both] - m[both]) <= 1e-5 * m[both])
        assert same_decision > 0.995 and close > 0.995, (r, same_decision, close)
    # dedup on the reference's own refined maps, against the oracle on the same maps
    ref_vis, ref_delta = R.dedup(opt, views, problems, ref_refined)
    vis, delta = O.cross_filter_dedup(opt, views, problems, ref_refined)
    for k in range(len(views)):
        assert np.mean(ref_vis[k] == vis[k]) > 0.995
    for r in ref_delta:
        keep = (ref_vis[r] & 0x80000000) != 0
        if not keep.any():  # e.g. the first problem: every consistent pixel is still kept by a later view
            continue
        assert np.mean(np.abs(ref_delta[r][keep] - delta[r][keep]) <= 1e-4 + 1e-4 * np.abs(delta[r][keep])) > 0.99


def test_cross_filter_pool_reuse_and_release():
    """Filters allocate from a stream-ordered pool: a second filter on the same
    set reuses the freed blocks and gives the same maps; the cache can be
    returned to the device."""
    scene, views, problems = filter_set(seed=13, n_views=4)
    opt = PatchMatchOptions()
    a = _gpu_run(opt, views, problems)
    b = _gpu_run(opt, views, problems)
    for r in a["refined"]:
        assert np.array_equal(a["refined"][r], b["refined"][r])
    assert N.lib().smvs_cross_filter_release_cache(-1) == N.SMVS_OK
    c = _gpu_run(opt, views, problems)
    for k in range(len(views)):
        assert np.array_equal(a["vis"][k], c["vis"][k])
