"""CPU checks of the cross-view filter's oracle and host-side pieces.

The oracle (oracle/smvs_oracle_filter.c) restates CrossFilterKernel /
DeduplicFilterKernel (kernel_functions.cu:3561-3916) and CrossFilterCuda's
host flow (patch_match_cuda.cu:1493-1625); it is pinned against the
reference's own kernels by tests/golden/ref_crossfilter_planes.npz (see
test_golden.py) and, on a GPU, by test_cross_filter_gpu.py.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from sensemap_b200 import _native as N
from sensemap_b200.patch_match import PatchMatchOptions
from tests.helpers import filter_set


def _product_encode(normal):
    n = np.ascontiguousarray(normal, np.float32)
    out = np.zeros(n.shape[1:], np.uint32)
    N.check(N.lib().smvs_encode_normal_map(n.ctypes.data, n.shape[2], n.shape[1], out.ctypes.data))
    return out


def test_encode_matches_oracle_bit_exact():
    rng = np.random.default_rng(0)
    n = rng.standard_normal((3, 37, 53)).astype(np.float32)
    n /= np.linalg.norm(n, axis=0, keepdims=True)
    # edge cases: the poles, n0 = -1 (NaN inside Encode, clamps to +0.999999), axis-aligned
    n[:, 0, 0] = (-1, 0, 0)
    n[:, 0, 1] = (1, 0, 0)
    n[:, 0, 2] = (0, 1, 0)
    n[:, 0, 3] = (0, 0, -1)
    n[:, 0, 4] = (0, -1, 0)
    a, b = _product_encode(n), O.encode_normal_map(n)
    assert np.array_equal(a, b)
    # (-1, 0, 0): s = 1, m = inf, q = 0 * inf = NaN -> std::min(0.999999, NaN) = 0.999999
    iq = int((np.float32(0.999999) + np.float32(1)) * np.float32(32767))
    assert a[0, 0] == (iq << 16) | iq


def test_oracle_run_properties():
    scene, views, problems = filter_set(seed=3)
    opt = PatchMatchOptions()
    refined = O.cross_filter_run(opt, views, problems)
    assert sorted(refined) == list(range(len(views)))
    for r, d in refined.items():
        H, W = d.shape
        # CrossFilterKernel zeroes the 3-pixel border (col < 3 || col > W - 3, :3580-3584)
        assert not d[:3].any() and not d[:, :3].any() and not d[H - 2:].any() and not d[:, W - 2:].any()
        assert not d[views[r].depth < 1e-6].any()
        gt = scene.views[r].depth_gt
        m = d > 0
        assert m.mean() > 0.5
        # kept depths are consistent with the truth far more often than the input
        assert np.mean(np.abs(d[m] - gt[m]) <= 0.01 * gt[m]) > 0.995


def test_oracle_run_median_rule():
    """One consistent source: the sorted prefix is the reference depth alone, so
    the output is the input depth itself (BubbleSort over `good` of good + 1
    entries, kernel_functions.cu:3763-3767)."""
    scene, views, problems = filter_set(seed=5, n_views=2, rel_noise=0.0, outlier_frac=0.0, hole_frac=0.0)
    opt = PatchMatchOptions()
    refined = O.cross_filter_run(opt, views, problems)
    for r, d in refined.items():
        m = d > 0
        assert m.mean() > 0.3
        assert np.array_equal(d[m], views[r].depth[m])


def test_oracle_dedup_properties():
    scene, views, problems = filter_set(seed=4)
    opt = PatchMatchOptions()
    refined = O.cross_filter_run(opt, views, problems)
    vis, delta = O.cross_filter_dedup(opt, views, problems, refined)
    for r in range(len(views)):
        keep = (vis[r] & 0x80000000) != 0
        # a kept pixel has a non-zero dedup input and a non-negative delta
        assert (refined[r][keep] > 0).all()
        assert (delta[r] >= 0).all()
        assert not delta[r][~keep].any()
        dd = O.cross_filter_dedup_depth(views[r], refined[r], vis[r])
        assert np.array_equal(dd, np.where(keep, refined[r], 0))
    # the last problem sees every other view already deduplicated: it keeps most of its pixels
    assert ((vis[-1] & 0x80000000) != 0).mean() > ((vis[0] & 0x80000000) != 0).mean()


def test_oracle_rejects_bad_sets():
    scene, views, problems = filter_set(seed=1, n_views=3)
    opt = PatchMatchOptions()
    with pytest.raises(RuntimeError):
        O.cross_filter_run(opt, views, [(0, [0, 1])])  # a view is its own source
    with pytest.raises(RuntimeError):
        O.cross_filter_run(opt, views, [(0, [5])])  # out of range
    opt0 = PatchMatchOptions(filter_min_num_consistent=0)
    refined = O.cross_filter_run(opt0, views, problems)
    with pytest.raises(RuntimeError):
        O.cross_filter_dedup(opt0, views, problems, refined)


def test_cross_filter_abi_declared():
    lib = N.lib()
    for name in ("smvs_cross_filter_create", "smvs_cross_filter_run", "smvs_cross_filter_dedup_run",
                 "smvs_cross_filter_get_refined_depth_map", "smvs_cross_filter_get_dedup_depth_map",
                 "smvs_cross_filter_get_delta_depth_map", "smvs_cross_filter_get_visibility_map",
                 "smvs_cross_filter_get_device_maps", "smvs_cross_filter_launch_count",
                 "smvs_cross_filter_dedup_levels", "smvs_cross_filter_synchronize", "smvs_cross_filter_destroy"):
        assert hasattr(lib, name)
    # argument checks run before any device work
    o = N.smvs_options()
    lib.smvs_options_default(C.byref(o))
    h = C.c_void_p()
    assert lib.smvs_cross_filter_create(C.byref(o), None, 0, None, 0, N.MEM_HOST, None, C.byref(h)) == N.SMVS_EINVAL
    v = (N.smvs_filter_view * 2)()
    d = np.zeros((4, 4), np.float32)
    for k in range(2):
        v[k].width = v[k].height = 4
        v[k].depth = d.ctypes.data
    src = (C.c_int * 1)(0)
    p = (N.smvs_filter_problem * 2)()
    p[0].ref, p[0].src, p[0].num_src = 1, C.cast(src, C.POINTER(C.c_int)), 1
    p[1].ref, p[1].src, p[1].num_src = 1, C.cast(src, C.POINTER(C.c_int)), 1
    assert lib.smvs_cross_filter_create(C.byref(o), v, 2, p, 2, N.MEM_HOST, None, C.byref(h)) == N.SMVS_EINVAL
    assert b"share reference view" in lib.smvs_last_error()
    p[0].num_src = 32
    assert lib.smvs_cross_filter_create(C.byref(o), v, 2, p, 1, N.MEM_HOST, None, C.byref(h)) == N.SMVS_EINVAL


def test_decode_short_form_is_exact_for_every_code():
    """The CUDA filter decodes normal codes with (float)((double)iq * (1/32767))
    and 1 - 2s in float; both equal the reference's expressions
    ((float)iq / 32767.f and (float)(1.0 - 2.0 * s)) for every input it sees."""
    iq = np.arange(65536, dtype=np.float32)
    assert np.array_equal(iq / np.float32(32767), (iq.astype(np.float64) * (1.0 / 32767.0)).astype(np.float32))
    q = (iq / np.float32(32767) - np.float32(1)).astype(np.float32)
    rng = np.random.default_rng(0)
    q1, q2 = rng.choice(q, 2_000_000), rng.choice(q, 2_000_000)
    s = (q1 * q1 + q2 * q2).astype(np.float32)  # any float s in [0, 2]
    assert np.array_equal((1.0 - 2.0 * s.astype(np.float64)).astype(np.float32), np.float32(1) - np.float32(2) * s)


def test_float_forms_of_the_double_thresholds():
    """The CUDA filter tests depth <= 1e-6f and src_depth <= 1e-4f where the
    reference writes depth < 1e-6 and src_depth < 1e-4 with double constants:
    the same answer for every float around the thresholds and the specials."""
    for thr in (1e-4, 1e-6):
        lo, hi = np.float32(thr / 2).view(np.int32), np.float32(thr * 2).view(np.int32)
        xs = np.arange(lo, hi, dtype=np.int32).view(np.float32)
        xs = np.concatenate([xs, -xs, np.array([0, -0.0, np.inf, -np.inf, np.nan, 1.0, 3e-38], np.float32)])
        assert np.array_equal(xs.astype(np.float64) < thr, xs <= np.float32(thr))
