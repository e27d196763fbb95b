"""The fusion clean-up passes of the CPU oracle, pinned by independent
restatements (no GPU).

* RemoveDuplicatePoints (fusion.cc:2184-2266): the C oracle against a
  pure-Python restatement of the same greedy loop on a cloud with many
  duplicates (points projecting to shared pixels).
* RemoveOutliers' spacing (ComputeAverageDistance, patch_match_controller.cc:
  115-228): the oracle's brute-force neighbours against scipy's k-d tree
  (a separate k-nearest-neighbour implementation), the distances added in the
  same float/double order, bit for bit; then the score histogram and the drop
  rule against a Python restatement.
"""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from oracle import oracle as O
from sensemap_b200 import _native as N
from sensemap_b200.fusion import FusionImage


def _cloud(seed, n=3000, n_img=4, dup=0.3):
    rng = np.random.default_rng(seed)
    xyz = rng.uniform([-1, -1, 4], [1, 1, 6], (n, 3)).astype(np.float32)
    k = int(n * dup)
    xyz[n - k:] = xyz[rng.integers(0, n - k, k)] + rng.normal(0, 1e-3, (k, 3)).astype(np.float32)
    pts = np.zeros(n, dtype=N.FUSED_POINT_DTYPE)
    pts["x"], pts["y"], pts["z"] = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    pts["score"] = rng.uniform(0, 1, n).astype(np.float32)
    counts = rng.integers(1, n_img + 1, n)
    off = np.zeros(n + 1, dtype=np.uint64)
    off[1:] = np.cumsum(counts)
    vis = np.concatenate([np.sort(rng.choice(n_img, c, replace=False)) for c in counts]).astype(np.uint32)
    ims = []
    for i in range(n_img):
        a = 0.1 * (i - n_img / 2)
        R = np.array([[np.cos(a), 0, -np.sin(a)], [0, 1, 0], [np.sin(a), 0, np.cos(a)]], np.float32)
        T = np.array([0.2 * i, 0, 0], np.float32)
        K = np.array([[100, 0, 80], [0, 100, 60], [0, 0, 1]], np.float32)
        ims.append(FusionImage(K=K, R=R, T=T, depth=np.ones((120, 160), np.float32)))
    return ims, pts, off, vis


def _py_duplicates(ims, pts, off, vis):
    occ = [np.full((im.depth.shape[0], im.depth.shape[1]), -1, np.int64) for im in ims]
    removal = np.zeros(len(pts), bool)
    f = np.float32
    for i in range(len(pts)):
        if removal[i]:
            continue
        X = [pts["x"][i], pts["y"][i], pts["z"][i]]
        nvis = int(off[i + 1] - off[i])
        for k in range(int(off[i]), int(off[i + 1])):
            im = ims[int(vis[k])]
            R, T, K = np.asarray(im.R, f), np.asarray(im.T, f), np.asarray(im.K, f)
            c = [f(f(f(R[r, 0] * X[0]) + f(R[r, 1] * X[1])) + f(R[r, 2] * X[2])) + T[r] for r in range(3)]
            q = [f(f(f(K[r, 0] * c[0]) + f(K[r, 1] * c[1])) + f(K[r, 2] * c[2])) for r in range(3)]
            u, v = f(q[0] / q[2]), f(q[1] / q[2])
            u = int(np.sign(u) * np.floor(abs(u) + f(0.5))) if abs(u) < 1e9 else -1
            v = int(np.sign(v) * np.floor(abs(v) + f(0.5))) if abs(v) < 1e9 else -1
            H, W = occ[int(vis[k])].shape
            if u < 0 or u >= W or v < 0 or v >= H:
                continue
            o = occ[int(vis[k])][v, u]
            if o == -1:
                occ[int(vis[k])][v, u] = i
                continue
            if int(off[o + 1] - off[o]) > nvis:
                removal[i] = True
                break
            occ[int(vis[k])][v, u] = i
            removal[o] = True
    return ~removal


def test_duplicate_removal_matches_python_restatement():
    ims, pts, off, vis = _cloud(1)
    kp, ko, kv, dropped = O.fusion_remove_duplicates(ims, pts, off, vis)
    keep = _py_duplicates(ims, pts, off, vis)
    assert dropped == int((~keep).sum()) and dropped > 100
    assert np.array_equal(kp.view(np.uint8), pts[keep].view(np.uint8))
    assert np.array_equal(np.diff(ko.astype(np.int64)), np.diff(off.astype(np.int64))[keep])


@pytest.mark.parametrize("nb", [1, 6, 12])
def test_outlier_spacing_matches_kdtree(nb):
    _, pts, off, vis = _cloud(2, n=4000)
    *_, spacing = O.fusion_remove_outliers(pts, off, vis, nb_neighbors=nb)
    xyz = np.stack([pts["x"], pts["y"], pts["z"]], 1).astype(np.float64)
    # The k-d tree gives the neighbour sets; each neighbour's squared distance
    # is recomputed the oracle's way before the float sum.
    _, idx = cKDTree(xyz).query(xyz, k=nb + 1)
    diff = xyz[:, None, :] - xyz[idx]
    d2 = (diff[..., 0] * diff[..., 0] + diff[..., 1] * diff[..., 1]) + diff[..., 2] * diff[..., 2]
    d2 = np.sort(d2, axis=1)
    expect = np.zeros(len(pts), np.float32)
    for k in range(nb + 1):
        expect = (expect.astype(np.float64) + np.sqrt(d2[:, k])).astype(np.float32)
    expect = (expect / np.float32(nb)).astype(np.float32)
    assert np.array_equal(spacing.view(np.uint32), expect.view(np.uint32))


def test_outlier_drop_rule_matches_python_restatement():
    _, pts, off, vis = _cloud(3, n=3000)
    # A handful of far-away points: large spacings push their scores up.
    pts["x"][:15] += np.float32(50)
    kp, ko, kv, dropped, spacing = O.fusion_remove_outliers(pts, off, vis, nb_neighbors=6, max_spacing_factor=6.0)
    avg = np.float32(0)
    for v in spacing:
        avg = np.float32(avg + v)
    avg = np.float32(avg / np.float32(len(spacing)))
    factor = (spacing.astype(np.float64) / (6.0 * np.float64(avg))).astype(np.float32)
    scores = (pts["score"].astype(np.float64) * 0.6 + factor.astype(np.float64) * 0.4).astype(np.float32)
    smin, smax = scores.min(), scores.max()
    rng_ = np.float32(smax - smin)
    bins = (((scores - smin) / rng_).astype(np.float32) * np.float32(255)).astype(np.int64)
    ratios = np.zeros(256, np.float32)
    for b in bins:
        ratios[b] = np.float32(ratios[b] + np.float32(1))
    ratios = (ratios / np.float32(len(scores))).astype(np.float32)
    acc = np.zeros(256, np.float32)
    s = np.float32(0)
    for k in range(256):
        s = np.float32(s + ratios[k])
        acc[k] = s
    keep = ~((ratios[bins].astype(np.float64) < 0.01) & (acc[bins].astype(np.float64) >= 0.9))
    assert dropped == int((~keep).sum()) and dropped >= 15
    assert np.array_equal(kp["score"].view(np.uint32), scores[keep].view(np.uint32))
