"""The Delaunay triangulation behind the Delaunay initial map (host code of
libsmvs.so, no GPU), and the oracle's raster of it.

The triangulation is pinned against scipy's Qhull triangulation (an
independent implementation): on point sets whose Delaunay triangulation is
unique (no four co-circular points) the triangle sets must be equal; on integer
grids with co-circular points every triangle must still have an empty
circumcircle and the triangles must tile the convex hull. The oracle's raster
of a plane's points must give that plane's depth and normal.
"""
import numpy as np
import pytest
from scipy.spatial import ConvexHull, Delaunay

from oracle import oracle as O
from sensemap_b200.init_maps import delaunay_triangles


def _sets(t):
    return {tuple(sorted(r)) for r in np.asarray(t).tolist()}


def _first_unique(xy):
    _, idx = np.unique(xy, axis=0, return_index=True)
    return np.sort(idx)


def _incircle(a, b, c, d):
    m = [[a[0] - d[0], a[1] - d[1], (a[0] - d[0]) ** 2 + (a[1] - d[1]) ** 2],
         [b[0] - d[0], b[1] - d[1], (b[0] - d[0]) ** 2 + (b[1] - d[1]) ** 2],
         [c[0] - d[0], c[1] - d[1], (c[0] - d[0]) ** 2 + (c[1] - d[1]) ** 2]]
    return (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
            m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]))


@pytest.mark.parametrize("seed", range(6))
def test_equals_qhull_in_general_position(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 3000))
    xy = np.stack([rng.integers(0, 1 << 20, n), rng.integers(0, 1 << 20, n)], 1)
    xy[rng.integers(0, n, n // 10)] = xy[rng.integers(0, n, n // 10)]  # repeated positions
    keep = _first_unique(xy)
    ref = _sets(keep[Delaunay(xy[keep].astype(np.float64)).simplices])
    got = delaunay_triangles(xy)
    assert _sets(got) == ref
    # counter-clockwise, and no repeated position is a vertex
    p = xy.astype(np.int64)
    a, b, c = p[got[:, 0]], p[got[:, 1]], p[got[:, 2]]
    assert np.all((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0]) > 0)
    assert set(np.unique(got)).issubset(set(keep.tolist()))


def test_integer_grid_with_cocircular_points_is_delaunay():
    rng = np.random.default_rng(7)
    xy = np.stack([rng.integers(0, 40, 600), rng.integers(0, 30, 600)], 1)
    got = delaunay_triangles(xy)
    pts = [tuple(int(v) for v in q) for q in xy[_first_unique(xy)]]
    P = [tuple(int(v) for v in q) for q in xy]
    for t in got.tolist():
        for q in pts:
            assert _incircle(P[t[0]], P[t[1]], P[t[2]], q) <= 0
    area = 0.0
    for t in got.tolist():
        (ax, ay), (bx, by), (cx, cy) = P[t[0]], P[t[1]], P[t[2]]
        area += 0.5 * ((bx - ax) * (cy - ay) - (by - ay) * (cx - ax))
    assert area == pytest.approx(ConvexHull(np.array(pts, float)).volume)


def test_degenerate_inputs():
    assert len(delaunay_triangles(np.zeros((0, 2), np.int32))) == 0
    assert len(delaunay_triangles([[0, 0], [5, 5], [10, 10], [3, 3]])) == 0  # collinear
    assert len(delaunay_triangles([[1, 1], [1, 1], [1, 1]])) == 0
    t = delaunay_triangles([[0, 0], [0, 0], [4, 0], [0, 3]])
    assert _sets(t) == {(0, 2, 3)}


def test_oracle_raster_of_a_plane():
    # Points on the plane z = 5 + 0.1 x seen by a camera at the origin.
    rng = np.random.default_rng(3)
    W, H = 160, 120
    K = np.array([[120.0, 0, 80], [0, 120.0, 60], [0, 0, 1]])
    R, T = np.eye(3), np.zeros(3)
    u = rng.uniform(0, W, 400)
    v = rng.uniform(0, H, 400)
    ray = np.stack([(u - 80) / 120, (v - 60) / 120, np.ones_like(u)], 1)
    z = 5.0 / (1 - 0.1 * ray[:, 0])
    xyz = (ray * z[:, None]).astype(np.float32)
    uv, zz, _ = O.delaunay_points(W, H, K, R, T, xyz)
    tris = delaunay_triangles(uv)
    d, n, rng_ = O.init_from_delaunay(W, H, K, R, T, xyz, tris)
    covered = d > 0
    assert covered.mean() > 0.8
    ys, xs = np.nonzero(covered)
    rx = (xs - 80) / 120.0
    gt = 5.0 / (1 - 0.1 * rx)
    assert np.max(np.abs(d[covered] - gt) / gt) < 2e-2
    nz = n[:, covered]
    expect = np.array([-0.1, 0, 1]) / np.linalg.norm([-0.1, 0, 1])
    cos = np.abs(expect @ nz)
    assert np.quantile(cos, 0.05) > np.cos(np.radians(10))
    assert rng_[0] == pytest.approx(1e-6) and rng_[1] == pytest.approx(float(zz.max()) * 1.1, rel=1e-6)
