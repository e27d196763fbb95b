"""Pure-Python restatement of the source-view selection (test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker of smvs_select_views /
smvs_compute_depth_ranges (sensemap_b200/csrc/smvs_view_select.cpp). Follows
Model::GetMaxOverlappingImages (src/mvs/model.cc:701-935),
ComputeSharedPoints (:961-999), CalculateTriangulationAngle
(src/base/triangulation.cc:203-224), Percentile (src/util/math.h:260-275) and
ComputeDepthRanges / ComputeDepthRangeFromBBox (model.cc:23-36, 941-959),
line by line in Python loops: single-precision steps use numpy.float32
scalars and the C library's acosf, double-precision ones Python floats. Ties
between equal scores keep ascending image order (the reference leaves them
unspecified).
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math

import numpy as np

f32 = np.float32
_LIBM = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_LIBM.acosf.restype = ctypes.c_float
_LIBM.acosf.argtypes = [ctypes.c_float]
DEG2RAD = 0.0174532925199432954743716805978692718781530857086181640625


def _center(R, T):
    R = [f32(a) for a in np.asarray(R, np.float64).reshape(9)]
    T = [f32(a) for a in np.asarray(T, np.float64).reshape(3)]
    return [float(-(R[r] * T[0] + R[3 + r] * T[1] + R[6 + r] * T[2])) for r in range(3)]


def _sqnorm(a, b):
    d = [a[0] - b[0], a[1] - b[1], a[2] - b[2]]
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2]


def _tri_angle(c1, c2, p):
    base = _sqnorm(c1, c2)
    r1, r2 = _sqnorm(p, c1), _sqnorm(p, c2)
    den = 2.0 * math.sqrt(r1 * r2)
    if den == 0.0:
        return 0.0
    angle = abs(math.acos((r1 + r2 - base) / den))
    return min(angle, math.pi - angle)


def _percentile(vals, p):
    idx = int(math.floor(p / 100 * (len(vals) - 1) + 0.5))  # std::round of a non-negative value
    idx = max(0, min(len(vals) - 1, idx))
    return sorted(vals)[idx]


def get_max_overlapping_images(Rs, Ts, points, tracks, max_num_images, min_triangulation_angle,
                               unique_image_idxs=None, is_rig=None):
    n = len(Rs)
    unique = set(range(n)) if unique_image_idxs is None else set(unique_image_idxs)
    rig = [False] * n if is_rig is None else [bool(r) for r in is_rig]
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    image_points = [[] for _ in range(n)]
    for i, tr in enumerate(tracks):
        for im in tr:
            image_points[im].append(i)
    C = [_center(Rs[i], Ts[i]) for i in range(n)]
    shared = [dict() for _ in range(n)]
    for tr in tracks:
        for a in range(len(tr)):
            for b in range(a):
                if tr[a] != tr[b]:
                    shared[tr[a]][tr[b]] = shared[tr[a]].get(tr[b], 0) + 1
                    shared[tr[b]][tr[a]] = shared[tr[b]].get(tr[a], 0) + 1
    m_dist, m_cnt = f32(0), 0
    for i in range(n):
        md = f32(np.finfo(np.float32).max)
        for j in shared[i]:
            d = f32(math.sqrt(_sqnorm(C[i], C[j])))
            if d <= 1e-5:
                continue
            md = min(d, md)
        if md < np.finfo(np.float32).max:
            m_dist = f32(m_dist + md)
            m_cnt += 1
    m_dist = f32(m_dist / f32(m_cnt)) if m_cnt else f32("nan")
    min_dist, max_dist = f32(0.1 * float(m_dist)), f32(100 * float(m_dist))
    min_angle, max_angle = f32(0.0 * DEG2RAD), f32(60.0 * DEG2RAD)
    min_tri = f32(min_triangulation_angle * DEG2RAD)
    out = [[] for _ in range(n)]

    def neighbours(i1):
        if not image_points[i1]:
            return False
        count, angles = {}, {}
        for pi in image_points[i1]:
            X = [float(pts[pi, 0]), float(pts[pi, 1]), float(pts[pi, 2])]
            for i2 in tracks[pi]:
                if i2 not in unique or i2 == i1:
                    continue
                count[i2] = count.get(i2, 0) + 1
                angles.setdefault(i2, []).append(f32(_tri_angle(C[i1], C[i2], X)))
        ordered = []
        for i2 in sorted(count):
            if _percentile(angles[i2], 75) >= min_tri:
                factor = 1.5 if rig[i2] == rig[i1] else 1.0
                ordered.append((i2, int(count[i2] * factor)))
        ordered.sort(key=lambda e: -e[1])  # stable: ties keep ascending image order
        out[i1] = [e[0] for e in ordered[:min(len(ordered), max_num_images)]]
        return True

    def spatial(i1):
        r1 = [f32(a) for a in np.asarray(Rs[i1], np.float64).reshape(9)[6:9]]
        scores = []
        for i in range(n):
            if i == i1:
                continue
            r2 = [f32(a) for a in np.asarray(Rs[i], np.float64).reshape(9)[6:9]]
            dist = f32(math.sqrt(_sqnorm(C[i], C[i1])))
            if dist < min_dist or dist > max_dist:
                continue
            cos_angle = f32(r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2])
            angle = f32(_LIBM.acosf(float(cos_angle)))
            if angle < min_angle or angle > max_angle:
                continue
            wangle = f32(f32(1.1) - cos_angle)
            wdist = max(f32(dist / m_dist), f32(1.0))
            scores.append((i, f32(wangle * wdist)))
        scores.sort(key=lambda e: e[1])
        eff = min(len(scores), max_num_images)
        if eff < 1:
            return
        sel = [i1]
        while len(sel) <= eff and scores:
            for k, (nxt, _) in enumerate(scores):
                if all(math.sqrt(_sqnorm(C[nxt], C[o])) >= min_dist for o in sel):
                    sel.append(nxt)
                    del scores[k]
                    break
            else:
                break
        out[i1] = sel[1:]

    for i in range(n):
        if i in unique and not neighbours(i):
            spatial(i)
    return out


def compute_depth_ranges(Rs, Ts, lt, rb):
    lt = [f32(a) for a in lt]
    rb = [f32(a) for a in rb]
    corners = [(lt[0], lt[1], lt[2]), (rb[0], lt[1], lt[2]), (rb[0], rb[1], lt[2]), (lt[0], rb[1], lt[2]),
               (lt[0], lt[1], rb[2]), (rb[0], lt[1], rb[2]), (rb[0], rb[1], rb[2]), (lt[0], rb[1], rb[2])]
    out = []
    for R, T in zip(Rs, Ts):
        R = [f32(a) for a in np.asarray(R, np.float64).reshape(9)]
        t2 = f32(np.asarray(T, np.float64).reshape(3)[2])
        zs = [f32(R[6] * c[0] + R[7] * c[1] + R[8] * c[2] + t2) for c in corners]
        out.append((max(f32(1e-6), min(zs)), max(zs)))
    return np.array(out, np.float32)
