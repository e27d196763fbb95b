"""Pure-Python restatement of the depth-map fusion (test infrastructure only).

An independent second restatement of StereoFusion's image loop (SenseMap
src/mvs/fusion.cc: Run :1160-1215, FindNextImage :697-727, FuseImage
:1730-1792, Fuse :1794-2182), written from the reference with numpy float32
scalars in the evaluation order of the reference's Eigen expressions (the same
conventions as oracle/smvs_oracle_fusion.c: packet products reduced as
(p0 + p2) + (p1 + p3), homogeneous products as ((p0 + p1) + p2) + p3, Vector3f
products as (p0 + p1) + p2, the inverse projection computed in double and
rounded once, medians in the sign-first total order of floats). Loops in
Python: for images of a few thousand pixels. The tests check the C oracle
against it bit for bit.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32
BLANK = 3


def _p(K, R, T):
    K = np.asarray(K, F).reshape(9)
    R = np.asarray(R, F).reshape(9)
    T = np.asarray(T, F).reshape(3)
    M = [[R[0], R[1], R[2], T[0]], [R[3], R[4], R[5], T[1]], [R[6], R[7], R[8], T[2]]]
    P = np.zeros(12, F)
    for i in range(3):
        for j in range(4):
            P[4 * i + j] = (K[3 * i] * M[0][j] + K[3 * i + 1] * M[1][j]) + K[3 * i + 2] * M[2][j]
    return P


def _inv_p(P):
    m = [float(P[k]) for k in (0, 1, 2, 4, 5, 6, 8, 9, 10)]
    m0, m1, m2, m3, m4, m5, m6, m7, m8 = m
    c00, c01, c02 = m4 * m8 - m5 * m7, m2 * m7 - m1 * m8, m1 * m5 - m2 * m4
    c10, c11, c12 = m5 * m6 - m3 * m8, m0 * m8 - m2 * m6, m2 * m3 - m0 * m5
    c20, c21, c22 = m3 * m7 - m4 * m6, m1 * m6 - m0 * m7, m0 * m4 - m1 * m3
    det = m0 * c00 + m1 * c10 + m2 * c20
    inv = [c00 / det, c01 / det, c02 / det, c10 / det, c11 / det, c12 / det, c20 / det, c21 / det, c22 / det]
    p = [float(P[3]), float(P[7]), float(P[11])]
    iP = np.zeros(12, F)
    for i in range(3):
        iP[4 * i:4 * i + 3] = [inv[3 * i], inv[3 * i + 1], inv[3 * i + 2]]
        iP[4 * i + 3] = -(inv[3 * i] * p[0] + inv[3 * i + 1] * p[1] + inv[3 * i + 2] * p[2])
    return iP


def _dot4p(a, x, y, z, w):
    return (a[0] * x + a[2] * z) + (a[1] * y + a[3] * w)


def _dot3h(a, x, y, z):
    return ((a[0] * x + a[1] * y) + a[2] * z) + a[3]


def _roundf(x):
    x = float(x)
    if math.isnan(x) or math.isinf(x):
        return x
    return math.copysign(math.floor(abs(x) + 0.5), x)


def _key(f):
    u = int(np.asarray(f, F).view(np.uint32))
    return (~u) & 0xFFFFFFFF if u & 0x80000000 else u | 0x80000000


def _median(vals):
    v = sorted(vals, key=_key)
    n = len(v)
    mid = n // 2
    if n % 2 == 0:
        return F((F(v[mid]) + F(v[mid - 1])) / F(2.0))
    return F(v[mid])


def fuse(options, images, overlaps):
    """StereoFusion's loop over host maps (sensemap_b200.fusion.FusionImage).
    Returns (points as a list of dicts, visibility lists, order, masks)."""
    nv = len(images)
    used = [im.depth is not None for im in images]
    fused = [False] * nv
    P, iP, iR, W, H, masks = [], [], [], [], [], []
    for im in images:
        p = _p(im.K, im.R, im.T)
        P.append(p)
        iP.append(_inv_p(p))
        R = np.asarray(im.R, F).reshape(3, 3)
        iR.append(R.T.copy())
        if im.depth is not None:
            h, w = im.depth.shape
        else:
            h, w = 0, 0
        W.append(w)
        H.append(h)
        masks.append(np.zeros((h, w), np.uint8))
    max_sq = F(options.max_reproj_error * options.max_reproj_error)
    min_cos = F(math.cos(options.max_normal_error * 0.0174532925199432954743716805978692718781530857086181640625))
    points, vis_lists, order = [], [], []

    def find_next(prev):
        for rig_ok in (False, True):
            for i in overlaps[prev]:
                if used[i] and not fused[i] and (rig_ok or not images[i].is_rig):
                    return i
        for rig_ok in (False, True):
            for i in range(nv):
                if used[i] and not fused[i] and (rig_ok or not images[i].is_rig):
                    return i
        return -1

    def fuse_seed(image, row0, col0):
        xs, ys, zs, nxs, nys, nzs, cs, rs, gs, bs, errs, vis = ([] for _ in range(12))
        ref = [F(0)] * 3
        ref_n = [F(0)] * 3
        stack = [(image, row0, col0, 0)]
        while stack:
            v, row, col, td = stack.pop()
            if masks[v][row, col]:
                continue
            depth = F(images[v].depth[row, col])
            if not (depth > 0) or not math.isfinite(depth):
                continue
            derr = F(0)
            if td > 0:
                p0 = _dot4p(P[v][0:4], ref[0], ref[1], ref[2], F(1))
                p1 = _dot4p(P[v][4:8], ref[0], ref[1], ref[2], F(1))
                p2 = _dot4p(P[v][8:12], ref[0], ref[1], ref[2], F(1))
                cd = p0 / p2 - F(col)
                rd = p1 / p2 - F(row)
                if cd * cd + rd * rd > max_sq:
                    continue
                derr = F(abs(p2 - depth) / depth)
                if float(derr) > options.max_depth_error:
                    continue
            nrm = [F(0)] * 3
            if options.with_normal:
                n = [F(images[v].normal[k, row, col]) for k in range(3)]
                nrm = [(iR[v][i, 0] * n[0] + iR[v][i, 1] * n[1]) + iR[v][i, 2] * n[2] for i in range(3)]
                if td > 0 and (ref_n[0] * nrm[0] + ref_n[1] * nrm[1]) + ref_n[2] * nrm[2] < min_cos:
                    continue
            cdp, rdp = F(col) * depth, F(row) * depth
            xyz = [_dot4p(iP[v][4 * i:4 * i + 4], cdp, rdp, depth, F(1)) for i in range(3)]
            rgb = [0, 0, 0]
            grad = F(0)
            img = images[v].color
            if img is not None:
                rgb = [int(img[row, col, k]) for k in range(3)]
                if 1 < col < W[v] - 1 and 1 < row < H[v] - 1:
                    gx = F(int(img[row, col - 1, 0]) - int(img[row, col + 1, 0])) / F(255)
                    gy = F(int(img[row - 1, col, 0]) - int(img[row + 1, col, 0])) / F(255)
                    grad = F(np.sqrt(gx * gx + gy * gy))
            masks[v][row, col] = 1
            xs.append(xyz[0]); ys.append(xyz[1]); zs.append(xyz[2])
            nxs.append(nrm[0]); nys.append(nrm[1]); nzs.append(nrm[2])
            cs.append(grad); rs.append(F(rgb[0])); gs.append(F(rgb[1])); bs.append(F(rgb[2]))
            vis.append(v)
            if td > 0:
                errs.append(derr)
            if td == 0:
                ref, ref_n = xyz, nrm
            if len(xs) >= options.max_num_pixels:
                break
            if td + 1 >= options.max_traversal_depth:
                continue
            for u in overlaps[v]:
                if not used[u] or fused[u]:
                    continue
                q = [_dot3h(P[u][4 * i:4 * i + 4], xyz[0], xyz[1], xyz[2]) for i in range(3)]
                uc, ur = _roundf(q[0] / q[2]), _roundf(q[1] / q[2])
                if not (uc >= BLANK and ur >= BLANK and uc < W[u] - BLANK and ur < H[u] - BLANK):
                    continue
                stack.append((u, int(ur), int(uc), td + 1))
        n = len(xs)
        vis_set = sorted(set(vis))
        if n < options.min_num_pixels or len(vis_set) < options.min_num_visible_images:
            return
        pt = {"x": _median(xs), "y": _median(ys), "z": _median(zs), "nx": F(0), "ny": F(0), "nz": F(0)}
        if not all(math.isfinite(pt[k]) for k in ("x", "y", "z")):
            return
        if options.with_normal:
            fn = [_median(nxs), _median(nys), _median(nzs)]
            norm = F(np.sqrt((fn[0] * fn[0] + fn[1] * fn[1]) + fn[2] * fn[2]))
            if norm < F(np.finfo(np.float32).eps):
                return
            pt["nx"], pt["ny"], pt["nz"] = fn[0] / norm, fn[1] / norm, fn[2] / norm
        for name, vals in (("r", rs), ("g", gs), ("b", bs)):
            m = _roundf(_median(vals))
            pt[name] = int(max(0.0, min(255.0, m)))
        m_conf = F(0)
        for c in cs:
            m_conf = F(m_conf + c)
        m_conf = F(m_conf / F(n))
        if len(vis_set) >= 3:
            m_conf = F(1)
        m_conf = F(1) - m_conf
        score = F(float(_median(errs)) / options.max_depth_error)
        mixed = F(0.6) * score + F(0.4) * m_conf
        score = F(1) if F(1) < mixed else mixed
        if not math.isfinite(score):
            return
        pt["score"] = score
        points.append(pt)
        vis_lists.append(vis_set)

    start = next((i for i in range(nv) if not images[i].is_rig), 0)
    image = start
    while image >= 0:
        if used[image]:
            w, h, T = W[image], H[image], options.num_slices
            hs = (h + T - 1) // T
            for t in range(T):
                row_end = min(min(hs * (t + 1), h), h - BLANK)
                for row in range(max(hs * t, BLANK), row_end, options.step_size):
                    for col in range(BLANK, w - BLANK, options.step_size):
                        if not masks[image][row, col]:
                            fuse_seed(image, row, col)
            fused[image] = True
            order.append(image)
        image = find_next(image)
    return points, vis_lists, order, masks
