"""Initial depth/normal maps from the sparse or prior model (GPU, C ABI).

Mirrors the map builders PatchMatchController runs before a PatchMatch pass
(src/controllers/patch_match_controller.cc): ``InitDepthMap`` (:1205-1307,
sparse points the view observes, splatted by InitDepthMapFromSparsePoint
:483-518), ``Model2Depth`` (:520-642, a triangle mesh) and ``Ply2Depth``
(:643-750, oriented dense points), and the Delaunay variant of InitDepthMap
(InitDepthMapFromDelaunay :398-474). Each returns ``(depth, normal,
depth_range)``: depth H x W, normal 3 x H x W, and the (first, second) pair
the reference returns. Inputs may be numpy arrays (host) or CUDA tensors
(device; outputs are then CUDA tensors too).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .patch_match import _addr, _is_cuda_tensor

PLY_INIT_DEPTH_LEVEL = 2  # src/mvs/utils.h:40


def _view(width, height, K, R, T) -> N.smvs_view:
    v = N.smvs_view()
    v.width, v.height = int(width), int(height)
    v.K[:] = [float(a) for a in np.asarray(K, np.float64).reshape(9)]
    v.R[:] = [float(a) for a in np.asarray(R, np.float64).reshape(9)]
    v.T[:] = [float(a) for a in np.asarray(T, np.float64).reshape(3)]
    return v


def _prep(arrays, dtypes):
    dev = any(_is_cuda_tensor(a) for a in arrays if a is not None)
    keep, ptrs = [], []
    for a, dt in zip(arrays, dtypes):
        if dev:
            import torch
            t = a if _is_cuda_tensor(a) else torch.as_tensor(np.asarray(a, dt)).cuda()
            t = t.to({np.float32: torch.float32, np.float64: torch.float64, np.int32: torch.int32}[dt]).contiguous()
            keep.append(t)
            ptrs.append(t.data_ptr() if t.numel() else None)
        else:
            x = np.ascontiguousarray(a, dtype=dt)
            keep.append(x)
            ptrs.append(x.ctypes.data if x.size else None)
    return dev, keep, ptrs


def _outputs(dev, height, width):
    if dev:
        import torch
        d = torch.empty((height, width), dtype=torch.float32, device="cuda")
        n = torch.empty((3, height, width), dtype=torch.float32, device="cuda")
        return d, n, d.data_ptr(), n.data_ptr()
    d = np.empty((height, width), np.float32)
    n = np.empty((3, height, width), np.float32)
    return d, n, d.ctypes.data, n.ctypes.data


def init_depth_from_sparse_points(width, height, K, R, T, xyz, stream=None):
    """InitDepthMap + InitDepthMapFromSparsePoint for the points the view observes."""
    dev, keep, (p,) = _prep([np.asarray(xyz).reshape(-1, 3) if not _is_cuda_tensor(xyz) else xyz.reshape(-1, 3)],
                            [np.float32])
    d, n, dp, np_ = _outputs(dev, height, width)
    rng = (C.c_float * 2)()
    N.check(N.lib().smvs_init_depth_from_sparse_points(
        C.byref(_view(width, height, K, R, T)), p, int(keep[0].shape[0]), N.MEM_DEVICE if dev else N.MEM_HOST,
        dp, np_, rng, C.c_void_p(int(stream)) if stream is not None else None))
    return d, n, (rng[0], rng[1])


def init_depth_from_delaunay(width, height, K, R, T, xyz, stream=None):
    """InitDepthMap with init_from_delaunay: the points the view observes,
    triangulated over their pixel positions (InitDepthMapFromDelaunay)."""
    dev, keep, (p,) = _prep([np.asarray(xyz).reshape(-1, 3) if not _is_cuda_tensor(xyz) else xyz.reshape(-1, 3)],
                            [np.float32])
    d, n, dp, np_ = _outputs(dev, height, width)
    rng = (C.c_float * 2)()
    N.check(N.lib().smvs_init_depth_from_delaunay(
        C.byref(_view(width, height, K, R, T)), p, int(keep[0].shape[0]), N.MEM_DEVICE if dev else N.MEM_HOST,
        dp, np_, rng, C.c_void_p(int(stream)) if stream is not None else None))
    return d, n, (rng[0], rng[1])


def delaunay_triangles(xy) -> np.ndarray:
    """The triangulation the Delaunay initial map uses: (m, 3) counter-clockwise
    vertex indices into the (n, 2) integer positions `xy` (host)."""
    xy = np.ascontiguousarray(xy, dtype=np.int32).reshape(-1, 2)
    cap = 2 * len(xy) + 8
    out = np.zeros((cap, 3), np.int32)
    cnt = C.c_int()
    N.check(N.lib().smvs_test_delaunay(xy.ctypes.data if len(xy) else None, len(xy), out.ctypes.data, cap,
                                       C.byref(cnt)))
    return out[:cnt.value].copy()


def init_depth_from_mesh(width, height, K, R, T, vertices, faces, face_normals, stream=None):
    """Model2Depth: rasterise a TriangleMesh (vertices_, faces_, face_normals_)."""
    dev, keep, (pv, pf, pn) = _prep([vertices, faces, face_normals], [np.float64, np.int32, np.float64])
    d, n, dp, np_ = _outputs(dev, height, width)
    rng = (C.c_float * 2)()
    N.check(N.lib().smvs_init_depth_from_mesh(
        C.byref(_view(width, height, K, R, T)), pv, int(keep[0].shape[0]), pf, int(keep[1].shape[0]), pn,
        N.MEM_DEVICE if dev else N.MEM_HOST, dp, np_, rng, C.c_void_p(int(stream)) if stream is not None else None))
    return d, n, (rng[0], rng[1])


def init_depth_from_dense_points(width, height, K, R, T, xyz, normals, level=PLY_INIT_DEPTH_LEVEL, stream=None):
    """Ply2Depth: splat oriented dense points (PlyPoint positions and normals)."""
    dev, keep, (px, pn) = _prep([xyz, normals], [np.float32, np.float32])
    d, n, dp, np_ = _outputs(dev, height, width)
    rng = (C.c_float * 2)()
    N.check(N.lib().smvs_init_depth_from_dense_points(
        C.byref(_view(width, height, K, R, T)), px, pn, int(keep[0].shape[0]), int(level),
        N.MEM_DEVICE if dev else N.MEM_HOST, dp, np_, rng, C.c_void_p(int(stream)) if stream is not None else None))
    return d, n, (rng[0], rng[1])
