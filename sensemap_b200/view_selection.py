"""Source-view selection and depth ranges from the sparse model (host, C ABI).

Mirrors ``Model::GetMaxOverlappingImages`` (src/mvs/model.cc:701-935) and
``Model::ComputeDepthRanges`` (:941-959), which PatchMatchController uses to
build its problems (patch_match_controller.cc:3153-3171). A model is given as
images (world-to-camera R, T and the rig flag) and sparse points with tracks.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _native as N


def _images(Rs, Ts, rig) -> "C.Array":
    n = len(Rs)
    arr = (N.smvs_model_image * n)()
    for i in range(n):
        arr[i].R[:] = [float(a) for a in np.asarray(Rs[i], np.float64).reshape(9)]
        arr[i].T[:] = [float(a) for a in np.asarray(Ts[i], np.float64).reshape(3)]
        arr[i].is_rig = int(bool(rig[i])) if rig is not None else 0
    return arr


def tracks_to_csr(tracks: Sequence[Sequence[int]]):
    offsets = np.zeros(len(tracks) + 1, np.int32)
    offsets[1:] = np.cumsum([len(t) for t in tracks])
    flat = np.fromiter((i for t in tracks for i in t), np.int32, int(offsets[-1]))
    return offsets, flat


def get_max_overlapping_images(Rs, Ts, points, tracks, max_num_images: int, min_triangulation_angle: float,
                               unique_image_idxs: Optional[Sequence[int]] = None, is_rig=None) -> list:
    """Per image, its selected source images (best first); [] for images not in
    unique_image_idxs (default: all)."""
    n = len(Rs)
    ims = _images(Rs, Ts, is_rig)
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    off, flat = tracks_to_csr(tracks)
    cand = np.ascontiguousarray(range(n) if unique_image_idxs is None else sorted(set(unique_image_idxs)), np.int32)
    out_off = np.zeros(n + 1, np.int32)
    out = np.zeros(max(n * max_num_images, 1), np.int32)
    N.check(N.lib().smvs_select_views(ims, n, pts.ctypes.data if len(pts) else None, len(pts), off.ctypes.data,
                                      flat.ctypes.data if len(flat) else None, cand.ctypes.data if len(cand) else None,
                                      len(cand), int(max_num_images), float(min_triangulation_angle),
                                      out_off.ctypes.data, out.ctypes.data))
    return [out[out_off[i]:out_off[i + 1]].tolist() for i in range(n)]


def compute_depth_ranges(Rs, Ts, bbox_lt, bbox_rb) -> np.ndarray:
    """(num_images, 2) depth ranges of the bounding box corners."""
    n = len(Rs)
    ims = _images(Rs, Ts, None)
    lt = np.ascontiguousarray(bbox_lt, np.float32)
    rb = np.ascontiguousarray(bbox_rb, np.float32)
    out = np.zeros((n, 2), np.float32)
    N.check(N.lib().smvs_compute_depth_ranges(ims, n, lt.ctypes.data, rb.ctypes.data, out.ctypes.data))
    return out
