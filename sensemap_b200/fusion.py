"""Python mirror of SenseMap's depth-map fusion over the C ABI.

``StereoFusion`` follows ``sensemap::mvs::StereoFusion`` (src/mvs/fusion.h:43-280,
fusion.cc:648-2182) for one cluster holding every image: construct with the
options, the images (size, K/R/T, depth map, normal map, color bitmap, rig
flag) and ``overlapping_images_`` (the source lists Model::GetMaxOverlappingImages
gives, see ``view_selection.get_max_overlapping_images``), call ``Run()``, then
``GetFusedPoints()`` / ``GetFusedPointsVisibility()`` /
``GetFusedPointsScore()``. Maps are numpy arrays on the host or CUDA tensors on
the device: depth H x W float32, normal 3 x H x W float32 (camera frame),
color H x W x 3 uint8 RGB. All compute runs in ``libsmvs.so``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .patch_match import _addr, _is_cuda_tensor, _sync_producers


@dataclass
class FusionOptions:
    """StereoFusion::Options (fusion.h:48-139), the fields the fusion loop reads."""
    step_size: int = 1
    min_num_pixels: int = 5
    max_num_pixels: int = 10000
    min_num_visible_images: int = 3
    max_traversal_depth: int = 100
    max_reproj_error: float = 2.0
    max_depth_error: float = float(np.float32(0.01))  # 0.01f stored in a double
    max_normal_error: float = 10.0
    with_normal: bool = True
    num_slices: int = 1
    gpu_index: int = 0

    def to_c(self) -> N.smvs_fusion_options:
        o = N.smvs_fusion_options()
        for name, _ in N.smvs_fusion_options._fields_:
            setattr(o, name, type(getattr(o, name))(getattr(self, name)))
        return o


@dataclass
class FusionImage:
    """One image of the workspace: mvs::Image plus its DepthMap, NormalMap and bitmap."""
    K: np.ndarray
    R: np.ndarray
    T: np.ndarray
    depth: object = None         # H x W; None = image not used
    normal: object = None        # 3 x H x W
    color: object = None         # H x W x 3 uint8
    is_rig: bool = False
    width: Optional[int] = None  # taken from depth when None
    height: Optional[int] = None


def fusion_structs(images: Sequence[FusionImage], overlapping_images: Sequence[Sequence[int]]):
    """(views array, overlap offsets, overlap images, memory kind, keep-alive list)."""
    n = len(images)
    if len(overlapping_images) != n:
        raise N.SmvsError(N.SMVS_EINVAL, "one overlapping-image list per image")
    views = (N.smvs_fusion_view * n)()
    keep, memories = [], set()
    for k, im in enumerate(images):
        cv = views[k]
        cv.K[:] = [float(a) for a in np.asarray(im.K, dtype=np.float64).reshape(9)]
        cv.R[:] = [float(a) for a in np.asarray(im.R, dtype=np.float64).reshape(9)]
        cv.T[:] = [float(a) for a in np.asarray(im.T, dtype=np.float64).reshape(3)]
        cv.is_rig = int(bool(im.is_rig))
        w, h = im.width, im.height
        for name, dtype in (("depth", np.float32), ("normal", np.float32), ("color", np.uint8)):
            a = getattr(im, name)
            if a is None:
                continue
            if not _is_cuda_tensor(a):
                a = np.ascontiguousarray(a, dtype=dtype)
            if name == "depth":
                h, w = int(a.shape[0]), int(a.shape[1])
            p, o, d = _addr(a)
            keep.append(o)
            memories.add(d)
            setattr(cv, name, p)
        cv.width = int(w) if w is not None else 0
        cv.height = int(h) if h is not None else 0
    if len(memories) > 1:
        raise N.SmvsError(N.SMVS_EINVAL, "all maps must live in the same memory (host or device)")
    off = np.zeros(n + 1, dtype=np.int32)
    for k, lst in enumerate(overlapping_images):
        off[k + 1] = off[k] + len(lst)
    flat = np.ascontiguousarray(np.concatenate([np.asarray(lst, dtype=np.int32) for lst in overlapping_images])
                                if off[-1] else np.zeros(1, dtype=np.int32))
    keep += [off, flat]
    memory = N.MEM_DEVICE if memories == {True} else N.MEM_HOST
    return views, off, flat, memory, keep


def split_visibility(offsets: np.ndarray, images: np.ndarray) -> list:
    return [images[offsets[i]:offsets[i + 1]] for i in range(len(offsets) - 1)]


class StereoFusion:
    """Drop-in for the fusion loop of sensemap::mvs::StereoFusion."""

    def __init__(self, options: FusionOptions, images: Sequence[FusionImage],
                 overlapping_images: Sequence[Sequence[int]], stream=None):
        self.options = options
        self._shape = []
        for im in images:
            if im.depth is not None:
                self._shape.append((int(im.depth.shape[0]), int(im.depth.shape[1])))
            else:
                self._shape.append((int(im.height or 0), int(im.width or 0)))
        views, off, flat, memory, keep = fusion_structs(images, overlapping_images)
        _sync_producers(keep, stream)
        handle = C.c_void_p()
        stream_ptr = C.c_void_p(int(stream)) if stream is not None else None
        N.check(N.lib().smvs_fusion_create(C.byref(options.to_c()), views, len(images), off.ctypes.data,
                                           flat.ctypes.data, memory, stream_ptr, C.byref(handle)))
        self._h = handle
        self._points = None

    def _handle(self):
        if self._h is None:
            raise N.SmvsError(N.SMVS_ESTATE, "fusion closed")
        return self._h

    def Run(self) -> None:
        N.check(N.lib().smvs_fusion_run(self._handle()))
        self._points = None

    def RemoveDuplicatePoints(self) -> int:
        """StereoFusion::RemoveDuplicatePoints (fusion.cc:2184-2266), which the
        reference's Run applies after the image loop when
        Options::remove_duplicate_pnts (its default). Returns the points dropped."""
        n = C.c_size_t()
        N.check(N.lib().smvs_fusion_remove_duplicate_points(self._handle(), C.byref(n)))
        self._points = None
        return int(n.value)

    def RemoveOutliers(self, nb_neighbors: int = 6, max_spacing_factor: float = 6.0) -> int:
        """StereoFusion::RemoveOutliers (fusion.cc:2542-2611), applied by the
        reference's Run when Options::outlier_removal (off by default); the
        defaults are Options::nb_neighbors and max_spacing_factor. Returns the
        points dropped; the remaining points' scores are updated."""
        n = C.c_size_t()
        N.check(N.lib().smvs_fusion_remove_outliers(self._handle(), int(nb_neighbors), float(max_spacing_factor),
                                                     C.byref(n)))
        self._points = None
        return int(n.value)

    def _fetch(self):
        if self._points is None:
            npts, nvis = C.c_size_t(), C.c_size_t()
            N.check(N.lib().smvs_fusion_get_sizes(self._handle(), C.byref(npts), C.byref(nvis)))
            pts = np.zeros(npts.value, dtype=N.FUSED_POINT_DTYPE)
            off = np.zeros(npts.value + 1, dtype=np.uint64)
            vis = np.zeros(max(nvis.value, 1), dtype=np.uint32)
            N.check(N.lib().smvs_fusion_get_points(self._handle(), pts.ctypes.data, off.ctypes.data, vis.ctypes.data))
            self._points = (pts, off, vis[:nvis.value])
        return self._points

    def GetFusedPoints(self) -> np.ndarray:
        """Structured array (x, y, z, nx, ny, nz, r, g, b, pad, score), in fusion order."""
        return self._fetch()[0]

    def GetFusedPointsVisibility(self) -> list:
        _, off, vis = self._fetch()
        return split_visibility(off, vis)

    def GetFusedPointsScore(self) -> np.ndarray:
        return self._fetch()[0]["score"].copy()

    def VisibilityCSR(self):
        """(offsets[num_points + 1] uint64, image indices uint32)."""
        _, off, vis = self._fetch()
        return off, vis

    def ImageOrder(self) -> list:
        order = np.zeros(max(len(self._shape), 1), dtype=np.int32)
        cnt = C.c_int()
        N.check(N.lib().smvs_fusion_get_image_order(self._handle(), order.ctypes.data, C.byref(cnt)))
        return [int(i) for i in order[:cnt.value]]

    def FusedPixelMask(self, view: int) -> np.ndarray:
        h, w = self._shape[view]
        out = np.zeros((h, w), dtype=np.uint8)
        N.check(N.lib().smvs_fusion_get_mask(self._handle(), int(view), out.ctypes.data))
        return out

    def SetProfiling(self, enable: bool = True) -> None:
        N.check(N.lib().smvs_fusion_set_profiling(self._handle(), int(bool(enable))))

    def Profile(self) -> dict:
        out = {}
        for kind, name in enumerate(N.FUSION_KERNEL_NAMES):
            cnt, ms = C.c_int(), C.c_double()
            N.check(N.lib().smvs_fusion_get_profile(self._handle(), kind, C.byref(cnt), C.byref(ms)))
            out[name] = (cnt.value, ms.value)
        return out

    def DependencyChains(self, with_shear: bool = False):
        """Per fused image, the longest chain of seeds that waited on one another
        (recorded when profiling was on during Run); with_shear also returns the
        shear K of each image's ticket order."""
        buf = np.zeros(max(len(self._shape), 1), dtype=np.uint32)
        shr = np.zeros_like(buf)
        cnt = C.c_int()
        N.check(N.lib().smvs_test_fusion_chains(self._handle(), buf.ctypes.data, shr.ctypes.data, len(buf),
                                                C.byref(cnt)))
        n = min(cnt.value, len(buf))
        chains = [int(x) for x in buf[:n]]
        return (chains, [int(x) for x in shr[:n]]) if with_shear else chains

    def ImageProfile(self) -> list:
        """With profiling: per fused image, {kernel kind: device ms}."""
        buf = np.zeros(4 * max(len(self._shape), 1), dtype=np.float64)
        cnt = C.c_int()
        N.check(N.lib().smvs_test_fusion_image_ms(self._handle(), buf.ctypes.data, len(buf) // 4, C.byref(cnt)))
        n = min(cnt.value, len(buf) // 4)
        return [{name: round(float(buf[4 * i + k]), 3) for k, name in enumerate(N.FUSION_KERNEL_NAMES)}
                for i in range(n)]

    def ReplayTimes(self) -> list:
        """With profiling: per fused image (mean us waiting, mean us from the end
        of the wait to the release, seeds with a record, mean record size, mean
        reachable set, seeds replayed one pixel at a time, mean us reading masks,
        finding the fused pixels, marking and releasing)."""
        buf = np.zeros(9 * max(len(self._shape), 1), dtype=np.float64)
        cnt = C.c_int()
        N.check(N.lib().smvs_test_fusion_replay_times(self._handle(), buf.ctypes.data, len(buf) // 9,
                                                      C.byref(cnt)))
        n = min(cnt.value, len(buf) // 9)
        return [tuple(round(float(x), 3) for x in buf[9 * i:9 * i + 9]) for i in range(n)]

    def LaunchCount(self) -> int:
        return int(N.lib().smvs_fusion_launch_count(self._handle()))

    def close(self) -> None:
        if self._h is not None:
            N.lib().smvs_fusion_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
