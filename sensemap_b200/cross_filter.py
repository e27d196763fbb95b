"""Python mirror of SenseMap's cross-view filter over the C ABI.

``CrossFilterCuda`` keeps the constructor arguments, methods and call order of
``sensemap::mvs::CrossFilterCuda`` (src/mvs/patch_match_cuda.h:205-269,
patch_match_cuda.cu:1111-1710): construct with (options, problems, whole_ids,
ref_flags), ``Run()``, ``GetRefineDepthMap(image_id)``, then ``DedupRun()`` and
``GetDeduplicDepthMap`` / ``GetDeltDepthMap`` / ``GetVisibilyMap``. Each
problem's reference and ``src_image_extend_idxs`` are image ids looked up in
``whole_ids`` (FindSrcImageIds, :1427-1455): ids not in the set are skipped, a
problem left without sources is skipped. Depth and normal maps are the views'
``depth`` (H x W) and ``normal`` (3 x H x W) arrays, numpy on the host or CUDA
tensors on the device. All compute runs in ``libsmvs.so``.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _native as N
from .patch_match import PatchMatchOptions, Problem, _addr, _is_cuda_tensor, _sync_producers


class CrossFilterCuda:
    """Drop-in for sensemap::mvs::CrossFilterCuda."""

    def __init__(self, options: PatchMatchOptions, problems: Sequence[Problem], whole_ids: Sequence[int],
                 ref_flags: Sequence[bool], stream=None):
        if len(whole_ids) != len(ref_flags):
            raise N.SmvsError(N.SMVS_EINVAL, "whole_ids and ref_flags differ in length")
        if not problems:
            raise N.SmvsError(N.SMVS_EINVAL, "no problems")
        images = problems[0].images
        self.whole_ids = [int(i) for i in whole_ids]
        self._pos = {image_id: k for k, image_id in enumerate(self.whole_ids)}
        keep, memories = [], set()
        views = (N.smvs_filter_view * len(self.whole_ids))()
        self._shape = []
        for k, image_id in enumerate(self.whole_ids):
            v = images[image_id]
            cv = views[k]
            depth = v.depth if _is_cuda_tensor(v.depth) else np.asarray(v.depth, dtype=np.float32)
            h, w = int(depth.shape[0]), int(depth.shape[1])
            cv.width, cv.height = w, h
            cv.K[:] = [float(a) for a in np.asarray(v.K, dtype=np.float64).reshape(9)]
            cv.R[:] = [float(a) for a in np.asarray(v.R, dtype=np.float64).reshape(9)]
            cv.T[:] = [float(a) for a in np.asarray(v.T, dtype=np.float64).reshape(3)]
            p, o, d = _addr(depth)
            keep.append(o)
            memories.add(d)
            cv.depth = p
            if v.normal is not None:
                normal = v.normal if _is_cuda_tensor(v.normal) else np.asarray(v.normal, dtype=np.float32)
                p, o, d = _addr(normal)
                keep.append(o)
                memories.add(d)
                cv.normal = p
            cv.ref_flag = int(bool(ref_flags[k]))
            self._shape.append((h, w))
        if len(memories) > 1:
            raise N.SmvsError(N.SMVS_EINVAL, "all maps must live in the same memory (host or device)")
        probs = (N.smvs_filter_problem * len(problems))()
        n_used = 0
        for pr in problems:
            if pr.ref_image_idx not in self._pos:  # :1430-1434
                continue
            srcs = [self._pos[i] for i in pr.src_image_extend_idxs if i in self._pos]
            arr = (C.c_int * max(len(srcs), 1))(*srcs)
            keep.append(arr)
            probs[n_used].ref = self._pos[pr.ref_image_idx]
            probs[n_used].src = C.cast(arr, C.POINTER(C.c_int))
            probs[n_used].num_src = len(srcs)
            n_used += 1
        handle = C.c_void_p()
        memory = N.MEM_DEVICE if memories == {True} else N.MEM_HOST
        _sync_producers(keep, stream)
        stream_ptr = C.c_void_p(int(stream)) if stream is not None else None
        N.check(N.lib().smvs_cross_filter_create(C.byref(options.to_c()), views, len(self.whole_ids), probs, n_used,
                                                 memory, stream_ptr, C.byref(handle)))
        self._h = handle
        self._keep = keep

    def _index(self, image_id: int) -> int:
        if image_id not in self._pos:
            raise N.SmvsError(N.SMVS_EINVAL, f"image {image_id} is not in whole_ids")
        return self._pos[image_id]

    def _get(self, fn, image_id: int, dtype) -> np.ndarray:
        k = self._index(image_id)
        out = np.empty(self._shape[k], dtype=dtype)
        N.check(fn(self._h, k, out.ctypes.data))
        return out

    # -- reference API ------------------------------------------------------
    def Run(self) -> bool:
        N.check(N.lib().smvs_cross_filter_run(self._h))
        return True

    def DedupRun(self) -> bool:
        N.check(N.lib().smvs_cross_filter_dedup_run(self._h))
        return True

    def GetRefineDepthMap(self, image_id: int) -> np.ndarray:
        return self._get(N.lib().smvs_cross_filter_get_refined_depth_map, image_id, np.float32)

    def GetDeduplicDepthMap(self, image_id: int) -> np.ndarray:
        return self._get(N.lib().smvs_cross_filter_get_dedup_depth_map, image_id, np.float32)

    def GetDeltDepthMap(self, image_id: int) -> np.ndarray:
        return self._get(N.lib().smvs_cross_filter_get_delta_depth_map, image_id, np.float32)

    def GetVisibilyMap(self, image_id: int) -> np.ndarray:
        return self._get(N.lib().smvs_cross_filter_get_visibility_map, image_id, np.uint32)

    # -- additions ----------------------------------------------------------
    def DeviceMaps(self, image_id: int) -> dict:
        """Device addresses of the view's refined, delta and visibility maps (0 = absent)."""
        k = self._index(image_id)
        r, d, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        N.check(N.lib().smvs_cross_filter_get_device_maps(self._h, k, C.byref(r), C.byref(d), C.byref(v)))
        return {"refined": r.value or 0, "delta": d.value or 0, "visibility": v.value or 0}

    def SetProfiling(self, enable: bool = True) -> None:
        N.check(N.lib().smvs_cross_filter_set_profiling(self._h, int(enable)))

    def Profile(self) -> dict:
        """{kernel kind: (launches, summed device ms)} of the timed launches."""
        out = {}
        for k, name in enumerate(N.CF_KERNEL_NAMES):
            n, ms = C.c_int(), C.c_double()
            N.check(N.lib().smvs_cross_filter_get_profile(self._h, k, C.byref(n), C.byref(ms)))
            if n.value:
                out[name] = (n.value, ms.value)
        return out

    def LaunchCount(self) -> int:
        return int(N.lib().smvs_cross_filter_launch_count(self._h))

    def DedupLevels(self) -> int:
        return int(N.lib().smvs_cross_filter_dedup_levels(self._h))

    def Synchronize(self) -> None:
        N.check(N.lib().smvs_cross_filter_synchronize(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().smvs_cross_filter_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def filter_problems(ref_ids: Sequence[int], neighbours: Sequence[Sequence[int]], images) -> list:
    """Problems in the cross filter's shape: one per reference id, with
    src_image_extend_idxs = its neighbour ids."""
    return [Problem(ref_image_idx=int(r), src_image_idxs=[], images=images,
                    src_image_extend_idxs=[int(s) for s in nb]) for r, nb in zip(ref_ids, neighbours)]
