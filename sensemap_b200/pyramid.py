"""Coarse-to-fine PatchMatch over an image pyramid, on the GPU.

The reference's controller runs its passes per pyramid level
(PatchMatchController::ClusterReconstruction's pass list,
patch_match_controller.cc:3486-3554, 3569-3610): at the coarsest level a
photometric pass from random hypotheses and a geometric pass; at every finer
level a geometric pass of 3 iterations (:3599-3601) that starts from the
coarser level's maps. Images are rescaled per level from the full-resolution
image (ProcessProblem, :4407-4410, 4610; Image::Rescale, src/mvs/image.cc:
44-70) and maps are carried to the finer level by DepthMap::Rescale /
NormalMap::Rescale (FillDepthMap, :751-861). Here every rescale runs on the
device (smvs_rescale_image, smvs_resample_maps) and the passes run through the
engine with device-resident inputs; nothing goes through host memory between
levels.

``refine`` names the views refined at the finer levels. The other views keep
their coarsest-level maps, resampled to each level, as the geometric term of
the refined views (the large-single-view case: one reference view refined at
full resolution against sources solved at the coarse level).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .patch_match import PatchMatchACMMCuda, PatchMatchOptions, Problem, View


def level_size(width: int, height: int, level: int):
    """(width, height, factor) of pyramid level `level`."""
    w, h, f = C.c_int(), C.c_int(), C.c_float()
    N.check(N.lib().smvs_pyramid_level_size(int(width), int(height), int(level), C.byref(w), C.byref(h),
                                            C.byref(f)))
    return w.value, h.value, f.value


def rescale_image(image, width: int, height: int, stream=None):
    """Device grey image (torch, H x W float32) resampled to width x height."""
    import torch
    H, W = image.shape
    out = torch.empty((height, width), dtype=torch.float32, device=image.device)
    tmp = torch.empty((H, width), dtype=torch.float32, device=image.device)
    N.check(N.lib().smvs_rescale_image(image.data_ptr(), W, H, out.data_ptr(), width, height, tmp.data_ptr(),
                                       C.c_void_p(int(stream)) if stream is not None else None))
    return out, tmp  # tmp must live until the stream has run the kernels


def resample_maps(depth, normal, width: int, height: int, stream=None):
    """Device depth (H x W) and normal (3 x H x W) maps resampled to width x height."""
    import torch
    H, W = depth.shape
    od = torch.empty((height, width), dtype=torch.float32, device=depth.device)
    on = torch.empty((3, height, width), dtype=torch.float32, device=depth.device)
    N.check(N.lib().smvs_resample_maps(depth.data_ptr(), normal.data_ptr(), W, H, od.data_ptr(), on.data_ptr(),
                                       width, height, C.c_void_p(int(stream)) if stream is not None else None))
    return od, on


def scaled_K(K, width, height, new_width, new_height):
    """Image::Rescale's intrinsics (image.cc:58-63)."""
    K = np.array(K, np.float64, copy=True)
    sx, sy = new_width / float(width), new_height / float(height)
    K[0, 0] *= sx
    K[0, 2] *= sx
    K[1, 1] *= sy
    K[1, 2] *= sy
    return K


@dataclass
class PyramidResult:
    depth: dict          # view -> device depth map at level 0 (refined views) or the last level they ran
    normal: dict
    level_seconds: list  # wall seconds per level (coarsest first)
    peak_device_bytes: int
    passes: int


class PyramidPatchMatch:
    """Coarse-to-fine depth maps for `problems` [(ref, [src, ...]), ...] over
    `views` (View with device-resident torch images, full resolution)."""

    def __init__(self, options: PatchMatchOptions, views: Sequence[View], problems, levels: int = 3,
                 refine: Optional[Sequence[int]] = None, fine_iterations: int = 3, stream=None, tuning=None):
        self.options = options
        self.views = list(views)
        self.problems = {int(r): list(s) for r, s in problems}
        self.levels = int(levels)
        self.refine = set(self.problems) if refine is None else set(int(r) for r in refine)
        self.fine_iterations = int(fine_iterations)
        self.stream = stream
        self.tuning = tuning

    def _device_used(self):
        import torch
        free, total = torch.cuda.mem_get_info()
        return total - free

    def _pass(self, opts, ref, level_views, maps, seed):
        o = replace(opts, random_seed=seed)
        vs = []
        for i, v in enumerate(level_views):
            d, n = maps.get(i, (None, None))
            vs.append(View(v.image, v.K, v.R, v.T, depth=d, normal=n))
        pm = PatchMatchACMMCuda(o, Problem(ref, self.problems[ref], vs), stream=self.stream)
        if self.tuning:
            pm.SetTuning(**self.tuning)
        pm.Run()
        return pm

    def Run(self) -> PyramidResult:
        import time
        import torch
        top = self.levels - 1
        maps = {}      # view -> (depth, normal) at the current level
        sizes = {}
        times = []
        peak = self._device_used()
        passes = 0
        for level in range(top, -1, -1):
            t0 = time.perf_counter()
            level_views, keep = [], []
            for v in self.views:
                H, W = v.image.shape
                w, h, _ = level_size(W, H, level)
                img, tmp = rescale_image(v.image, w, h, self.stream) if (w, h) != (W, H) else (v.image, None)
                keep.append(tmp)
                level_views.append(View(img, scaled_K(v.K, W, H, w, h), v.R, v.T))
                sizes[len(level_views) - 1] = (w, h)
            if level == top:
                # Photometric pass from random hypotheses, then a geometric pass.
                photo = {}
                for r in self.problems:
                    pm = self._pass(replace(self.options, geom_consistency=False, init_depth_random=True), r,
                                    level_views, {}, r)
                    photo[r] = pm
                    passes += 1
                peak = max(peak, self._device_used())
                maps = {r: pm.DeviceDepthNormal() for r, pm in photo.items()}
                maps = {r: (_as_tensor(d), _as_tensor(n)) for r, (d, n) in maps.items()}
                geo = {}
                for r in self.problems:
                    pm = self._pass(replace(self.options, geom_consistency=True, init_depth_random=False), r,
                                    level_views, maps, 1000 + r)
                    geo[r] = pm
                    passes += 1
                peak = max(peak, self._device_used())
                maps = {r: tuple(_as_tensor(x) for x in pm.DeviceDepthNormal()) for r, pm in geo.items()}
                for pm in list(photo.values()) + list(geo.values()):
                    pm.Synchronize()
                holders = list(photo.values()) + list(geo.values())
            else:
                # Carry every view's maps to this level, then refine.
                new_maps = {}
                for r, (d, n) in maps.items():
                    w, h = sizes[r]
                    new_maps[r] = resample_maps(d, n, w, h, self.stream)
                torch.cuda.synchronize()
                for pm in holders:
                    pm.close()
                maps = new_maps
                holders = []
                refined = {}
                for r in sorted(self.refine):
                    o = replace(self.options, geom_consistency=True, init_depth_random=False,
                                num_iterations=self.fine_iterations)
                    pm = self._pass(o, r, level_views, maps, 2000 + 100 * level + r)
                    refined[r] = pm
                    passes += 1
                    peak = max(peak, self._device_used())
                for r, pm in refined.items():
                    maps[r] = tuple(_as_tensor(x) for x in pm.DeviceDepthNormal())
                holders = list(refined.values())
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        out_d = {r: maps[r][0].clone() for r in self.refine}
        out_n = {r: maps[r][1].clone() for r in self.refine}
        torch.cuda.synchronize()
        for pm in holders:
            pm.close()
        return PyramidResult(out_d, out_n, times, peak, passes)


def _as_tensor(buf):
    """A torch view of an engine's device map (DeviceBuffer); the engine must
    stay open while it is used."""
    import torch
    if isinstance(buf, torch.Tensor):
        return buf
    return _wrap_device(buf.ptr, buf.shape)


def _wrap_device(ptr: int, shape):
    """Zero-copy torch tensor over a device pointer (via the CUDA array interface)."""
    import torch

    class _Holder:
        def __init__(self, p, s):
            self.__cuda_array_interface__ = {"shape": tuple(s), "typestr": "<f4", "data": (int(p), False),
                                             "version": 3, "strides": None}
    return torch.as_tensor(_Holder(ptr, shape), device="cuda")
