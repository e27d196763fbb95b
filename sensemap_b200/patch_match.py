"""Python mirror of SenseMap's depth-map operator over the C ABI.

``PatchMatchOptions``, ``Problem`` and ``PatchMatchACMMCuda`` keep the names,
fields, defaults and call sequence of the reference's
``sensemap::mvs::PatchMatchOptions`` / ``Problem`` (src/controllers/
patch_match_options.h:42-353) and ``PatchMatchACMMCuda`` (src/mvs/
patch_match_cuda.h:154-203): construct with (options, problem), call ``Run()``
(or ``RunFilter()``), then ``GetDepthMap()`` / ``GetNormalMap()`` /
``GetConfMap()``. Errors raise ``SmvsError`` instead of exiting the process.
All compute runs in ``libsmvs.so``; this module only marshals arguments.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, fields
from typing import Optional, Sequence

import numpy as np

from . import _native as N


@dataclass
class PatchMatchOptions:
    """Field-for-field mirror of PatchMatchOptions (patch_match_options.h:42-304)
    for the fields the depth-map path reads, with the reference's defaults."""
    depth_min: float = -1.0
    depth_max: float = -1.0
    window_radius: int = 5
    window_step: int = 2
    sigma_spatial: float = 5.0
    sigma_color: float = 0.2
    num_samples: int = 15
    num_iterations: int = 5
    geom_consistency: bool = True
    geom_consistency_regularizer: float = 0.3
    geom_consistency_max_cost: float = 3.0
    filter: bool = True
    filter_min_num_consistent: int = 1
    filter_geom_consistency_max_cost: float = 1.0
    max_normal_error: float = 15.0
    init_depth_random: bool = False
    random_depth_ratio: float = 0.004
    random_angle1_range: float = math.radians(20.0)
    random_angle2_range: float = math.radians(12.0)
    init_ncc_matching_cost: float = 0.8
    max_ncc_matching_cost: float = 1.2
    alpha: float = 90.0
    beta: float = 0.3
    thk: int = 4
    num_good_hypothesis: int = 2
    num_bad_hypothesis: int = 3
    random_optimization: bool = True
    local_optimization: bool = True
    est_curvature: bool = False
    median_filter: bool = False
    conf_filter: bool = False
    depth_diff_threshold: float = 0.02
    conf_threshold: float = 0.5
    has_prior_depth: bool = False
    propagate_depth: bool = False
    # No counterpart in the reference:
    random_seed: int = 0
    image_storage: int = N.STORE_U8
    gpu_index: int = -1

    def to_c(self) -> N.smvs_options:
        o = N.smvs_options()
        for f in fields(self):
            setattr(o, f.name, int(getattr(self, f.name)) if isinstance(getattr(self, f.name), bool)
                    else getattr(self, f.name))
        return o

    def check(self) -> None:
        N.check(N.lib().smvs_options_check(C.byref(self.to_c())))


@dataclass
class View:
    """One view: grey image (uint8 or float32, 0..255), K (3x3), world-to-camera
    R (3x3) and T (3,), as the reference's Image (src/mvs/image.h)."""
    image: object
    K: np.ndarray
    R: np.ndarray
    T: np.ndarray
    depth: Optional[object] = None   # H x W float32
    normal: Optional[object] = None  # 3 x H x W float32 (planar)
    scale: float = 1.0

    @property
    def width(self) -> int:
        return int(self.image.shape[1])

    @property
    def height(self) -> int:
        return int(self.image.shape[0])


@dataclass
class Problem:
    """Mirror of Problem (patch_match_options.h:306-353): reference index,
    source indices and scales into a shared list of views."""
    ref_image_idx: int
    src_image_idxs: Sequence[int]
    images: Sequence[View]
    src_image_scales: Sequence[float] = field(default_factory=list)
    mask: Optional[object] = None  # H x W uint8 mask of the reference view
    src_image_extend_idxs: Sequence[int] = field(default_factory=list)  # cross-filter neighbours (:314)
    prior_wgt: Optional[object] = None  # H x W prior weights of the reference view (prior_wgt_maps, :333)


class DeviceBuffer:
    """A raw device pointer (e.g. another engine's map from DeviceMaps()) with
    its shape, usable wherever a View takes an array. The owner must outlive
    every engine that reads it."""

    def __init__(self, ptr: int, shape, dtype=np.float32):
        self.ptr = int(ptr)
        self.shape = tuple(shape)
        self.dtype = np.dtype(dtype)
        self.is_cuda = True

    def data_ptr(self) -> int:
        return self.ptr

    def is_contiguous(self) -> bool:
        return True


def _is_cuda_tensor(x) -> bool:
    return hasattr(x, "is_cuda") and bool(getattr(x, "is_cuda"))


def _sync_producers(keep, stream) -> None:
    """The library reads device inputs on its own stream: when no stream is
    given, wait for the torch stream that produced them (and for any
    contiguous() copy made here) before handing their addresses over."""
    if stream is None and any(_is_cuda_tensor(o) for o in keep if o is not None):
        import torch
        torch.cuda.current_stream().synchronize()


def _addr(x):
    """(pointer, keep-alive object, is_device) of an array-like."""
    if x is None:
        return None, None, None
    if _is_cuda_tensor(x):
        if not x.is_contiguous():
            x = x.contiguous()
        return x.data_ptr(), x, True
    if hasattr(x, "numpy") and not isinstance(x, np.ndarray):  # CPU torch tensor
        x = x.numpy()
    x = np.ascontiguousarray(x)
    return x.ctypes.data, x, False


def _problem_struct(problem: Problem):
    """(smvs_problem, objects that must stay alive) for a Problem."""
    keep = []
    memories = set()

    def fill_view(cv: N.smvs_view, v: View, scale: float) -> None:
        img = v.image
        if _is_cuda_tensor(img):
            fmt = N.PIX_U8 if str(img.dtype) in ("torch.uint8", "uint8") else N.PIX_F32
            if fmt == N.PIX_F32 and str(img.dtype) not in ("torch.float32", "float32"):
                img = img.float()
        else:
            img = np.asarray(img)
            if img.dtype == np.uint8:
                fmt = N.PIX_U8
            else:
                img = img.astype(np.float32, copy=False)
                fmt = N.PIX_F32
        ptr, obj, dev = _addr(img)
        keep.append(obj)
        memories.add(dev)
        cv.width, cv.height, cv.pixel_format, cv.row_stride = v.width, v.height, fmt, 0
        cv.pixels = ptr
        cv.K[:] = [float(a) for a in np.asarray(v.K, dtype=np.float64).reshape(9)]
        cv.R[:] = [float(a) for a in np.asarray(v.R, dtype=np.float64).reshape(9)]
        cv.T[:] = [float(a) for a in np.asarray(v.T, dtype=np.float64).reshape(3)]
        cv.scale = float(scale)
        for name in ("depth", "normal"):
            arr = getattr(v, name)
            if arr is None:
                setattr(cv, name, None)
                continue
            if not _is_cuda_tensor(arr):
                arr = np.asarray(arr, dtype=np.float32)
            p, o, d = _addr(arr)
            keep.append(o)
            memories.add(d)
            setattr(cv, name, p)

    prob = N.smvs_problem()
    fill_view(prob.ref, problem.images[problem.ref_image_idx], 1.0)
    srcs = (N.smvs_view * len(problem.src_image_idxs))()
    scales = list(problem.src_image_scales) or [1.0] * len(problem.src_image_idxs)
    for i, idx in enumerate(problem.src_image_idxs):
        fill_view(srcs[i], problem.images[idx], scales[i])
    prob.src = srcs
    prob.num_src = len(problem.src_image_idxs)
    if problem.mask is not None:
        m = problem.mask if _is_cuda_tensor(problem.mask) else np.asarray(problem.mask, dtype=np.uint8)
        p, o, d = _addr(m)
        keep.append(o)
        memories.add(d)
        prob.ref_mask = p
    if problem.prior_wgt is not None:
        w = problem.prior_wgt if _is_cuda_tensor(problem.prior_wgt) else np.asarray(problem.prior_wgt, dtype=np.float32)
        p, o, d = _addr(w)
        keep.append(o)
        memories.add(d)
        prob.ref_prior_wgt = p
    if len(memories) > 1:
        raise N.SmvsError(N.SMVS_EINVAL, "all images and maps must live in the same memory (host or device)")
    prob.memory = N.MEM_DEVICE if memories == {True} else N.MEM_HOST
    return prob, keep


class PatchMatchACMMCuda:
    """Drop-in for sensemap::mvs::PatchMatchACMMCuda (patch_match_cuda.h:154-203)."""

    def __init__(self, options: PatchMatchOptions, problem: Problem, stream=None):
        self.options = options
        self.problem = problem
        lib = N.lib()
        prob, keep = _problem_struct(problem)
        _sync_producers(keep, stream)
        handle = C.c_void_p()
        stream_ptr = C.c_void_p(int(stream)) if stream is not None else None
        N.check(lib.smvs_create(C.byref(options.to_c()), C.byref(prob), stream_ptr, C.byref(handle)))
        self._h = handle
        self._keep = keep  # device inputs must outlive the engine's queued copies
        self.width = problem.images[problem.ref_image_idx].width
        self.height = problem.images[problem.ref_image_idx].height
        self.num_src = prob.num_src

    # -- reference API ------------------------------------------------------
    def Run(self) -> bool:
        N.check(N.lib().smvs_run(self._h))
        return True

    def RunFilter(self, deduplication_flag: bool = False) -> bool:
        N.check(N.lib().smvs_run_filter(self._h, int(deduplication_flag)))
        return True

    def _get(self, fn, shape, dtype):
        out = np.empty(shape, dtype=dtype)
        N.check(fn(self._h, out.ctypes.data))
        return out

    def GetDepthMap(self) -> np.ndarray:
        return self._get(N.lib().smvs_get_depth_map, (self.height, self.width), np.float32)

    def GetNormalMap(self) -> np.ndarray:
        """3 x H x W planar, like NormalMap's slices."""
        return self._get(N.lib().smvs_get_normal_map, (3, self.height, self.width), np.float32)

    def GetConfMap(self) -> np.ndarray:
        return self._get(N.lib().smvs_get_conf_map, (self.height, self.width), np.float32)

    def GetCostMap(self) -> np.ndarray:
        return self._get(N.lib().smvs_get_cost_map, (self.num_src, self.height, self.width), np.float32)

    def GetViewSelMap(self) -> np.ndarray:
        return self._get(N.lib().smvs_get_view_sel_map, (self.height, self.width), np.uint32)

    def GetCurvatureMap(self) -> np.ndarray:
        return self._get(N.lib().smvs_get_curvature_map, (2, self.height, self.width), np.uint16)

    # -- additions ----------------------------------------------------------
    def WriteMaps(self, stereo_dir: str, image_name: str, output_type: str = "photometric") -> None:
        N.check(N.lib().smvs_write_maps(self._h, stereo_dir.encode(), image_name.encode(), output_type.encode()))

    def Synchronize(self) -> None:
        N.check(N.lib().smvs_synchronize(self._h))

    def DeviceMaps(self) -> N.smvs_device_maps:
        m = N.smvs_device_maps()
        N.check(N.lib().smvs_get_device_maps(self._h, C.byref(m)))
        return m

    def DeviceDepthNormal(self):
        """(depth, normal) as DeviceBuffers over this engine's maps (valid until close())."""
        m = self.DeviceMaps()
        return (DeviceBuffer(m.depth, (self.height, self.width)),
                DeviceBuffer(m.normal, (3, self.height, self.width)))

    def LaunchCount(self) -> int:
        return int(N.lib().smvs_launch_count(self._h))

    def SetTuning(self, sweep_block_x: int = 32, ref_tile_tma: bool = True, threads_per_pixel: int = 1,
                  persistent: bool = False) -> None:
        t = N.smvs_tuning(sweep_block_x=sweep_block_x, ref_tile_tma=int(ref_tile_tma),
                          threads_per_pixel=int(threads_per_pixel), persistent=int(persistent))
        N.check(N.lib().smvs_set_tuning(self._h, C.byref(t)))

    def Tuning(self) -> dict:
        """Launch shape in use and whether the last Run staged reference tiles with TMA."""
        t = N.smvs_tuning()
        N.check(N.lib().smvs_get_tuning(self._h, C.byref(t)))
        return {"sweep_block_x": t.sweep_block_x, "ref_tile_tma": bool(t.ref_tile_tma),
                "threads_per_pixel": t.threads_per_pixel, "persistent": bool(t.persistent)}

    def SetProfiling(self, enable: bool = True) -> None:
        N.check(N.lib().smvs_set_profiling(self._h, int(enable)))

    def Profile(self) -> dict:
        """{kernel name: (launches, total device ms)} of the timed launches."""
        out = {}
        for kind, name in enumerate(N.KERNEL_NAMES):
            cnt, ms = C.c_int(), C.c_double()
            N.check(N.lib().smvs_get_profile(self._h, kind, C.byref(cnt), C.byref(ms)))
            if cnt.value:
                out[name] = (cnt.value, ms.value)
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().smvs_destroy(self._h)
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


def autotune(options: PatchMatchOptions, problem: Problem, stream=None, repeats: int = 3) -> dict:
    """Launch-shape autotuner (smvs_autotune): the fastest sweep launch shape for
    this problem, with every candidate's ms per sweep launch."""
    prob, keep = _problem_struct(problem)
    best = N.smvs_tuning()
    cap = 32
    tried = (N.smvs_tuning * cap)()
    ms = (C.c_double * cap)()
    n = C.c_int()
    stream_ptr = C.c_void_p(int(stream)) if stream is not None else None
    N.check(N.lib().smvs_autotune(C.byref(options.to_c()), C.byref(prob), stream_ptr, int(repeats), C.byref(best),
                                  tried, ms, cap, C.byref(n)))
    return {"sweep_block_x": best.sweep_block_x, "ref_tile_tma": bool(best.ref_tile_tma),
            "threads_per_pixel": best.threads_per_pixel, "persistent": bool(best.persistent),
            "candidates": [{"sweep_block_x": tried[i].sweep_block_x, "ref_tile_tma": bool(tried[i].ref_tile_tma),
                            "threads_per_pixel": tried[i].threads_per_pixel, "persistent": bool(tried[i].persistent),
                            "ms_per_sweep": ms[i]}
                           for i in range(min(n.value, cap))]}
