"""ctypes front end of the reference's own kernels (oracle/_ref/libref_pm.so,
built by oracle/ref_build.py). Test infrastructure only; needs a GPU.

Runs a Problem through the reference's InitConfMapKernel / Black/Red
PixelUpdateOpt / LocalOptimization / FilterDepthMapsKernel in the order
PatchMatchACMMCuda::Run issues them. The reference draws from cuRAND, so
full runs are compared statistically; cost-level results and the filter are
deterministic.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from sensemap_b200.patch_match import PatchMatchOptions, Problem

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libref_pm.so"
_LIB = None


class RefJob(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("N", C.c_int),
                ("ref", C.c_void_p), ("src", C.POINTER(C.c_void_p)), ("src_w", C.POINTER(C.c_int)),
                ("src_h", C.POINTER(C.c_int)), ("poses", C.c_void_p),
                ("refK", C.c_float * 4), ("refiK", C.c_float * 4),
                ("R", C.c_int), ("S", C.c_int), ("sigma_s", C.c_float), ("sigma_c", C.c_float),
                ("depth_min", C.c_float), ("depth_max", C.c_float),
                ("num_iterations", C.c_int), ("geom", C.c_int), ("init_depth_random", C.c_int),
                ("local_opt", C.c_int), ("random_opt", C.c_int), ("num_samples", C.c_int), ("thk", C.c_int),
                ("good", C.c_int), ("bad", C.c_int),
                ("geom_reg", C.c_float), ("geom_max", C.c_float), ("rand_depth_ratio", C.c_float),
                ("a1", C.c_float), ("a2", C.c_float), ("init_mc", C.c_float), ("max_mc", C.c_float),
                ("alpha", C.c_float), ("beta", C.c_float),
                ("init_depth", C.c_void_p), ("init_normal", C.c_void_p), ("src_depth", C.POINTER(C.c_void_p)),
                ("prior_mode", C.c_int), ("prior_wgt", C.c_void_p)]


class RefOut(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("depth", "normal", "conf", "cost", "view_sel")]


class RefCfView(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("depth", C.c_void_p), ("code", C.c_void_p), ("ref_flag", C.c_int)]


class RefCfProblem(C.Structure):
    _fields_ = [("ref", C.c_int), ("num_src", C.c_int), ("src", C.POINTER(C.c_int)), ("poses", C.c_void_p),
                ("refK", C.c_float * 4), ("refiK", C.c_float * 4)]


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} missing: run oracle/ref_build.py where the reference tree exists")
        h = C.CDLL(str(LIB_PATH))
        h.ref_run.restype = C.c_int
        h.ref_run.argtypes = [C.POINTER(RefJob), C.POINTER(RefOut)]
        h.ref_filter.restype = C.c_int
        h.ref_filter.argtypes = [C.POINTER(RefJob), C.c_void_p, C.c_int, C.c_float, C.c_void_p]
        h.ref_max_num_src.restype = C.c_int
        h.ref_propagate_init.restype = C.c_int
        h.ref_propagate_init.argtypes = [C.POINTER(RefJob), C.c_void_p, C.c_void_p, C.c_void_p]
        h.ref_cross_filter.restype = C.c_int
        h.ref_cross_filter.argtypes = [C.c_int, C.POINTER(RefCfView), C.c_int, C.POINTER(RefCfProblem), C.c_float,
                                       C.c_float, C.c_float, C.c_int, C.c_void_p]
        h.ref_dedup.restype = C.c_int
        h.ref_dedup.argtypes = [C.c_int, C.POINTER(RefCfView), C.c_int, C.POINTER(RefCfProblem), C.c_float,
                                C.c_float, C.c_int, C.c_void_p, C.c_void_p]
        _LIB = h
    return _LIB


def _u8(img):
    return np.ascontiguousarray(np.clip(np.rint(np.asarray(img, np.float32)), 0, 255).astype(np.uint8))


def _job(options: PatchMatchOptions, problem: Problem, poses: np.ndarray, keep: list) -> RefJob:
    ref = problem.images[problem.ref_image_idx]
    srcs = [problem.images[i] for i in problem.src_image_idxs]
    j = RefJob()
    j.W, j.H, j.N = ref.width, ref.height, len(srcs)
    r = _u8(ref.image)
    keep.append(r)
    j.ref = r.ctypes.data
    s_imgs = [_u8(v.image) for v in srcs]
    keep.extend(s_imgs)
    arr = (C.c_void_p * len(srcs))(*[a.ctypes.data for a in s_imgs])
    keep.append(arr)
    j.src = C.cast(arr, C.POINTER(C.c_void_p))
    sw = (C.c_int * len(srcs))(*[v.width for v in srcs])
    sh = (C.c_int * len(srcs))(*[v.height for v in srcs])
    keep += [sw, sh]
    j.src_w, j.src_h = C.cast(sw, C.POINTER(C.c_int)), C.cast(sh, C.POINTER(C.c_int))
    p = np.ascontiguousarray(poses, np.float32)
    keep.append(p)
    j.poses = p.ctypes.data
    K = np.asarray(ref.K, np.float32)
    refK = np.array([K[0, 0], K[0, 2], K[1, 1], K[1, 2]], np.float32)
    j.refK[:] = list(refK)
    j.refiK[:] = [np.float32(1) / refK[0], -refK[1] / refK[0], np.float32(1) / refK[2], -refK[3] / refK[2]]
    o = options
    j.R, j.S, j.sigma_s, j.sigma_c = o.window_radius, o.window_step, o.sigma_spatial, o.sigma_color
    j.depth_min, j.depth_max = o.depth_min, o.depth_max
    j.num_iterations, j.geom, j.init_depth_random = o.num_iterations, int(o.geom_consistency), int(o.init_depth_random)
    j.local_opt, j.random_opt, j.num_samples, j.thk = int(o.local_optimization), int(o.random_optimization), \
        o.num_samples, o.thk
    j.good, j.bad = o.num_good_hypothesis, o.num_bad_hypothesis
    j.geom_reg, j.geom_max, j.rand_depth_ratio = o.geom_consistency_regularizer, o.geom_consistency_max_cost, \
        o.random_depth_ratio
    j.a1, j.a2, j.init_mc, j.max_mc = o.random_angle1_range, o.random_angle2_range, o.init_ncc_matching_cost, \
        o.max_ncc_matching_cost
    j.alpha, j.beta = o.alpha, o.beta
    if ref.depth is not None:
        d = np.ascontiguousarray(ref.depth, np.float32)
        keep.append(d)
        j.init_depth = d.ctypes.data
    if ref.normal is not None:
        n = np.ascontiguousarray(ref.normal, np.float32)
        keep.append(n)
        j.init_normal = n.ctypes.data
    if any(v.depth is not None for v in srcs):  # a source without a map is NULL (propagate_depth)
        ds = [None if v.depth is None else np.ascontiguousarray(v.depth, np.float32) for v in srcs]
        keep.extend(ds)
        da = (C.c_void_p * len(srcs))(*[None if a is None else a.ctypes.data for a in ds])
        keep.append(da)
        j.src_depth = C.cast(da, C.POINTER(C.c_void_p))
    j.prior_mode = 1 if o.has_prior_depth else (2 if o.propagate_depth else 0)
    if problem.prior_wgt is not None:
        w = np.ascontiguousarray(problem.prior_wgt, np.float32)
        keep.append(w)
        j.prior_wgt = w.ctypes.data
    return j


def run(options: PatchMatchOptions, problem: Problem, poses: np.ndarray) -> dict:
    keep = []
    j = _job(options, problem, poses, keep)
    H, W, Nn = j.H, j.W, j.N
    out = {"depth": np.zeros((H, W), np.float32), "normal": np.zeros((3, H, W), np.float32),
           "conf": np.zeros((H, W), np.float32), "cost": np.zeros((Nn, H, W), np.float32),
           "view_sel": np.zeros((H, W), np.uint32)}
    ro = RefOut(**{k: v.ctypes.data for k, v in out.items()})
    rc = lib().ref_run(C.byref(j), C.byref(ro))
    if rc != 0:
        raise RuntimeError(f"reference run failed (driver status {rc})")
    return out


def propagate_init(options: PatchMatchOptions, problem: Problem, poses: np.ndarray) -> dict:
    """The reference's propagate-depth initial maps (GenerateProjectDepthMaps,
    CompositeInitDepthMap, CompositeInitNormalMap) from the problem's given
    reference maps and source depth maps."""
    keep = []
    j = _job(options, problem, poses, keep)
    out = {"depth": np.zeros((j.H, j.W), np.float32), "normal": np.zeros((3, j.H, j.W), np.float32),
           "prior": np.zeros((j.H, j.W), np.float32)}
    rc = lib().ref_propagate_init(C.byref(j), out["depth"].ctypes.data, out["normal"].ctypes.data,
                                  out["prior"].ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference propagate init failed (driver status {rc})")
    return out


def run_filter(options: PatchMatchOptions, problem: Problem, poses: np.ndarray) -> np.ndarray:
    keep = []
    j = _job(options, problem, poses, keep)
    ref = problem.images[problem.ref_image_idx]
    d_in = np.ascontiguousarray(ref.depth, np.float32)
    out = np.zeros_like(d_in)
    min_cons = min(options.filter_min_num_consistent, j.N)
    if lib().ref_filter(C.byref(j), d_in.ctypes.data, min_cons, options.filter_geom_consistency_max_cost,
                        out.ctypes.data) != 0:
        raise RuntimeError("reference filter rejected the job")
    return out


# ---------------------------------------------------------------------------
# Cross-view filter through the reference's CrossFilterKernel /
# DeduplicFilterKernel. Views are oracle.oracle.FilterView; problems are
# (ref, [src, ...]) index pairs; pose records come from the CPU oracle.
# ---------------------------------------------------------------------------
def _cf_structs(views, problems, depths, codes):
    from oracle import oracle as O
    keep = []
    vs = (RefCfView * len(views))()
    for k, v in enumerate(views):
        d = np.ascontiguousarray(depths[k], np.float32)
        keep.append(d)
        vs[k].H, vs[k].W = d.shape
        vs[k].depth = d.ctypes.data
        if codes is not None and codes[k] is not None:
            c = np.ascontiguousarray(codes[k], np.uint32)
            keep.append(c)
            vs[k].code = c.ctypes.data
        vs[k].ref_flag = int(v.ref_flag)
    ps = (RefCfProblem * max(len(problems), 1))()
    for k, (ref, srcs) in enumerate(problems):
        arr = (C.c_int * max(len(srcs), 1))(*srcs)
        keep.append(arr)
        ps[k].ref, ps[k].num_src, ps[k].src = int(ref), len(srcs), C.cast(arr, C.POINTER(C.c_int))
        if srcs:
            refK, refiK, poses = O.cross_filter_poses(views, (ref, srcs))
            poses = np.ascontiguousarray(poses, np.float32)
            keep.append(poses)
            ps[k].poses = poses.ctypes.data
            ps[k].refK[:] = list(refK)
            ps[k].refiK[:] = list(refiK)
    return vs, ps, keep


def cross_filter(options: PatchMatchOptions, views, problems) -> dict:
    """{view index: refined map} from the reference's CrossFilterKernel."""
    from oracle import oracle as O
    codes = [None if v.normal is None else O.encode_normal_map(v.normal) for v in views]
    vs, ps, keep = _cf_structs(views, problems, [v.depth for v in views], codes)
    refined = {r: np.zeros(views[r].shape, np.float32) for r, s in problems if len(s) > 0}
    ptrs = (C.c_void_p * len(views))(*[refined[k].ctypes.data if k in refined else None for k in range(len(views))])
    rc = lib().ref_cross_filter(len(views), vs, len(problems), ps, options.filter_geom_consistency_max_cost,
                                options.max_normal_error, options.depth_diff_threshold,
                                options.filter_min_num_consistent, ptrs)
    if rc:
        raise RuntimeError(f"reference cross filter failed (driver status {rc})")
    return refined


def dedup(options: PatchMatchOptions, views, problems, refined: dict):
    """(visibility maps, {view index: delta map}) from the reference's
    DeduplicFilterKernel, on the dedup inputs ResetDepthMaps builds."""
    depths = [(refined[k] if k in refined else np.zeros(v.shape, np.float32)) if v.ref_flag else v.depth
              for k, v in enumerate(views)]
    vs, ps, keep = _cf_structs(views, problems, depths, None)
    vis = [np.zeros(v.shape, np.uint32) for v in views]
    delta = {r: np.zeros(views[r].shape, np.float32) for r, s in problems if len(s) > 0}
    vp = (C.c_void_p * len(views))(*[v.ctypes.data for v in vis])
    dp = (C.c_void_p * len(views))(*[delta[k].ctypes.data if k in delta else None for k in range(len(views))])
    rc = lib().ref_dedup(len(views), vs, len(problems), ps, options.filter_geom_consistency_max_cost,
                         options.depth_diff_threshold, options.filter_min_num_consistent, vp, dp)
    if rc:
        raise RuntimeError(f"reference dedup failed (driver status {rc})")
    return vis, delta
