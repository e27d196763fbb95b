"""ctypes front end of the CPU oracle (test infrastructure only).

Mirrors sensemap_b200.patch_match's calling convention so tests can run the
same Problem through the CUDA engine and through the oracle.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from sensemap_b200 import _native as N
from sensemap_b200.patch_match import PatchMatchOptions, Problem

from . import build as _build

_LIB = None


class orc_outputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("depth", "normal", "conf", "cost", "view_sel", "grad", "ref_sum",
                                           "ref_sqsum", "poses", "curvature")]


def lib():
    global _LIB
    if _LIB is None:
        path = _build.build()
        h = C.CDLL(str(path))
        h.orc_run.restype = C.c_int
        h.orc_run.argtypes = [C.POINTER(N.smvs_options), C.POINTER(N.smvs_problem), C.c_int, C.c_int,
                              C.POINTER(orc_outputs)]
        h.orc_run_filter.restype = C.c_int
        h.orc_run_filter.argtypes = [C.POINTER(N.smvs_options), C.POINTER(N.smvs_problem), C.c_void_p]
        h.orc_eval_costs.restype = C.c_int
        h.orc_eval_costs.argtypes = [C.POINTER(N.smvs_options), C.POINTER(N.smvs_problem), C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_uniform.restype = C.c_float
        h.orc_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        h.orc_tex_bilinear.restype = C.c_float
        h.orc_tex_bilinear.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float]
        h.orc_num_threads.restype = C.c_int
        vp = C.POINTER(N.smvs_filter_view)
        pp = C.POINTER(N.smvs_filter_problem)
        h.orc_cross_filter_run.restype = C.c_int
        h.orc_cross_filter_run.argtypes = [C.POINTER(N.smvs_options), vp, C.c_int, pp, C.c_int, C.c_void_p]
        h.orc_cross_filter_dedup.restype = C.c_int
        h.orc_cross_filter_dedup.argtypes = [C.POINTER(N.smvs_options), vp, C.c_int, pp, C.c_int, C.c_void_p,
                                             C.c_void_p, C.c_void_p]
        h.orc_cross_filter_dedup_depth.restype = C.c_int
        h.orc_cross_filter_dedup_depth.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_encode_normal_map.restype = C.c_int
        h.orc_encode_normal_map.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        for name in ("orc_init_from_sparse_points", "orc_init_from_mesh", "orc_init_from_dense_points"):
            getattr(h, name).restype = C.c_int
        h.orc_init_from_sparse_points.argtypes = [C.POINTER(N.smvs_view), C.c_void_p, C.c_size_t, C.c_void_p,
                                                  C.c_void_p, C.c_void_p]
        h.orc_init_from_mesh.argtypes = [C.POINTER(N.smvs_view), C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_init_from_dense_points.argtypes = [C.POINTER(N.smvs_view), C.c_void_p, C.c_void_p, C.c_size_t, C.c_int,
                                                 C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_fusion_run.restype = C.c_void_p
        h.orc_fusion_run.argtypes = [C.POINTER(N.smvs_fusion_options), C.POINTER(N.smvs_fusion_view), C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_int]
        h.orc_fusion_run_threads.restype = C.c_void_p
        h.orc_fusion_run_threads.argtypes = [C.POINTER(N.smvs_fusion_options), C.POINTER(N.smvs_fusion_view), C.c_int,
                                             C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        h.orc_fusion_sizes.restype = C.c_int
        h.orc_fusion_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
        h.orc_fusion_copy.restype = C.c_int
        h.orc_fusion_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_fusion_mask.restype = C.c_int
        h.orc_fusion_mask.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        h.orc_fusion_duplicate_keep.restype = C.c_int
        h.orc_fusion_duplicate_keep.argtypes = [C.POINTER(N.smvs_fusion_view), C.c_int, C.c_void_p, C.c_size_t,
                                                C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_fusion_outlier_keep.restype = C.c_int
        h.orc_fusion_outlier_keep.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_double, C.c_void_p, C.c_void_p,
                                              C.c_void_p]
        h.orc_fusion_free.restype = None
        h.orc_fusion_free.argtypes = [C.c_void_p]
        h.orc_delaunay_points.restype = C.c_int
        h.orc_delaunay_points.argtypes = [C.POINTER(N.smvs_view), C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.POINTER(C.c_size_t)]
        h.orc_init_from_delaunay.restype = C.c_int
        h.orc_init_from_delaunay.argtypes = [C.POINTER(N.smvs_view), C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                             C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_resample_maps.restype = C.c_int
        h.orc_resample_maps.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
        h.orc_rescale_image.restype = C.c_int
        h.orc_rescale_image.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        h.orc_propagate_init_problem.restype = C.c_int
        h.orc_propagate_init_problem.argtypes = [C.POINTER(N.smvs_problem), C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_cross_filter_poses.restype = C.c_int
        h.orc_cross_filter_poses.argtypes = [vp, C.c_int, pp, C.c_void_p, C.c_void_p, C.c_void_p]
        _LIB = h
    return _LIB


def _problem_struct(problem: Problem):
    keep = []

    def fill(cv, v, scale):
        img = np.asarray(v.image)
        if img.dtype == np.uint8:
            fmt = N.PIX_U8
        else:
            img = np.ascontiguousarray(img, dtype=np.float32)
            fmt = N.PIX_F32
        img = np.ascontiguousarray(img)
        keep.append(img)
        cv.width, cv.height, cv.pixel_format, cv.row_stride = img.shape[1], img.shape[0], fmt, 0
        cv.pixels = img.ctypes.data
        cv.K[:] = list(np.asarray(v.K, np.float64).reshape(9))
        cv.R[:] = list(np.asarray(v.R, np.float64).reshape(9))
        cv.T[:] = list(np.asarray(v.T, np.float64).reshape(3))
        cv.scale = float(scale)
        for name in ("depth", "normal"):
            arr = getattr(v, name)
            if arr is None:
                setattr(cv, name, None)
            else:
                a = np.ascontiguousarray(arr, dtype=np.float32)
                keep.append(a)
                setattr(cv, name, a.ctypes.data)

    prob = N.smvs_problem()
    fill(prob.ref, problem.images[problem.ref_image_idx], 1.0)
    srcs = (N.smvs_view * len(problem.src_image_idxs))()
    scales = list(problem.src_image_scales) or [1.0] * len(problem.src_image_idxs)
    for i, idx in enumerate(problem.src_image_idxs):
        fill(srcs[i], problem.images[idx], scales[i])
    keep.append(srcs)
    prob.src = srcs
    prob.num_src = len(problem.src_image_idxs)
    if problem.mask is not None:
        m = np.ascontiguousarray(problem.mask, dtype=np.uint8)
        keep.append(m)
        prob.ref_mask = m.ctypes.data
    if problem.prior_wgt is not None:
        w = np.ascontiguousarray(problem.prior_wgt, dtype=np.float32)
        keep.append(w)
        prob.ref_prior_wgt = w.ctypes.data
    prob.memory = N.MEM_HOST
    return prob, keep


def propagate_init(problem: Problem) -> dict:
    """The oracle's propagate-depth initial maps (InitWorkspace,
    patch_match_cuda.cu:603-659) from the problem's given reference maps and
    source depth maps: depth, normal (3 x H x W) and prior depth."""
    prob, keep = _problem_struct(problem)
    ref = problem.images[problem.ref_image_idx]
    out = {"depth": np.zeros((ref.height, ref.width), np.float32),
           "normal": np.zeros((3, ref.height, ref.width), np.float32),
           "prior": np.zeros((ref.height, ref.width), np.float32)}
    rc = lib().orc_propagate_init_problem(C.byref(prob), out["depth"].ctypes.data, out["normal"].ctypes.data,
                                          out["prior"].ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle propagate init failed ({rc})")
    return out


def run(options: PatchMatchOptions, problem: Problem, rows=None) -> dict:
    """The oracle's PatchMatchACMMCuda(options, problem).Run(); returns all maps."""
    prob, keep = _problem_struct(problem)
    ref = problem.images[problem.ref_image_idx]
    H, W, Nn = ref.height, ref.width, len(problem.src_image_idxs)
    out = {"depth": np.zeros((H, W), np.float32), "normal": np.zeros((3, H, W), np.float32),
           "conf": np.zeros((H, W), np.float32), "cost": np.zeros((Nn, H, W), np.float32),
           "view_sel": np.zeros((H, W), np.uint32), "grad": np.zeros((H, W), np.float32),
           "ref_sum": np.zeros((H, W), np.float32), "ref_sqsum": np.zeros((H, W), np.float32),
           "poses": np.zeros((Nn, 43), np.float32), "curvature": np.zeros((2, H, W), np.uint16)}
    oo = orc_outputs(**{k: v.ctypes.data for k, v in out.items()})
    r0, r1 = (0, 0) if rows is None else rows
    st = lib().orc_run(C.byref(options.to_c()), C.byref(prob), r0, r1, C.byref(oo))
    if st != 0:
        raise N.SmvsError(st, "oracle run failed")
    return out


def run_filter(options: PatchMatchOptions, problem: Problem) -> np.ndarray:
    prob, keep = _problem_struct(problem)
    ref = problem.images[problem.ref_image_idx]
    out = np.zeros((ref.height, ref.width), np.float32)
    st = lib().orc_run_filter(C.byref(options.to_c()), C.byref(prob), out.ctypes.data)
    if st != 0:
        raise N.SmvsError(st, "oracle filter failed")
    return out


def eval_costs(options: PatchMatchOptions, problem: Problem, rows, cols, depths, normals):
    """FP32 transcription and FP64 evaluation of the NCC cost of one hypothesis
    per sampled pixel, for every source view: (n, N) float32, (n, N) float64."""
    prob, keep = _problem_struct(problem)
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    depths = np.ascontiguousarray(depths, np.float32)
    normals = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
    n = rows.shape[0]
    Nn = len(problem.src_image_idxs)
    c32 = np.zeros((n, Nn), np.float32)
    c64 = np.zeros((n, Nn), np.float64)
    st = lib().orc_eval_costs(C.byref(options.to_c()), C.byref(prob), n, rows.ctypes.data, cols.ctypes.data,
                              depths.ctypes.data, normals.ctypes.data, c32.ctypes.data, c64.ctypes.data)
    if st != 0:
        raise N.SmvsError(st, "oracle eval failed")
    return c32, c64


def uniform(seed: int, stage: int, pixel: int, draw: int) -> float:
    return float(lib().orc_uniform(seed, stage, pixel, draw))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---------------------------------------------------------------------------
# Cross-view filter (CrossFilterCuda). A view set is a list of FilterView and
# problems are (ref, [src, ...]) pairs of indices into it.
# ---------------------------------------------------------------------------
class FilterView:
    def __init__(self, K, R, T, depth, normal=None, ref_flag=False):
        self.K, self.R, self.T = K, R, T
        self.depth = np.ascontiguousarray(depth, dtype=np.float32)
        self.normal = None if normal is None else np.ascontiguousarray(normal, dtype=np.float32)
        self.ref_flag = bool(ref_flag)

    @property
    def shape(self):
        return self.depth.shape


def _filter_structs(views, problems):
    keep = []
    vs = (N.smvs_filter_view * len(views))()
    for k, v in enumerate(views):
        cv = vs[k]
        cv.height, cv.width = v.depth.shape
        cv.K[:] = list(np.asarray(v.K, np.float64).reshape(9))
        cv.R[:] = list(np.asarray(v.R, np.float64).reshape(9))
        cv.T[:] = list(np.asarray(v.T, np.float64).reshape(3))
        cv.depth = v.depth.ctypes.data
        cv.normal = None if v.normal is None else v.normal.ctypes.data
        cv.ref_flag = int(v.ref_flag)
    ps = (N.smvs_filter_problem * max(len(problems), 1))()
    for k, (ref, srcs) in enumerate(problems):
        arr = (C.c_int * max(len(srcs), 1))(*srcs)
        keep.append(arr)
        ps[k].ref, ps[k].src, ps[k].num_src = int(ref), C.cast(arr, C.POINTER(C.c_int)), len(srcs)
    return vs, ps, keep


def cross_filter_run(options: PatchMatchOptions, views, problems) -> dict:
    """{view index: refined map} for every problem with at least one source."""
    vs, ps, keep = _filter_structs(views, problems)
    refined = {r: np.zeros(views[r].shape, np.float32) for r, s in problems if len(s) > 0}
    ptrs = (C.c_void_p * len(views))(*[refined[k].ctypes.data if k in refined else None for k in range(len(views))])
    st = lib().orc_cross_filter_run(C.byref(options.to_c()), vs, len(views), ps, len(problems), ptrs)
    if st:
        raise RuntimeError(f"orc_cross_filter_run failed ({st})")
    return refined


def cross_filter_dedup(options: PatchMatchOptions, views, problems, refined: dict):
    """(visibility maps of every view, {view index: delta map})."""
    vs, ps, keep = _filter_structs(views, problems)
    vis = [np.zeros(v.shape, np.uint32) for v in views]
    delta = {r: np.zeros(views[r].shape, np.float32) for r, s in problems if len(s) > 0}
    rp = (C.c_void_p * len(views))(*[refined[k].ctypes.data if k in refined else None for k in range(len(views))])
    vp = (C.c_void_p * len(views))(*[v.ctypes.data for v in vis])
    dp = (C.c_void_p * len(views))(*[delta[k].ctypes.data if k in delta else None for k in range(len(views))])
    st = lib().orc_cross_filter_dedup(C.byref(options.to_c()), vs, len(views), ps, len(problems), rp, vp, dp)
    if st:
        raise RuntimeError(f"orc_cross_filter_dedup failed ({st})")
    return vis, delta


def cross_filter_dedup_depth(view: FilterView, refined, vis) -> np.ndarray:
    vs, _, keep = _filter_structs([view], [])
    out = np.zeros(view.shape, np.float32)
    r = None if refined is None else np.ascontiguousarray(refined, dtype=np.float32)
    st = lib().orc_cross_filter_dedup_depth(vs, None if r is None else r.ctypes.data,
                                            np.ascontiguousarray(vis, dtype=np.uint32).ctypes.data, out.ctypes.data)
    if st:
        raise RuntimeError(f"orc_cross_filter_dedup_depth failed ({st})")
    return out


def cross_filter_poses(views, problem):
    """(refK[4], refiK[4], poses[num_src, 43]) of one problem."""
    vs, ps, keep = _filter_structs(views, [problem])
    refK, refiK = np.zeros(4, np.float32), np.zeros(4, np.float32)
    poses = np.zeros((max(len(problem[1]), 1), N.SMVS_POSE_FLOATS), np.float32)
    st = lib().orc_cross_filter_poses(vs, len(views), ps, refK.ctypes.data, refiK.ctypes.data, poses.ctypes.data)
    if st:
        raise RuntimeError(f"orc_cross_filter_poses failed ({st})")
    return refK, refiK, poses[:len(problem[1])]


def encode_normal_map(normal) -> np.ndarray:
    """NormalMap::Encode of a 3 x H x W map (uint32 H x W)."""
    n = np.ascontiguousarray(normal, dtype=np.float32)
    out = np.zeros(n.shape[1:], np.uint32)
    if lib().orc_encode_normal_map(n.ctypes.data, n.shape[2], n.shape[1], out.ctypes.data):
        raise RuntimeError("orc_encode_normal_map failed")
    return out


# ---------------------------------------------------------------------------
# Initial maps from the model (InitDepthMap / Model2Depth / Ply2Depth).
# ---------------------------------------------------------------------------
def _init_view(width, height, K, R, T):
    from sensemap_b200.init_maps import _view
    return _view(width, height, K, R, T)


def _init_out(width, height):
    return np.zeros((height, width), np.float32), np.zeros((3, height, width), np.float32), np.zeros(2, np.float32)


def init_from_sparse_points(width, height, K, R, T, xyz):
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    d, n, r = _init_out(width, height)
    if lib().orc_init_from_sparse_points(C.byref(_init_view(width, height, K, R, T)), x.ctypes.data, len(x),
                                         d.ctypes.data, n.ctypes.data, r.ctypes.data):
        raise RuntimeError("orc_init_from_sparse_points failed")
    return d, n, (r[0], r[1])


def delaunay_points(width, height, K, R, T, xyz):
    """The projected points that land in the view (input order): (uv (m, 2)
    int32 truncated pixel positions, z (m,), input indices (m,))."""
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    uv = np.zeros((max(len(x), 1), 2), np.int32)
    z = np.zeros(max(len(x), 1), np.float32)
    idx = np.zeros(max(len(x), 1), np.int32)
    m = C.c_size_t()
    if lib().orc_delaunay_points(C.byref(_init_view(width, height, K, R, T)), x.ctypes.data, len(x), uv.ctypes.data,
                                 z.ctypes.data, idx.ctypes.data, C.byref(m)):
        raise RuntimeError("orc_delaunay_points failed")
    return uv[:m.value], z[:m.value], idx[:m.value]


def init_from_delaunay(width, height, K, R, T, xyz, tris):
    """InitDepthMapFromDelaunay over a given triangulation (index triples into
    the delaunay_points list)."""
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    d, n, r = _init_out(width, height)
    if lib().orc_init_from_delaunay(C.byref(_init_view(width, height, K, R, T)), x.ctypes.data, len(x),
                                    t.ctypes.data if len(t) else None, len(t), d.ctypes.data, n.ctypes.data,
                                    r.ctypes.data):
        raise RuntimeError("orc_init_from_delaunay failed")
    return d, n, (r[0], r[1])


def init_from_mesh(width, height, K, R, T, vertices, faces, face_normals):
    v = np.ascontiguousarray(vertices, np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.int32).reshape(-1, 3)
    fn = np.ascontiguousarray(face_normals, np.float64).reshape(-1, 3)
    d, n, r = _init_out(width, height)
    if lib().orc_init_from_mesh(C.byref(_init_view(width, height, K, R, T)), v.ctypes.data, len(v), f.ctypes.data,
                                len(f), fn.ctypes.data, d.ctypes.data, n.ctypes.data, r.ctypes.data):
        raise RuntimeError("orc_init_from_mesh failed")
    return d, n, (r[0], r[1])


def init_from_dense_points(width, height, K, R, T, xyz, normals, level=2):
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    nn = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
    d, n, r = _init_out(width, height)
    if lib().orc_init_from_dense_points(C.byref(_init_view(width, height, K, R, T)), x.ctypes.data, nn.ctypes.data,
                                        len(x), int(level), d.ctypes.data, n.ctypes.data, r.ctypes.data):
        raise RuntimeError("orc_init_from_dense_points failed")
    return d, n, (r[0], r[1])


def fusion_run(options, images, overlapping_images, max_images: int = 0, masks: bool = True,
               threads: int = 1) -> dict:
    """StereoFusion's image loop on the CPU (smvs_oracle_fusion.c) with the
    arguments of sensemap_b200.fusion.StereoFusion: points (structured array),
    visibility CSR (vis_offsets, vis_images), the image order and each image's
    fused-pixel mask. threads > 1 runs the reference's concurrent row slices
    (for timing only: the result then depends on the timing)."""
    from sensemap_b200.fusion import fusion_structs
    views, off, flat, memory, keep = fusion_structs(images, overlapping_images)
    if memory != N.MEM_HOST:
        raise ValueError("the oracle reads host arrays")
    h = lib().orc_fusion_run_threads(C.byref(options.to_c()), views, len(images), off.ctypes.data,
                                     flat.ctypes.data, int(max_images), int(threads))
    if not h:
        raise ValueError("orc_fusion_run rejected its arguments")
    try:
        npts, nvis, nord = C.c_size_t(), C.c_size_t(), C.c_int()
        lib().orc_fusion_sizes(h, C.byref(npts), C.byref(nvis), C.byref(nord))
        pts = np.zeros(npts.value, dtype=N.FUSED_POINT_DTYPE)
        voff = np.zeros(npts.value + 1, dtype=np.uint64)
        vis = np.zeros(max(nvis.value, 1), dtype=np.uint32)
        order = np.zeros(max(nord.value, 1), dtype=np.int32)
        lib().orc_fusion_copy(h, pts.ctypes.data, voff.ctypes.data, vis.ctypes.data, order.ctypes.data)
        out = {"points": pts, "vis_offsets": voff, "vis_images": vis[:nvis.value],
               "order": [int(i) for i in order[:nord.value]]}
        if masks:
            out["masks"] = []
            for k, v in enumerate(views):
                m = np.zeros((v.height, v.width), dtype=np.uint8)
                lib().orc_fusion_mask(h, k, v.width, v.height, m.ctypes.data)
                out["masks"].append(m)
        return out
    finally:
        lib().orc_fusion_free(h)


def _compact(pts, off, vis, keep):
    keep = keep.astype(bool)
    counts = np.diff(off.astype(np.int64))
    new_off = np.zeros(int(keep.sum()) + 1, dtype=np.uint64)
    new_off[1:] = np.cumsum(counts[keep])
    vmask = np.repeat(keep, counts)
    return pts[keep].copy(), new_off, vis[:len(vmask)][vmask].copy()


def fusion_remove_duplicates(images, pts, off, vis):
    """RemoveDuplicatePoints (smvs_oracle_fusion.c) over a fused cloud: the
    kept (points, offsets, images) and the number dropped."""
    from sensemap_b200.fusion import fusion_structs
    views, _, _, _, alive = fusion_structs(images, [[] for _ in images])
    pts = np.ascontiguousarray(pts)
    off = np.ascontiguousarray(off, dtype=np.uint64)
    vis = np.ascontiguousarray(vis, dtype=np.uint32)
    keep = np.zeros(len(pts), dtype=np.uint8)
    if lib().orc_fusion_duplicate_keep(views, len(images), pts.ctypes.data, len(pts), off.ctypes.data,
                                       vis.ctypes.data, keep.ctypes.data) != 0:
        raise ValueError("orc_fusion_duplicate_keep rejected its arguments")
    return _compact(pts, off, vis, keep) + (int(len(pts) - keep.sum()),)


def fusion_remove_outliers(pts, off, vis, nb_neighbors=6, max_spacing_factor=6.0):
    """RemoveOutliers (smvs_oracle_fusion.c, brute-force neighbours): the kept
    (points with updated scores, offsets, images), the number dropped and the
    per-point spacings."""
    pts = np.ascontiguousarray(pts).copy()
    scores = np.ascontiguousarray(pts["score"], dtype=np.float32).copy()
    keep = np.zeros(len(pts), dtype=np.uint8)
    spacing = np.zeros(len(pts), dtype=np.float32)
    if lib().orc_fusion_outlier_keep(pts.ctypes.data, len(pts), int(nb_neighbors), float(max_spacing_factor),
                                     scores.ctypes.data, keep.ctypes.data, spacing.ctypes.data) != 0:
        raise ValueError("orc_fusion_outlier_keep rejected its arguments")
    pts["score"] = scores
    kp, ko, kv = _compact(pts, np.ascontiguousarray(off, dtype=np.uint64), np.ascontiguousarray(vis, dtype=np.uint32),
                          keep)
    return kp, ko, kv, int(len(pts) - keep.sum()), spacing


def resample_maps(planes: np.ndarray, new_h: int, new_w: int, renormalise: bool) -> np.ndarray:
    """ResampleImageBilinear of a (P, H, W) float32 stack (+ normal re-normalisation)."""
    a = np.ascontiguousarray(planes, np.float32)
    P, H, W = a.shape
    out = np.zeros((P, new_h, new_w), np.float32)
    if lib().orc_resample_maps(a.ctypes.data, H, W, P, int(renormalise), out.ctypes.data, new_h, new_w) != 0:
        raise ValueError("orc_resample_maps rejected its arguments")
    return out


def rescale_image(image: np.ndarray, new_h: int, new_w: int) -> np.ndarray:
    """The bilinear-filter image rescale (grey 0..255 float32)."""
    a = np.ascontiguousarray(image, np.float32)
    H, W = a.shape
    tmp = np.zeros((H, new_w), np.float32)
    out = np.zeros((new_h, new_w), np.float32)
    if lib().orc_rescale_image(a.ctypes.data, W, H, tmp.ctypes.data, out.ctypes.data, new_w, new_h) != 0:
        raise ValueError("orc_rescale_image rejected its arguments")
    return out
