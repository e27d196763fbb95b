"""Shared test helpers: scenes -> Problems, and comparison statistics."""
from __future__ import annotations

import numpy as np

from sensemap_b200 import synthetic as syn
from sensemap_b200.patch_match import PatchMatchOptions, Problem, View


def problem_from_scene(scene, ref=None, src=None, depth_maps=None, normal_maps=None, init=None):
    """Problem over all scene views. depth_maps/normal_maps: per-view lists
    (source views' maps for the geometric pass); init: (depth, normal) of the ref."""
    ref = scene.ref_index if ref is None else ref
    src = [i for i in range(len(scene.views)) if i != ref] if src is None else src
    views = []
    for i, v in enumerate(scene.views):
        d = depth_maps[i] if depth_maps is not None else None
        n = normal_maps[i] if normal_maps is not None else None
        views.append(View(v.image, v.K, v.R, v.T, depth=d, normal=n))
    if init is not None:
        views[ref].depth, views[ref].normal = init
    return Problem(ref, src, views)


def small_planes(seed=0, w=160, h=120, f=125.0, n_src=4):
    return syn.planes_scene(seed=seed, width=w, height=h, focal=f, num_src=n_src)


def photometric_options(scene, iters=6, **kw):
    o = PatchMatchOptions(depth_min=scene.depth_min, depth_max=scene.depth_max, window_radius=5, window_step=1,
                          num_iterations=iters, geom_consistency=False, init_depth_random=True)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def perturbed_gt(scene, seed=1, rel=0.05, ang_deg=10.0, ref=None):
    """GT depth/normal of the ref view, perturbed (depth x (1 +- rel), normal
    tilted up to ang_deg), with every normal facing its camera ray."""
    ref = scene.ref_index if ref is None else ref
    v = scene.views[ref]
    rng = np.random.default_rng(seed)
    d = v.depth_gt * (1 + rng.uniform(-rel, rel, v.depth_gt.shape)).astype(np.float32)
    n = v.normal_gt + rng.normal(0, np.tan(np.radians(ang_deg)) / 2, v.normal_gt.shape).astype(np.float32)
    n /= np.linalg.norm(n, axis=0, keepdims=True)
    H, W = d.shape
    Ki = np.linalg.inv(v.K)
    ys, xs = np.mgrid[0:H, 0:W]
    ray = np.stack([Ki[0, 0] * xs + Ki[0, 2], Ki[1, 1] * ys + Ki[1, 2], np.ones_like(xs, dtype=np.float64)])
    flip = (n * ray).sum(0) >= 0
    n[:, flip] *= -1
    return d.astype(np.float32), n.astype(np.float32)


def frac_close(a, b, rel=0.01, mask=None):
    ok = np.abs(a - b) <= rel * np.abs(b)
    if mask is not None:
        ok = ok[mask]
    return float(np.mean(ok))


def filter_set(seed=0, w=160, h=120, f=125.0, n_views=6, ref_flags=None, neighbours=None, **noise):
    """A cross-filter view set from a planes scene: (scene, oracle FilterViews,
    problems as (ref, [src...]) with every view a reference of all others
    unless `neighbours` (a per-view source list) is given)."""
    from oracle import oracle as O
    scene = syn.planes_scene(seed=seed, width=w, height=h, focal=f, num_src=n_views - 1)
    maps = syn.noisy_maps(scene, seed=seed + 100, **noise)
    flags = [True] * n_views if ref_flags is None else ref_flags
    views = [O.FilterView(v.K, v.R, v.T, d, n, ref_flag=fl) for v, (d, n), fl in zip(scene.views, maps, flags)]
    if neighbours is None:
        neighbours = [[s for s in range(n_views) if s != r] for r in range(n_views)]
    problems = [(r, list(nb)) for r, nb in enumerate(neighbours)]
    return scene, views, problems


def filter_api_inputs(views, problems, device=False):
    """The same set as CrossFilterCuda arguments: (problems, whole_ids, ref_flags)
    over View objects (image ids = set indices)."""
    import torch
    ims = []
    for v in views:
        d, n = v.depth, v.normal
        if device:
            d = torch.from_numpy(d).cuda()
            n = None if n is None else torch.from_numpy(n).cuda()
        ims.append(View(None, v.K, v.R, v.T, depth=d, normal=n))
    probs = [Problem(r, [], ims, src_image_extend_idxs=list(s)) for r, s in problems]
    return probs, list(range(len(views))), [v.ref_flag for v in views]
