"""Seeded synthetic multi-view scenes with analytic ground truth.

These stand in for the public MVS benchmarks the reference evaluates on
(ETH3D, Tanks and Temples, DTU), which are not available here. Each scene is
rendered by ray casting the analytic surface (no graphics API): grey images
quantised to integers 0..255 (returned as float32), ground-truth depth (z in
the camera frame) and normals (camera frame, facing the camera), and
cameras as (K, R, T) with x_cam = R x_world + T.

Scenes:
  * ``planes_scene``      — 3..8 random planes, depths 2..8 m, 3-octave value
                            noise; 1 reference + 4 sources at 640x480, f=500,
                            on a 30 degree arc with 0.3 m between neighbours.
  * ``heightfield_scene`` — a plane plus 20 seeded Gaussians, depths ~3..15 m,
                            per-view gain U[0.8, 1.2] and Gaussian noise
                            sigma=2; 1 + 10 views at 1600x1200, f=1200.
Sizes are parameters so tests can render small versions of the same scenes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class SceneView:
    image: np.ndarray          # H x W float32, integer grey 0..255
    K: np.ndarray              # 3x3
    R: np.ndarray              # 3x3 world-to-camera
    T: np.ndarray              # 3
    depth_gt: np.ndarray       # H x W float32 (0 where nothing was hit)
    normal_gt: np.ndarray      # 3 x H x W float32 (camera frame)


@dataclass
class Scene:
    views: list
    ref_index: int
    src_indices: list
    depth_min: float
    depth_max: float
    name: str = ""
    meta: dict = field(default_factory=dict)


def look_at(pos, target, up=(0.0, 0.0, 1.0)):
    pos = np.asarray(pos, np.float64)
    fwd = np.asarray(target, np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    R = np.stack([right, down, fwd])
    T = -R @ pos
    return R, T


def intrinsics(f, W, H):
    return np.array([[f, 0, (W - 1) / 2.0], [0, f, (H - 1) / 2.0], [0, 0, 1]], np.float64)


def _hash(ix: torch.Tensor, iy: torch.Tensor, salt: int) -> torch.Tensor:
    """Integer lattice hash -> [0, 1) (a multiply-xorshift mix on int64)."""
    m = (1 << 31) - 1
    h = (ix * 73856093) ^ (iy * 19349663) ^ torch.full_like(ix, (salt * 83492791) & m)
    h = h & m
    h = ((h ^ (h >> 13)) * 1274126177) & m
    h = (h ^ (h >> 16)) & m
    h = (h * 2654435761) & m
    h = (h ^ (h >> 15)) & m
    return h.to(torch.float64) / float(m)


def value_noise(u: torch.Tensor, v: torch.Tensor, salt: int, octaves: int = 3) -> torch.Tensor:
    """Band-limited value noise: smooth (quintic) interpolation of lattice
    values, octaves at doubling frequency and halving amplitude, in [0, 1]."""
    total = torch.zeros_like(u)
    norm = 0.0
    amp = 1.0
    for o in range(octaves):
        s = float(1 << o)
        x, y = u * s, v * s
        x0, y0 = torch.floor(x), torch.floor(y)
        fx, fy = x - x0, y - y0
        ix, iy = x0.to(torch.int64), y0.to(torch.int64)
        sx = fx * fx * fx * (fx * (fx * 6 - 15) + 10)
        sy = fy * fy * fy * (fy * (fy * 6 - 15) + 10)
        salt_o = salt * 31 + o
        v00 = _hash(ix, iy, salt_o)
        v10 = _hash(ix + 1, iy, salt_o)
        v01 = _hash(ix, iy + 1, salt_o)
        v11 = _hash(ix + 1, iy + 1, salt_o)
        a = v00 + (v10 - v00) * sx
        b = v01 + (v11 - v01) * sx
        total = total + amp * (a + (b - a) * sy)
        norm += amp
        amp *= 0.5
    return total / norm


def _pixel_rays(K, R, T, W, H, device):
    """Ray origins (3,) and unit directions (H, W, 3) in world coordinates, plus
    the camera-frame ray with z = 1 per pixel (for depth = t * (d . fwd))."""
    Ki = np.linalg.inv(K)
    ys, xs = torch.meshgrid(torch.arange(H, dtype=torch.float64, device=device),
                            torch.arange(W, dtype=torch.float64, device=device), indexing="ij")
    pc = torch.stack([xs, ys, torch.ones_like(xs)], -1) @ torch.tensor(Ki.T, device=device)  # z = 1
    Rt = torch.tensor(R.T, device=device)
    d = pc @ Rt.T  # world direction (not normalised; camera z component = 1)
    origin = torch.tensor(-R.T @ T, device=device)
    return origin, d, pc


def _finish_image(albedo: torch.Tensor, gen: np.random.Generator, gain_range, noise_sigma) -> np.ndarray:
    g = albedo * 255.0
    if gain_range is not None:
        g = g * float(gen.uniform(*gain_range))
    if noise_sigma:
        noise = torch.from_numpy(gen.normal(0.0, noise_sigma, size=tuple(g.shape))).to(g.device)
        g = g + noise
    g = torch.clamp(torch.round(g), 0, 255)
    return g.to(torch.float32).cpu().numpy()


def _camera_normals(n_world: torch.Tensor, R, pc: torch.Tensor) -> torch.Tensor:
    Rm = torch.tensor(R, device=n_world.device)
    n_cam = n_world @ Rm.T
    flip = (n_cam * pc).sum(-1, keepdim=True) > 0
    n_cam = torch.where(flip, -n_cam, n_cam)
    return n_cam


# ---------------------------------------------------------------------------
# Planes scene
# ---------------------------------------------------------------------------
def planes_scene(seed: int = 0, width: int = 640, height: int = 480, focal: float = 500.0, num_src: int = 4,
                 arc_degrees: float = 30.0, baseline: float = 0.3, device: str = "cpu") -> Scene:
    gen = np.random.default_rng(seed)
    centre = np.array([0.0, 0.0, 5.0])
    n_cams = num_src + 1
    # Cameras on a circular arc spanning `arc_degrees` with `baseline` between
    # neighbours; the arc is centred on the middle camera's optical axis and
    # every camera looks at the scene centre.
    step = math.radians(arc_degrees) / max(n_cams - 1, 1)
    radius = (baseline / 2.0) / math.sin(step / 2.0)
    arc_centre = np.array([0.0, 0.0, radius])
    cams = []
    for i in range(n_cams):
        a = (i - (n_cams - 1) / 2.0) * step
        pos = arc_centre + radius * np.array([math.sin(a), 0.0, -math.cos(a)])
        R, T = look_at(pos, centre, up=(0.0, -1.0, 0.0))
        cams.append((R, T))
    ref_index = (n_cams - 1) // 2
    # Planes in the reference camera's frame (the middle camera sits at the
    # origin looking down +z). Plane 0 is the unbounded background.
    n_planes = int(gen.integers(3, 9))
    planes = []
    for k in range(n_planes):
        if k == 0:
            depth = 8.0
            half = (np.inf, np.inf)
        else:
            depth = float(gen.uniform(2.0, 7.0))
            half = (float(gen.uniform(0.3, 1.2)) * depth / 4, float(gen.uniform(0.3, 1.2)) * depth / 4)
        tilt = math.radians(float(gen.uniform(0, 35 if k else 15)))
        az = float(gen.uniform(0, 2 * math.pi))
        n = np.array([math.sin(tilt) * math.cos(az), math.sin(tilt) * math.sin(az), -math.cos(tilt)])
        c = np.array([float(gen.uniform(-0.35, 0.35)) * depth, float(gen.uniform(-0.25, 0.25)) * depth, depth])
        u = np.cross(n, [0.0, 1.0, 0.0]); u /= np.linalg.norm(u)
        v = np.cross(n, u)
        planes.append((c, n, u, v, half, int(gen.integers(1, 1 << 30))))
    K = intrinsics(focal, width, height)
    views = []
    for (R, T) in cams:
        origin, d, pc = _pixel_rays(K, R, T, width, height, device)
        best_t = torch.full(d.shape[:2], float("inf"), dtype=torch.float64, device=device)
        albedo = torch.zeros_like(best_t)
        n_world = torch.zeros_like(d)
        for (c, n, u, v, half, salt) in planes:
            ct, nt = torch.tensor(c, device=device), torch.tensor(n, device=device)
            denom = d @ nt
            t = ((ct - origin) @ nt) / denom
            hit = origin + t[..., None] * d
            lu = (hit - ct) @ torch.tensor(u, device=device)
            lv = (hit - ct) @ torch.tensor(v, device=device)
            ok = (t > 0) & torch.isfinite(t)
            if np.isfinite(half[0]):
                ok = ok & (lu.abs() <= half[0]) & (lv.abs() <= half[1])
            closer = ok & (t < best_t)
            tex = 0.12 + 0.76 * value_noise(lu / 0.10, lv / 0.10, salt)
            best_t = torch.where(closer, t, best_t)
            albedo = torch.where(closer, tex, albedo)
            n_world = torch.where(closer[..., None], nt.expand_as(d), n_world)
        depth = torch.where(torch.isfinite(best_t), best_t, torch.zeros_like(best_t))  # camera z (pc.z == 1)
        normal = _camera_normals(n_world, R, pc)
        img = _finish_image(albedo, gen, None, 0.0)
        views.append(SceneView(img, K.copy(), R, T, depth.to(torch.float32).cpu().numpy(),
                               normal.permute(2, 0, 1).to(torch.float32).cpu().numpy()))
    src = [i for i in range(n_cams) if i != ref_index]
    d_ref = views[ref_index].depth_gt
    valid = d_ref[d_ref > 0]
    return Scene(views, ref_index, src, float(valid.min()) * 0.9, float(valid.max()) * 1.1,
                 name=f"planes(seed={seed},{width}x{height},N={num_src})", meta={"n_planes": n_planes})


# ---------------------------------------------------------------------------
# Heightfield scene
# ---------------------------------------------------------------------------
def _gaussians(gen, count=20, extent=6.0):
    cx = gen.uniform(-extent, extent, count)
    cy = gen.uniform(-extent, extent, count)
    amp = gen.uniform(0.25, 1.2, count)
    sig = gen.uniform(0.5, 2.0, count)
    return cx, cy, amp, sig


def _height(X, Y, g):
    cx, cy, amp, sig = g
    h = torch.zeros_like(X)
    hx = torch.zeros_like(X)
    hy = torch.zeros_like(X)
    for i in range(len(cx)):
        dx, dy = X - cx[i], Y - cy[i]
        e = amp[i] * torch.exp(-(dx * dx + dy * dy) / (2 * sig[i] ** 2))
        h = h + e
        hx = hx - e * dx / sig[i] ** 2
        hy = hy - e * dy / sig[i] ** 2
    return h, hx, hy


def _render_heightfield(cams, target, g, hmax, tex_salt, gen, gain_range, noise_sigma, device, chunk):
    """Ray-march the heightfield for cameras (position, width, height, focal),
    each looking at `target`; returns SceneViews."""
    views = []
    for pos, width, height, focal in cams:
        K = intrinsics(focal, width, height)
        R, T = look_at(pos, target)
        origin, d, pc = _pixel_rays(K, R, T, width, height, device)
        dflat = d.reshape(-1, 3)
        depth = torch.zeros(dflat.shape[0], dtype=torch.float64, device=device)
        albedo = torch.zeros_like(depth)
        nwl = torch.zeros_like(dflat)
        for s in range(0, dflat.shape[0], chunk):
            dd = dflat[s:s + chunk]
            # Enter the slab 0 <= Z <= hmax, march in 2 cm steps of Z-extent, bisect.
            dz = dd[:, 2]
            t_top = (hmax - origin[2]) / dz
            t_bot = (0.0 - origin[2]) / dz
            t0 = torch.clamp(torch.minimum(t_top, t_bot), min=0.0)
            t1 = torch.maximum(t_top, t_bot)
            n_steps = 160
            lo = t0.clone()
            hi = t1.clone()
            found = torch.zeros_like(t0, dtype=torch.bool)
            prev_t = t0.clone()
            for i in range(1, n_steps + 1):
                t = t0 + (t1 - t0) * (i / n_steps)
                P = origin + t[:, None] * dd
                h, _, _ = _height(P[:, 0], P[:, 1], g)
                below = (P[:, 2] <= h) & ~found
                lo = torch.where(below, prev_t, lo)
                hi = torch.where(below, t, hi)
                found = found | below
                prev_t = t
            for _ in range(30):
                mid = 0.5 * (lo + hi)
                P = origin + mid[:, None] * dd
                h, _, _ = _height(P[:, 0], P[:, 1], g)
                below = P[:, 2] <= h
                hi = torch.where(below, mid, hi)
                lo = torch.where(below, lo, mid)
            t = 0.5 * (lo + hi)
            P = origin + t[:, None] * dd
            _, hx, hy = _height(P[:, 0], P[:, 1], g)
            nrm = torch.stack([-hx, -hy, torch.ones_like(hx)], -1)
            nrm = nrm / nrm.norm(dim=-1, keepdim=True)
            depth[s:s + chunk] = torch.where(found, t, torch.zeros_like(t))  # camera z, since d.z_cam == 1
            albedo[s:s + chunk] = 0.12 + 0.76 * value_noise(P[:, 0] / 0.06, P[:, 1] / 0.06, tex_salt)
            nwl[s:s + chunk] = nrm
        depth = depth.reshape(height, width)
        normal = _camera_normals(nwl.reshape(height, width, 3), R, pc)
        img = _finish_image(albedo.reshape(height, width), gen, gain_range, noise_sigma)
        views.append(SceneView(img, K.copy(), R, T, depth.to(torch.float32).cpu().numpy(),
                               normal.permute(2, 0, 1).to(torch.float32).cpu().numpy()))
    return views


def heightfield_scene(seed: int = 0, width: int = 1600, height: int = 1200, focal: float = 1200.0,
                      num_src: int = 10, gain_range=(0.8, 1.2), noise_sigma: float = 2.0, distance: float = 7.0,
                      elevation_deg: float = 45.0, ring_radius: float = 0.8, device: str = "cpu",
                      chunk: int = 1 << 20) -> Scene:
    gen = np.random.default_rng(seed)
    g = _gaussians(gen)
    hmax = float(np.sum(g[2])) + 0.01
    target = np.array([0.0, 0.0, 0.0])
    el = math.radians(elevation_deg)
    ref_pos = target + distance * np.array([0.0, -math.cos(el), math.sin(el)])
    R0, _ = look_at(ref_pos, target)
    positions = [ref_pos]
    for k in range(num_src):
        a = 2 * math.pi * k / num_src
        positions.append(ref_pos + ring_radius * (math.cos(a) * R0[0] + math.sin(a) * R0[1]))
    tex_salt = int(gen.integers(1, 1 << 30))
    cams = [(pos, width, height, focal) for pos in positions]
    views = _render_heightfield(cams, target, g, hmax, tex_salt, gen, gain_range, noise_sigma, device, chunk)
    d_ref = views[0].depth_gt
    valid = d_ref[d_ref > 0]
    return Scene(views, 0, list(range(1, num_src + 1)), float(valid.min()) * 0.9, float(valid.max()) * 1.1,
                 name=f"heightfield(seed={seed},{width}x{height},N={num_src})")


def depth_accuracy(depth: np.ndarray, gt: np.ndarray, rel: float = 0.01) -> float:
    """Fraction of pixels with ground truth whose depth is within `rel` of it."""
    m = gt > 0
    return float(np.mean(np.abs(depth[m] - gt[m]) <= rel * gt[m]))


def normal_accuracy(normal: np.ndarray, gt: np.ndarray, degrees: float = 10.0, mask=None) -> float:
    """Fraction of pixels whose normal is within `degrees` of the ground truth (3 x H x W inputs)."""
    nn = normal / np.maximum(np.linalg.norm(normal, axis=0, keepdims=True), 1e-12)
    cosang = np.clip((nn * gt).sum(0), -1, 1)
    ok = cosang >= math.cos(math.radians(degrees))
    if mask is not None:
        ok = ok[mask]
    return float(np.mean(ok))


def noisy_maps(scene: Scene, seed: int = 0, rel_noise: float = 0.002, outlier_frac: float = 0.03,
               hole_frac: float = 0.02, normal_noise_deg: float = 3.0) -> list:
    """(depth, normal) per view: the scene's ground truth with the errors a
    PatchMatch pass leaves — relative depth noise, outliers drawn from
    [0.5, 1.5] x depth, holes (0) and perturbed normals. The input of the
    cross-view filter."""
    gen = np.random.default_rng(seed)
    out = []
    for v in scene.views:
        gt = v.depth_gt.astype(np.float64)
        d = gt * (1.0 + rel_noise * gen.standard_normal(gt.shape))
        u = gen.random(gt.shape)
        out_m = u < outlier_frac
        d[out_m] = gt[out_m] * gen.uniform(0.5, 1.5, size=int(out_m.sum()))
        d[(u >= outlier_frac) & (u < outlier_frac + hole_frac)] = 0.0
        d[gt <= 0] = 0.0
        n = v.normal_gt.astype(np.float64) + math.radians(normal_noise_deg) * gen.standard_normal(v.normal_gt.shape)
        n /= np.maximum(np.linalg.norm(n, axis=0, keepdims=True), 1e-12)
        out.append((d.astype(np.float32), n.astype(np.float32)))
    return out


def _backproject(v: SceneView, ys: np.ndarray, xs: np.ndarray, fy=None, fx=None) -> np.ndarray:
    """World points of pixels (ys, xs) of a view at their ground-truth depth,
    optionally at sub-pixel positions (ys + fy, xs + fx)."""
    d = v.depth_gt[ys, xs].astype(np.float64)
    Ki = np.linalg.inv(v.K)
    px = xs.astype(np.float64) + (0 if fx is None else fx)
    py = ys.astype(np.float64) + (0 if fy is None else fy)
    pc = np.stack([px, py, np.ones_like(px)], -1) @ Ki.T * d[:, None]
    return (pc - v.T) @ v.R  # R^T (x_cam - T)


def sparse_points(scene: Scene, view: int, count: int = 2000, seed: int = 0, noise: float = 0.002) -> np.ndarray:
    """Stand-in for the SfM points a view observes: surface points at random
    sub-pixel positions (away from pixel borders) at the ground-truth depth
    along the view's ray, with relative depth noise (n x 3 float32)."""
    gen = np.random.default_rng(seed)
    v = scene.views[view]
    H, W = v.depth_gt.shape
    ys, xs = gen.integers(0, H, count), gen.integers(0, W, count)
    ok = v.depth_gt[ys, xs] > 0
    ys, xs = ys[ok], xs[ok]
    fy, fx = gen.uniform(0.2, 0.8, len(ys)), gen.uniform(0.2, 0.8, len(ys))
    C = -v.R.T @ v.T
    X = _backproject(v, ys, xs, fy, fx)
    X = C + (X - C) * (1.0 + noise * gen.standard_normal(len(X)))[:, None]
    return X.astype(np.float32)


def grid_mesh(scene: Scene, view: int, step: int = 8, duplicate_frac: float = 0.0, seed: int = 0):
    """Stand-in for a prior TriangleMesh: the view's ground-truth surface on a
    grid of `step` pixels, two triangles per cell, wound so that they are front
    facing; face normals point to the camera. Returns (vertices n x 3 float64,
    faces m x 3 int32, face_normals m x 3 float64). A fraction of faces is
    repeated (shared-depth ties)."""
    gen = np.random.default_rng(seed)
    v = scene.views[view]
    H, W = v.depth_gt.shape
    gy, gx = np.meshgrid(np.arange(0, H, step), np.arange(0, W, step), indexing="ij")
    ny, nx = gy.shape
    X = _backproject(v, gy.ravel(), gx.ravel())
    valid = (v.depth_gt[gy, gx] > 0).ravel()
    idx = np.arange(ny * nx).reshape(ny, nx)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[:-1, 1:].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel()
    # Model2Depth draws a triangle when the pixel is right of all three edges
    # (m1, m2, m3 < 0, patch_match_controller.cc:598-601): (a, c, b), (b, c, d).
    faces = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)])
    faces = faces[valid[faces].all(1)]
    C = -v.R.T @ v.T
    p0, p1, p2 = X[faces[:, 0]], X[faces[:, 1]], X[faces[:, 2]]
    n = np.cross(p1 - p0, p2 - p0)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-300)
    flip = np.einsum("ij,ij->i", (p0 + p1 + p2) / 3 - C, n) > 0
    n[flip] *= -1
    if duplicate_frac > 0:
        rep = gen.random(len(faces)) < duplicate_frac
        faces = np.concatenate([faces, faces[rep]])
        n = np.concatenate([n, n[rep]])
        order = gen.permutation(len(faces))
        faces, n = faces[order], n[order]
    return X, faces.astype(np.int32), n


def dense_points(scene: Scene, view: int, step: int = 3, seed: int = 0, duplicate_frac: float = 0.0):
    """Stand-in for a fused point cloud (PlyPoint x/y/z, nx/ny/nz): ground-truth
    surface points of a view on a grid with world-frame normals facing the
    camera. A fraction of points is repeated with depths moved by 1e-9
    relative (ties in float, not in double)."""
    gen = np.random.default_rng(seed)
    v = scene.views[view]
    H, W = v.depth_gt.shape
    gy, gx = np.meshgrid(np.arange(1, H, step), np.arange(1, W, step), indexing="ij")
    gy, gx = gy.ravel(), gx.ravel()
    ok = v.depth_gt[gy, gx] > 0
    gy, gx = gy[ok], gx[ok]
    X = _backproject(v, gy, gx)
    n_cam = v.normal_gt[:, gy, gx].T.astype(np.float64)
    n_w = n_cam @ v.R  # R^T n
    if duplicate_frac > 0:
        rep = gen.random(len(X)) < duplicate_frac
        C = -v.R.T @ v.T
        X = np.concatenate([X, C + (X[rep] - C) * (1 + 1e-9 * gen.standard_normal(int(rep.sum())))[:, None]])
        n_w = np.concatenate([n_w, n_w[rep]])
        order = gen.permutation(len(X))
        X, n_w = X[order], n_w[order]
    return X.astype(np.float32), n_w.astype(np.float32)


def ring_model(num_cameras: int = 40, num_points: int = 3000, radius: float = 20.0, width: int = 1600,
               height: int = 1200, focal: float = 1200.0, seed: int = 0, drop: float = 0.2):
    """Stand-in for a sparse SfM model around a ring of cameras (like the batched
    workload's 200-camera ring, radius 20 m, heights 2-6 m): cameras look at the scene
    centre; points lie on a seeded terrain inside the ring; a point's track is
    the cameras it projects into, each observation dropped with probability
    `drop`. Returns (Rs, Ts, K, points n x 3 float32, tracks, is_rig)."""
    gen = np.random.default_rng(seed)
    K = intrinsics(focal, width, height)
    Rs, Ts = [], []
    for i in range(num_cameras):
        a = 2 * math.pi * i / num_cameras + gen.uniform(-0.02, 0.02)
        pos = np.array([radius * math.cos(a), radius * math.sin(a), gen.uniform(2.0, 6.0)])
        R, T = look_at(pos, (0.0, 0.0, 0.0))
        Rs.append(R)
        Ts.append(T)
    r = 12.0 * np.sqrt(gen.random(num_points))
    th = 2 * math.pi * gen.random(num_points)
    x, y = r * np.cos(th), r * np.sin(th)
    z = 0.8 * np.sin(0.4 * x) * np.cos(0.3 * y) + gen.uniform(0, 3.0, num_points) * (gen.random(num_points) < 0.2)
    P = np.stack([x, y, z], 1)
    tracks = [[] for _ in range(num_points)]
    for c in range(num_cameras):
        Xc = P @ Rs[c].T + Ts[c]
        uv = Xc @ K.T
        ok = Xc[:, 2] > 0.1
        u = uv[:, 0] / np.where(ok, uv[:, 2], 1)
        v = uv[:, 1] / np.where(ok, uv[:, 2], 1)
        ok &= (u >= 0) & (u < width) & (v >= 0) & (v < height) & (gen.random(num_points) >= drop)
        for i in np.nonzero(ok)[0]:
            tracks[i].append(c)
    is_rig = (np.arange(num_cameras) % 3 == 0)
    return Rs, Ts, K, P.astype(np.float32), tracks, is_rig


def ring_scene(seed: int = 0, num_cameras: int = 24, scale: float = 0.125, radius: float = 20.0,
               num_refs: int = 8, min_src: int = 5, max_src: int = 20, device: str = "cpu",
               gain_range=(0.8, 1.2), noise_sigma: float = 2.0):
    """Stand-in for the batched configuration: cameras on a ring (radius 20 m,
    heights 2-6 m) around the seeded heightfield, all looking at its centre,
    each of one of three sizes (800x600, 1600x1200, 3000x2000, times `scale`,
    focal 0.75 x width). `num_refs` reference views each take their k nearest
    cameras on the ring as sources, k drawn from [min_src, max_src]. Returns
    (Scene with every camera, [(ref, [src...]), ...])."""
    gen = np.random.default_rng(seed)
    g = _gaussians(gen)
    hmax = float(np.sum(g[2])) + 0.01
    target = np.array([0.0, 0.0, 0.0])
    sizes = [(800, 600), (1600, 1200), (3000, 2000)]
    cams = []
    for i in range(num_cameras):
        a = 2 * math.pi * i / num_cameras
        pos = np.array([radius * math.cos(a), radius * math.sin(a), float(gen.uniform(2.0, 6.0))])
        w, h = sizes[int(gen.integers(0, len(sizes)))]
        w, h = max(16, int(round(w * scale))), max(16, int(round(h * scale)))
        cams.append((pos, w, h, 0.75 * w))
    tex_salt = int(gen.integers(1, 1 << 30))
    views = _render_heightfield(cams, target, g, hmax, tex_salt, gen, gain_range, noise_sigma, device, 1 << 20)
    refs = sorted(gen.choice(num_cameras, size=min(num_refs, num_cameras), replace=False).tolist())
    jobs = []
    for r in refs:
        k = int(gen.integers(min_src, max_src + 1))
        k = min(k, num_cameras - 1)
        order = sorted((i for i in range(num_cameras) if i != r),
                       key=lambda i: (min(abs(i - r), num_cameras - abs(i - r)), i))
        jobs.append((r, order[:k]))
    depths = np.concatenate([v.depth_gt[v.depth_gt > 0] for v in views])
    return Scene(views, refs[0], jobs[0][1], float(depths.min()) * 0.9, float(depths.max()) * 1.1,
                 name=f"ring(seed={seed},{num_cameras} cameras,scale={scale})", meta={"jobs": jobs}), jobs


def fusion_inputs(scene: Scene, seed: int = 0, rel_noise: float = 0.002, outlier_frac: float = 0.03,
                  hole_frac: float = 0.02, normal_noise_deg: float = 3.0, rig_every: int = 0):
    """(images, overlapping_images) for StereoFusion: every view's noisy depth
    and normal maps (``noisy_maps``), an RGB bitmap made from the grey image
    (red = grey, green and blue shifted so the channels differ), and as the
    overlapping list of each view every other view, nearest camera centre
    first. With rig_every > 0 every rig_every-th view is flagged as a rig image."""
    from .fusion import FusionImage
    maps = noisy_maps(scene, seed=seed, rel_noise=rel_noise, outlier_frac=outlier_frac, hole_frac=hole_frac,
                      normal_noise_deg=normal_noise_deg)
    images = []
    centres = []
    for k, (v, (d, n)) in enumerate(zip(scene.views, maps)):
        g = np.clip(np.rint(v.image), 0, 255).astype(np.int32)
        rgb = np.stack([g, (g * 3 + 17) % 256, 255 - g], -1).astype(np.uint8)
        images.append(FusionImage(K=v.K, R=v.R, T=v.T, depth=d, normal=n, color=rgb,
                                  is_rig=bool(rig_every and k % rig_every == 0)))
        centres.append(-np.asarray(v.R, np.float64).T @ np.asarray(v.T, np.float64))
    centres = np.array(centres)
    overlaps = []
    for k in range(len(images)):
        dist = np.linalg.norm(centres - centres[k], axis=1)
        order = [int(i) for i in np.argsort(dist, kind="stable") if i != k]
        overlaps.append(order)
    return images, overlaps


# ---------------------------------------------------------------------------
# Aerial scene: terrain heightfield with box buildings (GPU ray-caster)
# ---------------------------------------------------------------------------
@dataclass
class DeviceView:
    """A view whose image and ground truth stay on the GPU (large view sets)."""
    image: torch.Tensor        # H x W float32 on the device, integer grey 0..255
    K: np.ndarray
    R: np.ndarray
    T: np.ndarray
    depth_gt: torch.Tensor     # H x W float32 on the device
    normal_gt: object = None   # 3 x H x W float32 on the device, or None
    kind: str = "nadir"

    @property
    def centre(self) -> np.ndarray:
        return -np.asarray(self.R, np.float64).T @ np.asarray(self.T, np.float64)

    @property
    def axis(self) -> np.ndarray:
        return np.asarray(self.R, np.float64)[2]


@dataclass
class AerialTerrain:
    hills: np.ndarray          # k x 4 float32: centre x, centre y, amplitude, sigma (m)
    boxes: np.ndarray          # m x 5 float32: x0, y0, x1, y1, roof height (m)
    salt: int
    texel: float               # albedo lattice spacing (m)
    step: float = 0.25         # ray-march step (m)
    max_dist: float = 400.0    # rays end this far from the camera (m)


def aerial_terrain(seed: int = 0, extent=(600.0, 500.0), num_hills: int = 24, num_boxes: int = 260,
                   texel: float = 0.15, max_height: float = 20.0) -> AerialTerrain:
    """Seeded terrain (a sum of Gaussian hills 30..120 m wide, scaled so that
    the highest point over the extent is `max_height` m) centred on the origin,
    with box buildings (footprints 8..30 m, 5..40 m tall above the terrain at
    their centre, not overlapping)."""
    gen = np.random.default_rng(seed)
    ex, ey = extent
    hills = np.stack([gen.uniform(-ex / 2, ex / 2, num_hills), gen.uniform(-ey / 2, ey / 2, num_hills),
                      gen.uniform(2.0, 15.0, num_hills), gen.uniform(30.0, 120.0, num_hills)], 1)
    gx, gy = np.meshgrid(np.linspace(-ex / 2, ex / 2, 121), np.linspace(-ey / 2, ey / 2, 101))
    peak = np.max(np.sum(hills[:, 2, None, None] * np.exp(-((gx[None] - hills[:, 0, None, None]) ** 2 +
                                                            (gy[None] - hills[:, 1, None, None]) ** 2)
                                                          / (2 * hills[:, 3, None, None] ** 2)), 0))
    hills[:, 2] *= max_height / max(peak, 1e-6)

    def terrain(x, y):
        return float(np.sum(hills[:, 2] * np.exp(-((x - hills[:, 0]) ** 2 + (y - hills[:, 1]) ** 2)
                                                  / (2 * hills[:, 3] ** 2))))

    boxes = []
    tries = 0
    while len(boxes) < num_boxes and tries < 50 * num_boxes:
        tries += 1
        w, h = gen.uniform(8.0, 30.0, 2)
        cx, cy = gen.uniform(-ex / 2 + w, ex / 2 - w), gen.uniform(-ey / 2 + h, ey / 2 - h)
        b = (cx - w / 2, cy - h / 2, cx + w / 2, cy + h / 2)
        if any(b[0] < o[2] + 2 and o[0] < b[2] + 2 and b[1] < o[3] + 2 and o[1] < b[3] + 2 for o in boxes):
            continue
        boxes.append((*b, terrain(cx, cy) + gen.uniform(5.0, 40.0)))
    return AerialTerrain(hills.astype(np.float32), np.array(boxes, np.float32).reshape(-1, 5),
                         int(gen.integers(1, 1 << 30)), texel)


def nadir_rotation() -> np.ndarray:
    """World-to-camera rotation of a camera looking straight down (image x along
    world x, image y along world -y)."""
    return np.array([[1.0, 0.0, 0.0], [0.0, -1.0, 0.0], [0.0, 0.0, -1.0]])


def render_aerial(terrain: AerialTerrain, K, R, T, width: int, height: int, stream=None):
    """(albedo in [0, 1], depth, normal) of one view as device tensors."""
    from . import _native as N
    import ctypes as C
    dev = torch.device("cuda")
    albedo = torch.empty((height, width), dtype=torch.float32, device=dev)
    depth = torch.empty_like(albedo)
    normal = torch.empty((3, height, width), dtype=torch.float32, device=dev)
    Kd = (C.c_double * 9)(*np.asarray(K, np.float64).reshape(9))
    Rd = (C.c_double * 9)(*np.asarray(R, np.float64).reshape(9))
    Td = (C.c_double * 3)(*np.asarray(T, np.float64).reshape(3))
    hills = np.ascontiguousarray(terrain.hills, np.float32)
    boxes = np.ascontiguousarray(terrain.boxes, np.float32)
    N.check(N.lib().smvs_synth_render_aerial(
        hills.ctypes.data, len(hills), boxes.ctypes.data if len(boxes) else None, len(boxes), terrain.salt,
        float(terrain.texel), float(terrain.step), float(terrain.max_dist), Kd, Rd, Td, width, height, albedo.data_ptr(), depth.data_ptr(), normal.data_ptr(),
        C.c_void_p(int(stream)) if stream is not None else None))
    return albedo, depth, normal


def _finish_image_device(albedo: torch.Tensor, gen: np.random.Generator, gain_range, noise_sigma) -> torch.Tensor:
    g = albedo * 255.0
    if gain_range is not None:
        g = g * float(gen.uniform(*gain_range))
    if noise_sigma:
        t = torch.Generator(device=g.device)
        t.manual_seed(int(gen.integers(0, 1 << 62)))
        g = g + noise_sigma * torch.randn(g.shape, generator=t, device=g.device, dtype=g.dtype)
    return torch.clamp(torch.round(g), 0, 255)


def aerial_grid_cameras(stations=(20, 20), altitude: float = 100.0, width: int = 2000, height: int = 1500,
                        focal: float = 2000.0, overlap: float = 0.8, tilt_deg: float = 45.0):
    """An aerial survey: a grid of stations at `altitude` spaced for `overlap`
    between neighbouring nadir footprints; at each station the camera is nadir
    or tilted by `tilt_deg` towards +x, +y, -x or -y, cycling over the five
    kinds. Returns [(K, R, T, kind)]."""
    K = intrinsics(focal, width, height)
    fx = width * altitude / focal
    fy = height * altitude / focal
    sx, sy = (1 - overlap) * fx, (1 - overlap) * fy
    nx, ny = stations
    cams = []
    kinds = ["nadir", "+x", "+y", "-x", "-y"]
    t = math.radians(tilt_deg)
    for j in range(ny):
        for i in range(nx):
            pos = np.array([(i - (nx - 1) / 2) * sx, (j - (ny - 1) / 2) * sy, altitude])
            kind = kinds[(i + 2 * j) % 5]
            if kind == "nadir":
                R = nadir_rotation()
            else:
                a = {"+x": 0.0, "+y": math.pi / 2, "-x": math.pi, "-y": -math.pi / 2}[kind]
                fwd = np.array([math.cos(a) * math.sin(t), math.sin(a) * math.sin(t), -math.cos(t)])
                R, _ = look_at(pos, pos + fwd)
            cams.append((K.copy(), R, -R @ pos, kind))
    return cams


def aerial_views(terrain: AerialTerrain, cams, seed: int = 0, gain_range=(0.8, 1.2), noise_sigma: float = 2.0,
                 normals: bool = False, stream=None) -> list:
    """Render cameras [(K, R, T, kind)] into DeviceViews."""
    gen = np.random.default_rng(seed)
    out = []
    for K, R, T, kind in cams:
        H_, W_ = int(round(2 * K[1, 2] + 1)), int(round(2 * K[0, 2] + 1))
        albedo, depth, normal = render_aerial(terrain, K, R, T, W_, H_, stream)
        img = _finish_image_device(albedo, gen, gain_range, noise_sigma)
        del albedo
        out.append(DeviceView(img, K, R, T, depth, normal if normals else None, kind))
    return out


def nearest_sources(views, ref: int, k: int, max_angle_deg: float = 50.0) -> list:
    """The k cameras nearest to view `ref` (camera centres) among those whose
    viewing directions are within max_angle_deg of its own."""
    c0, a0 = views[ref].centre, views[ref].axis
    cos_lim = math.cos(math.radians(max_angle_deg))
    cand = [i for i in range(len(views)) if i != ref and float(views[i].axis @ a0) >= cos_lim]
    cand.sort(key=lambda i: (float(np.linalg.norm(views[i].centre - c0)), i))
    return cand[:k]


def depth_range_of(view: DeviceView) -> tuple:
    d = view.depth_gt
    valid = d[d > 0]
    return float(valid.min()) * 0.9, float(valid.max()) * 1.1


def ring_terrain(seed: int = 0) -> AerialTerrain:
    """The heightfield of ``heightfield_scene`` (20 seeded Gaussians over a
    plane, extent 6 m) as a terrain for the GPU ray-caster, no buildings."""
    gen = np.random.default_rng(seed)
    cx, cy, amp, sig = _gaussians(gen)
    hills = np.stack([cx, cy, amp, sig], 1).astype(np.float32)
    return AerialTerrain(hills, np.zeros((0, 5), np.float32), int(gen.integers(1, 1 << 30)), 0.06, 0.02, 60.0)


def ring_cameras(num_cameras: int = 200, radius: float = 20.0, seed: int = 0):
    """Cameras on a ring (radius 20 m, heights 2..6 m) looking at the origin,
    each of one of three sizes (800x600, 1600x1200, 3000x2000; focal 0.75 x
    width). Returns [(K, R, T, kind)]."""
    gen = np.random.default_rng(seed + 1)
    sizes = [(800, 600), (1600, 1200), (3000, 2000)]
    cams = []
    for i in range(num_cameras):
        a = 2 * math.pi * i / num_cameras
        pos = np.array([radius * math.cos(a), radius * math.sin(a), float(gen.uniform(2.0, 6.0))])
        w, h = sizes[int(gen.integers(0, len(sizes)))]
        R, T = look_at(pos, (0.0, 0.0, 0.0))
        cams.append((intrinsics(0.75 * w, w, h), R, T, f"{w}x{h}"))
    return cams
