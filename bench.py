"""Benchmark: PatchMatch depth maps/s at 1600x1200 with 10 source views.

Workload (one step): a seeded synthetic heightfield scene of 11 views at
1600x1200 (f=1200, per-view gain, noise sigma=2). Every view is a reference
view once: a photometric PatchMatch pass (random init, 6 iterations, window
radius 5, step 1) against the other 10 views, then a geometric-consistency
pass (initialised from its photometric maps, the 10 sources' photometric
depth maps as the geometric term) — 11 depth maps per step.

  value  device-resident: images already in HBM; engines read them there and
         chain maps on the device; timed with CUDA events on the launching
         stream, max over ranks.
  e2e    the same step through the reference-facing API with host buffers:
         pinned host images in, depth/normal maps back to host every pass.

Under torchrun every rank runs its own scene replica (different seed): the
reference views shard across GPUs with no data-path collective ("weak").
``--impl reference`` times the CPU oracle (OpenMP transcription of the
reference kernel logic; the reference itself has no CPU PatchMatch) on a
bounded band of the same workload, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W, H, NSRC, ITERS, RADIUS, STEP = 1600, 1200, 10, 6, 5, 1
HYP_PER_PIXEL = 14          # 10 propagated + 4 refinement hypotheses per pixel per iteration
FLOP_PER_TAP = 25           # incremental warp, 1/z, bilinear, 4 moment updates
METRIC = "depth maps/s (1.6MP,10 src)"
CPU_BAND_ROWS = 16         # rows of the CPU oracle's band sample (both passes)
# DRAM bytes (read + write) of one sweep launch of the bench workload per source
# storage, from ncu (dram__bytes_read.sum + dram__bytes_write.sum of one
# SweepKernelL<5,1,12> launch, profiles/sweep_kernel_1600x1200_n10_f16.md).
SWEEP_DRAM_BYTES: dict = {"f16": 0.548e9 + 0.587e9}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 3; 200 for the cross-filter workload, whose step is milliseconds)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f16", choices=["u8", "f16", "f32"],
                    help="source image storage: f16 = precision form (FP16 storage, FP32 accumulation), "
                         "f32 = plain FP32 path, u8 = the reference's 8-bit texture format")
    ap.add_argument("--views", type=int, default=NSRC + 1, help="views per scene (each is a reference once)")
    ap.add_argument("--width", type=int, default=W)
    ap.add_argument("--height", type=int, default=H)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mode", default="batched", choices=["batched", "engine"],
                    help="batched: views resident once, all jobs of a pass in one batch (smvs_pool); "
                         "engine: one smvs_create/smvs_run per reference view and pass")
    ap.add_argument("--serving-seconds", type=float, default=10.0,
                    help="length of the Poisson-arrival serving measurement (0 = skip)")
    ap.add_argument("--serving-rate", type=float, default=2.0, help="job arrivals per second")
    ap.add_argument("--serving-rates", default="2,5,10,20", help="arrival rates of --workload serving")
    ap.add_argument("--serving-jobs", type=int, default=200, help="jobs per rate of --workload serving")
    ap.add_argument("--single", action="store_true",
                    help="profiling mode: run one photometric pass of view 0 per step (for ncu captures)")
    ap.add_argument("--single-step", type=int, default=STEP,
                    help="window step of the --single profiling pass (1 = the plain path's, 2 = the autotuned one)")
    ap.add_argument("--workload", default="patchmatch",
                    choices=["patchmatch", "cross-filter", "fusion", "large", "batched", "serving"],
                    help="patchmatch: the depth-map stage (default); cross-filter: CrossFilterCuda::Run + "
                         "DedupRun over the views' depth/normal maps; fusion: StereoFusion of the views' maps "
                         "into a point cloud; large: one 6000x4000 view with 20 sources through a 3-level "
                         "pyramid; batched: 64 references of uneven size on a 200-camera ring in one batch; "
                         "serving: Poisson job streams over a 400-camera aerial survey")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = {"cross-filter": 200, "fusion": 10}.get(args.workload, 3)
    return args


# ---------------------------------------------------------------------------
def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.file.name)
        loaded = [s for s in sm if smax and s > 0.3 * max(smax)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def make_options(scene, storage, geometric, step=STEP):
    from sensemap_b200.patch_match import PatchMatchOptions
    o = PatchMatchOptions(depth_min=scene.depth_min, depth_max=scene.depth_max, window_radius=RADIUS,
                          window_step=step, sigma_spatial=RADIUS, num_iterations=ITERS,
                          geom_consistency=geometric, init_depth_random=not geometric,
                          geom_consistency_regularizer=0.1,  # config/mvs.yaml value
                          image_storage=storage)
    return o


class Workload:
    def __init__(self, scene, storage, device_images, host_images):
        self.scene = scene
        self.storage = storage
        self.dev = device_images    # list of cuda float32 tensors (H x W)
        self.host = host_images     # list of pinned float32 tensors
        self.V = len(scene.views)

    def views(self, images, depth=None, normal=None):
        from sensemap_b200.patch_match import View
        out = []
        for i, v in enumerate(self.scene.views):
            out.append(View(images[i], v.K, v.R, v.T,
                            depth=None if depth is None else depth[i],
                            normal=None if normal is None else normal[i]))
        return out

    def problem(self, ref, views):
        from sensemap_b200.patch_match import Problem
        return Problem(ref, [i for i in range(self.V) if i != ref], views)

    def step_device(self, stream, keep):
        """One scene step with device-resident inputs; engines are kept alive
        (in `keep`) until the caller has synchronised."""
        from sensemap_b200.patch_match import PatchMatchACMMCuda
        sc = self.scene
        views = self.views(self.dev)
        opt_p = make_options(sc, self.storage, False)
        photo = []
        for r in range(self.V):
            opt_p.random_seed = r
            pm = PatchMatchACMMCuda(opt_p, self.problem(r, views), stream=stream)
            pm.Run()
            photo.append(pm)
        maps = [pm.DeviceDepthNormal() for pm in photo]
        gviews = self.views(self.dev, [m[0] for m in maps], [m[1] for m in maps])
        opt_g = make_options(sc, self.storage, True)
        geo = []
        for r in range(self.V):
            opt_g.random_seed = 1000 + r
            pm = PatchMatchACMMCuda(opt_g, self.problem(r, gviews), stream=stream)
            pm.Run()
            geo.append(pm)
        keep.extend(photo + geo)
        return geo

    def step_host(self):
        """The same step through host buffers (reference-facing call pattern)."""
        from sensemap_b200.patch_match import PatchMatchACMMCuda
        sc = self.scene
        views = self.views(self.host)
        opt_p = make_options(sc, self.storage, False)
        depth, normal = [], []
        h2d = d2h = launches = 0
        img_bytes = sum(int(t.numel()) * 4 for t in self.host)
        for r in range(self.V):
            opt_p.random_seed = r
            with PatchMatchACMMCuda(opt_p, self.problem(r, views)) as pm:
                pm.Run()
                depth.append(pm.GetDepthMap())
                normal.append(pm.GetNormalMap())
                launches += pm.LaunchCount()
            h2d += img_bytes
            d2h += depth[-1].nbytes + normal[-1].nbytes
        gviews = self.views(self.host, depth, normal)
        opt_g = make_options(sc, self.storage, True)
        out = []
        for r in range(self.V):
            opt_g.random_seed = 1000 + r
            with PatchMatchACMMCuda(opt_g, self.problem(r, gviews)) as pm:
                pm.Run()
                out.append(pm.GetDepthMap())
                launches += pm.LaunchCount()
            h2d += img_bytes + sum(d.nbytes for d in depth) + normal[r].nbytes
            d2h += out[-1].nbytes
        return out, h2d, d2h, launches


class PoolWorkload:
    """The same scene step through the batched pool: every view resident once,
    11 photometric jobs in one batch, then 11 geometric jobs in one batch."""

    def __init__(self, wl: Workload, block_x: int = 32, ref_tile_tma: bool = True, threads_per_pixel: int = 1,
                 step: int = STEP, persistent: bool = False):
        self.wl = wl
        self.block_x = block_x
        self.ref_tile_tma = ref_tile_tma
        self.tpp = threads_per_pixel
        self.step = step
        self.persistent = persistent

    def _run(self, pool, images, on_photo_done=None, base=0):
        """Both passes of every view; view ids base .. base + V - 1 (a fresh base
        makes the pool upload the images again)."""
        from sensemap_b200.patch_match import View
        wl, sc = self.wl, self.wl.scene
        for i, v in enumerate(sc.views):
            pool.add_view(base + i, View(images[i], v.K, v.R, v.T))
        opt_p = make_options(sc, wl.storage, False, self.step)
        photo = []
        for r in range(wl.V):
            opt_p.random_seed = r
            photo.append(pool.submit(opt_p, base + r, [base + i for i in range(wl.V) if i != r]))
        pool.run_until_done(photo)
        for j in photo:
            if on_photo_done is not None:
                on_photo_done(j)
            pool.keep_maps(j)
            pool.release(j)
        opt_g = make_options(sc, wl.storage, True, self.step)
        geo = []
        for r in range(wl.V):
            opt_g.random_seed = 1000 + r
            geo.append(pool.submit(opt_g, base + r, [base + i for i in range(wl.V) if i != r]))
        pool.run_until_done(geo)
        return geo

    def new_pool(self, stream):
        from sensemap_b200.pool import DepthMapPool
        return DepthMapPool(memory_budget_bytes=64 << 30, max_active_jobs=self.wl.V, image_storage=self.wl.storage,
                            sweep_block_x=self.block_x, stream=stream, ref_tile_tma=self.ref_tile_tma,
                            threads_per_pixel=self.tpp, persistent=self.persistent)

    def step_device(self, stream):
        """Device-resident images in. One pool serves every device step, as a
        long-running process keeps it (and as step_host does): each step adds
        the images under fresh view ids, so they are converted again, releases
        the previous step's jobs and runs both passes of every view. Returns
        the pool, this step's geometric jobs and the kernels it launched."""
        if getattr(self, "_dev_pool", None) is None:
            self._dev_pool = self.new_pool(stream)
            self._dev_steps = 0
            self._dev_prev = []
        pool = self._dev_pool
        for j in self._dev_prev:
            pool.release(j)
        before = pool.stats()["launches"]
        base = 1000 * self._dev_steps
        self._dev_steps += 1
        geo = self._run(pool, self.wl.dev, base=base)
        self._dev_prev = geo
        return pool, geo, pool.stats()["launches"] - before

    def close_device_pool(self):
        if getattr(self, "_dev_pool", None) is not None:
            self._dev_pool.close()
            self._dev_pool = None

    def step_host(self, stream):
        """Host images in; every job's depth, normal and confidence maps back to
        host, for the photometric and the geometric pass (what ProcessProblem
        reads back and writes, patch_match_controller.cc:4679-4720). One pool
        serves every host step, as a long-running process keeps it: each step
        adds the pinned host images under fresh view ids (so they are uploaded
        again) and reads the maps back into pinned host buffers allocated on the
        first call and reused."""
        import torch
        import sensemap_b200._native as NN
        kinds = (NN.MAP_DEPTH, NN.MAP_NORMAL, NN.MAP_CONF)
        wl = self.wl
        if getattr(self, "_host_pool", None) is None:
            self._host_pool = self.new_pool(stream)
            self._host_steps = 0
            H, W = wl.scene.views[0].image.shape
            shapes = {NN.MAP_DEPTH: (H, W), NN.MAP_NORMAL: (3, H, W), NN.MAP_CONF: (H, W)}
            self._host_out = [torch.empty(shapes[k], dtype=torch.float32).pin_memory()
                              for _ in range(2 * wl.V) for k in kinds]
        pool, out = self._host_pool, self._host_out
        slot = iter(range(len(out)))
        reads = []

        def read(j):
            for k in kinds:
                reads.append(pool.get_map(j, k, out=out[next(slot)]))
        base = 1000 * self._host_steps
        self._host_steps += 1
        geo = self._run(pool, wl.host, on_photo_done=read, base=base)
        for j in geo:
            read(j)
            pool.release(j)
        st = pool.stats()
        h2d = sum(int(t.numel()) * 4 for t in wl.host)
        d2h = sum(int(o.numel()) * 4 for o in reads)
        return reads, h2d, d2h, st["launches"]

    def close_host_pool(self):
        if getattr(self, "_host_pool", None) is not None:
            self._host_pool.close()
            self._host_pool = None


def storage_code(name):
    from sensemap_b200 import STORE_F16, STORE_F32, STORE_U8
    return {"u8": STORE_U8, "f16": STORE_F16, "f32": STORE_F32}[name]


# ---------------------------------------------------------------------------
def cpu_band(scene, maps, rows: int) -> dict:
    """The oracle (OpenMP transcription of the reference kernel logic, every
    host thread) on a band of `rows` rows at the middle of view 0, both passes
    of a depth map: the photometric pass (random initialisation, 6
    iterations), then the geometric pass (6 iterations) initialised from the
    band's photometric maps, with the other views' noisy ground-truth maps as
    the source depth maps. Each pass scores the initial hypotheses of its band
    and of the rows its sweeps read, and sweeps the band; the pixels of a
    colour are spread over the threads. Returns both pass times and the depth
    maps/s a full view would take at this rate (extrapolated by H / rows)."""
    import oracle.oracle as orc
    from sensemap_b200 import STORE_U8
    from sensemap_b200.patch_match import Problem, View
    V = len(scene.views)
    H = scene.views[0].image.shape[0]
    r0 = H // 2 - rows // 2
    srcs = list(range(1, V))
    # The reference samples 8-bit textures (patch_match_cuda.cu:229-278): the CPU
    # transcription runs with that storage whatever the GPU form uses.
    photo = Problem(0, srcs, [View(v.image, v.K, v.R, v.T) for v in scene.views])
    t = time.perf_counter()
    ph = orc.run(make_options(scene, STORE_U8, False), photo, rows=(r0, r0 + rows))
    tp = time.perf_counter() - t
    d0, n0 = maps[0][0].copy(), maps[0][1].copy()
    d0[r0:r0 + rows] = ph["depth"][r0:r0 + rows]
    n0[:, r0:r0 + rows] = ph["normal"][:, r0:r0 + rows]
    gviews = [View(v.image, v.K, v.R, v.T, depth=d, normal=n) for v, (d, n) in zip(scene.views, maps)]
    gviews[0] = View(scene.views[0].image, scene.views[0].K, scene.views[0].R, scene.views[0].T, depth=d0, normal=n0)
    t = time.perf_counter()
    orc.run(make_options(scene, STORE_U8, True), Problem(0, srcs, gviews), rows=(r0, r0 + rows))
    tg = time.perf_counter() - t
    per_map = (tp + tg) * H / rows
    return {"value": 1.0 / per_map, "unit": "depth maps/s", "cores": orc.num_threads(), "kind": "port",
            "band_rows": rows, "photometric_band_s": tp, "geometric_band_s": tg,
            "sample": (f"oracle (OpenMP transcription of the reference kernel logic, 8-bit sources), rows "
                       f"{r0}..{r0 + rows} of view 0 ({scene.views[0].image.shape[1]}x{H}, N={V - 1}): photometric "
                       f"pass {tp:.2f} s + geometric pass {tg:.2f} s measured; depth maps/s extrapolated by "
                       f"{H}/{rows} rows")}


def cpu_baseline(scene, maps, rows: int) -> dict:
    out = cpu_band(scene, maps, rows)
    out["config1_full"] = config1_full_leg()
    return out


def config1_full_leg(seed: int = 0) -> dict:
    """A full depth map, measured and not extrapolated: the small planes
    configuration (640x480, 1 reference + 4 source views, f = 500, window
    radius 5 step 1, 6 iterations, photometric only, FP32 sources) through the
    oracle on every host thread and through the engine (device-resident
    images, smvs_create + Run timed with CUDA events, best of 3 after a
    warm-up), with both maps' ground-truth accuracy and their agreement."""
    import torch
    import oracle.oracle as orc
    from sensemap_b200 import STORE_F32
    from sensemap_b200 import synthetic as syn
    from sensemap_b200.patch_match import PatchMatchACMMCuda, PatchMatchOptions, Problem, View
    sc = syn.planes_scene(seed=seed, width=640, height=480, focal=500.0, num_src=4)
    opt = PatchMatchOptions(depth_min=sc.depth_min, depth_max=sc.depth_max, window_radius=5, window_step=1,
                            sigma_spatial=5, num_iterations=6, geom_consistency=False, init_depth_random=True,
                            image_storage=STORE_F32, random_seed=seed)
    host = Problem(sc.ref_index, sc.src_indices, [View(v.image, v.K, v.R, v.T) for v in sc.views])
    t = time.perf_counter()
    cpu_maps = orc.run(opt, host)
    cpu_s = time.perf_counter() - t
    dev = Problem(sc.ref_index, sc.src_indices,
                  [View(torch.from_numpy(v.image).cuda(), v.K, v.R, v.T) for v in sc.views])
    stream = torch.cuda.Stream()  # the engine's launching stream (a non-default one, as in the other legs)
    gpu_ms = []
    for rep in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        pm = PatchMatchACMMCuda(opt, dev, stream=stream.cuda_stream)
        pm.Run()
        e1.record(stream)
        pm.Synchronize()
        e1.synchronize()
        depth = pm.GetDepthMap()
        pm.close()
        if rep:
            gpu_ms.append(e0.elapsed_time(e1))
    gt = sc.views[sc.ref_index].depth_gt
    m = gt > 0
    agree = float(np.mean(np.abs(depth[m] - cpu_maps["depth"][m]) <= 0.01 * np.abs(cpu_maps["depth"][m])))
    gpu_s = min(gpu_ms) / 1000.0
    return {"what": "planes scene 640x480, 1 + 4 views, R=5, S=1, 6 iterations, photometric, FP32 sources; one "
                    "full depth map, no extrapolation",
            "cpu_s": cpu_s, "cpu_depth_maps_per_s": 1.0 / cpu_s, "cpu_cores": orc.num_threads(),
            "gpu_s": gpu_s, "gpu_depth_maps_per_s": 1.0 / gpu_s, "gpu_over_cpu": cpu_s / gpu_s,
            "gpu_within_1pct_gt": syn.depth_accuracy(depth, gt),
            "cpu_within_1pct_gt": syn.depth_accuracy(cpu_maps["depth"], gt),
            "gpu_cpu_depth_agreement": agree}


def run_reference(args):
    """The reference arm: the oracle's band of both passes (cpu_band), one band
    per step, on all host threads. The band is sized from the first warm-up
    step so that the whole run takes about two minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    from sensemap_b200 import synthetic as syn
    from oracle import build as oracle_build
    oracle_build.build()
    scene = syn.heightfield_scene(seed=0, width=args.width, height=args.height, num_src=args.views - 1,
                                  device="cuda" if torch.cuda.is_available() else "cpu")
    maps = syn.noisy_maps(scene, seed=100)
    total = args.warmup + args.steps
    rows = CPU_BAND_ROWS
    samples, band_ms, cb = [], [], None
    for i in range(total):
        cb = cpu_band(scene, maps, rows)
        if i == 0:  # size the band: ~120 s for the whole run, 4..64 rows
            per_row = (cb["photometric_band_s"] + cb["geometric_band_s"]) / rows
            rows = int(min(64, max(4, 120.0 / max(1, total) / max(per_row, 1e-6))))
        if i >= args.warmup:
            samples.append(cb["value"])
            band_ms.append(1000.0 * (cb["photometric_band_s"] + cb["geometric_band_s"]))
    value = statistics.median(samples)
    line = {"metric": METRIC, "value": value, "unit": "depth maps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.median(band_ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"heightfield scene, {args.views} views {args.width}x{args.height}, each view "
                                   f"photometric + geometric PatchMatch (R={RADIUS}, S={STEP}, {ITERS} iterations); "
                                   f"each step is a {rows}-row band of view 0 through both passes, value extrapolated "
                                   f"to full views (ms_per_step is the measured band)",
                       "global_batch": args.views, "parallelism": "cpu-openmp"},
            "cpu_baseline": {**cb, "value": value},
            "e2e": {"value": value, "unit": "depth maps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def timed_steps(step_fn, steps, warmup, stream, world, clocks=None):
    """W untimed steps, then K steps bracketed by barrier + synchronize and CUDA
    events on the launching stream. step_fn() -> (objects to close, launches,
    getter of (depth, normal) per view). Returns (max-over-ranks ms, launches,
    getter of the last step, objects of the last step)."""
    import torch
    for _ in range(warmup):
        objs, _, _ = step_fn()
        torch.cuda.synchronize()
        for o in objs:
            o.close()
    barrier(world)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    keep, launches, getter = [], 0, None
    ev0.record(stream)
    for _ in range(steps):
        objs, n, getter = step_fn()
        launches += n
        keep.append(objs)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clock_info = clocks.stop() if clocks is not None else None
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    for objs in keep[:-1]:
        for o in objs:
            o.close()
    return ms, launches, getter, keep[-1], clock_info


def accuracy_of(getter, scene):
    """Fraction of ground-truth pixels within 1 % depth and within 10 degrees
    normal, per view and mean."""
    from sensemap_b200 import synthetic as syn
    d_acc, n_acc = [], []
    for i, v in enumerate(scene.views):
        d, n = getter(i)
        d_acc.append(syn.depth_accuracy(d, v.depth_gt))
        n_acc.append(syn.normal_accuracy(n, v.normal_gt, mask=v.depth_gt > 0))
    return {"within_1pct_gt": float(np.mean(d_acc)), "within_10deg_normal": float(np.mean(n_acc)),
            "per_view_1pct": [round(a, 4) for a in d_acc]}


def pool_step_fn(pw, stream):
    import sensemap_b200._native as NN

    def step():  # the pool outlives the step (PoolWorkload.close_device_pool)
        pool, geo, launches = pw.step_device(stream)
        return [], launches, \
            (lambda i: (pool.get_map(geo[i], NN.MAP_DEPTH), pool.get_map(geo[i], NN.MAP_NORMAL)))
    return step


def engine_step_fn(wl, stream):
    def step():
        keep = []
        geo = wl.step_device(stream, keep)
        return keep, sum(pm.LaunchCount() for pm in keep), (lambda i: (geo[i].GetDepthMap(), geo[i].GetNormalMap()))
    return step


def reference_kernels_leg(scene, ours_view0, repeats=3) -> dict:
    """Baseline leg: the reference's own PatchMatch kernels (compiled from its
    sources into the checker library) on this GPU for view 0 of the bench scene:
    their launch order, launch shapes, 8-bit layered source texture and a device
    sync after every launch. The geometric pass of view 0 uses the reference
    kernels' own photometric maps of every view. Reports seconds per depth map
    (photometric + geometric pass of view 0, best of `repeats`), its accuracy
    against ground truth and the agreement of our map of view 0 with it."""
    import torch
    from oracle import oracle as O
    from oracle import ref_oracle as R
    from sensemap_b200 import STORE_U8
    from sensemap_b200 import synthetic as syn
    from sensemap_b200.patch_match import Problem, View
    if not R.available():
        return {"unavailable": "reference kernels not built (oracle/_ref)"}
    V = len(scene.views)
    fviews = [O.FilterView(v.K, v.R, v.T, v.depth_gt, v.normal_gt) for v in scene.views]
    plain = [View(v.image, v.K, v.R, v.T) for v in scene.views]
    photo_maps, poses_of = [], {}
    for r in range(V):
        srcs = [i for i in range(V) if i != r]
        poses_of[r] = O.cross_filter_poses(fviews, (r, srcs))[2]
        o = make_options(scene, STORE_U8, False)
        o.random_seed = r
        res = R.run(o, Problem(r, srcs, plain), poses_of[r])
        photo_maps.append((res["depth"], res["normal"]))
    gviews = [View(v.image, v.K, v.R, v.T, depth=d, normal=n) for v, (d, n) in zip(scene.views, photo_maps)]
    srcs0 = list(range(1, V))
    t_photo, t_geo, geo = [], [], None
    for _ in range(repeats):
        torch.cuda.synchronize()
        t = time.perf_counter()
        R.run(make_options(scene, STORE_U8, False), Problem(0, srcs0, plain), poses_of[0])
        torch.cuda.synchronize()
        t_photo.append(time.perf_counter() - t)
        t = time.perf_counter()
        o = make_options(scene, STORE_U8, True)
        o.random_seed = 1000
        geo = R.run(o, Problem(0, srcs0, gviews), poses_of[0])
        torch.cuda.synchronize()
        t_geo.append(time.perf_counter() - t)
    v0 = scene.views[0]
    m = v0.depth_gt > 0
    d_ours, n_ours = ours_view0
    agree_d = float(np.mean(np.abs(d_ours[m] - geo["depth"][m]) <= 0.01 * np.abs(geo["depth"][m])))
    agree_n = syn.normal_accuracy(n_ours, geo["normal"] / np.maximum(
        np.linalg.norm(geo["normal"], axis=0, keepdims=True), 1e-12), mask=m)
    per_map = min(t_photo) + min(t_geo)
    return {"what": "the reference's kernel_functions.cu (built with its own flags, --use_fast_math) on this GPU, "
                    "PatchMatchACMMCuda::Run's launch order and syncs, 8-bit layered source texture; host wall time "
                    "of one photometric + one geometric pass of view 0 (best of %d)" % repeats,
            "seconds_per_depth_map": per_map, "depth_maps_per_s": 1.0 / per_map,
            "photometric_s": min(t_photo), "geometric_s": min(t_geo),
            "within_1pct_gt": syn.depth_accuracy(geo["depth"], v0.depth_gt),
            "within_10deg_normal": syn.normal_accuracy(geo["normal"], v0.normal_gt, mask=m),
            "ours_vs_reference_view0": {"within_1pct_depth": agree_d, "within_10deg_normal": agree_n}}


def ncc_fp64_leg(scene, storage, tune, stream, samples=10000) -> dict:
    """Per-pixel NCC cost error of the GPU against the oracle's FP64 evaluator:
    one photometric pass of view 0 in the measured form, then for `samples`
    seeded pixels the GPU's per-view cost of its final hypothesis against the
    FP64 evaluation of the same hypothesis (direct homography per tap, exact
    bilinear weights, exact exp)."""
    import oracle.oracle as orc
    from sensemap_b200.patch_match import PatchMatchACMMCuda, Problem, View
    V = len(scene.views)
    opt = make_options(scene, storage, False)
    dev_prob = Problem(0, list(range(1, V)), [View(v.image, v.K, v.R, v.T) for v in scene.views])
    with PatchMatchACMMCuda(opt, dev_prob, stream=stream) as pm:
        pm.SetTuning(tune["sweep_block_x"], tune["ref_tile_tma"], tune["threads_per_pixel"], tune["persistent"])
        pm.Run()
        depth, normal, cost = pm.GetDepthMap(), pm.GetNormalMap(), pm.GetCostMap()
    rng = np.random.default_rng(11)
    Hh, Ww = depth.shape
    rows = rng.integers(0, Hh, samples)
    cols = rng.integers(0, Ww, samples)
    _, c64 = orc.eval_costs(opt, dev_prob, rows, cols, depth[rows, cols], normal[:, rows, cols].T)
    gpu = cost[:, rows, cols].T.astype(np.float64)
    err = np.abs(gpu - c64).ravel()
    return {"samples": int(samples) * (V - 1), "median": float(np.median(err)), "p99": float(np.percentile(err, 99)),
            "frac_below_1e-2": float(np.mean(err < 1e-2)),
            "what": "GPU per-view NCC cost of the final hypothesis (photometric pass of view 0, %s storage) vs the "
                    "FP64 evaluation of the same hypothesis" % {0: "u8", 1: "f16", 2: "f32"}.get(storage, "?")}


def main():
    args = parse()
    if args.workload == "cross-filter":
        if args.impl == "reference":
            run_cross_filter_reference(args)
        else:
            run_cross_filter(args)
        return
    if args.workload == "fusion":
        if args.impl == "reference":
            run_fusion_reference(args)
        else:
            run_fusion(args)
        return
    if args.workload in ("large", "batched", "serving"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the default workload "
                              "(the CPU transcription); this workload has no CPU sample"}), flush=True)
            return
        {"large": run_large, "batched": run_batched, "serving": run_serving_aerial}[args.workload](args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    world, rank, local = dist_setup()
    from sensemap_b200 import build as engine_build
    from sensemap_b200 import _native as N
    from sensemap_b200 import synthetic as syn
    from sensemap_b200 import STORE_F32
    engine_build.build()
    N.lib()
    storage = storage_code(args.storage)
    t0 = time.perf_counter()
    scene = syn.heightfield_scene(seed=rank, width=args.width, height=args.height, num_src=args.views - 1,
                                  device="cuda")
    log(f"[rank {rank}] scene rendered in {time.perf_counter() - t0:.1f} s; depth range "
        f"{scene.depth_min:.2f}..{scene.depth_max:.2f}")
    dev_imgs = [torch.from_numpy(v.image).cuda() for v in scene.views]
    host_imgs = [torch.from_numpy(v.image).pin_memory() for v in scene.views]
    wl = Workload(scene, storage, dev_imgs, host_imgs)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    if args.single:
        run_single(args, wl, sptr)
        return

    # Launch shape from the autotuner (one iteration of view 0's photometric
    # pass per candidate, before the timed region; maps do not depend on it).
    from sensemap_b200.patch_match import PatchMatchACMMCuda, autotune
    tune = autotune(make_options(scene, storage, False), wl.problem(0, wl.views(dev_imgs)), stream=sptr, repeats=2)
    log(f"autotune: block_x={tune['sweep_block_x']} tpp={tune['threads_per_pixel']} tma={tune['ref_tile_tma']} "
        f"persistent={tune['persistent']} ({', '.join(f'{c['sweep_block_x']}/{c['threads_per_pixel']}'
                                                      f'{'p' if c['persistent'] else ''}: {c['ms_per_sweep']:.2f} ms'
                                                      for c in tune['candidates'])})")
    pw = PoolWorkload(wl, block_x=tune["sweep_block_x"], ref_tile_tma=tune["ref_tile_tma"],
                      threads_per_pixel=tune["threads_per_pixel"], persistent=tune["persistent"])

    # Timed region: the batched form, device-resident inputs.
    clocks = ClockSampler(local)
    ms, launches, getter, last, clock_info = timed_steps(
        pool_step_fn(pw, sptr) if args.mode == "batched" else engine_step_fn(wl, sptr),
        args.steps, args.warmup, stream, world, clocks)
    depth_maps = args.steps * wl.V * world
    value = depth_maps / (ms / 1000.0)
    acc = accuracy_of(getter, scene)
    ours_view0 = getter(0)
    for o in last:
        o.close()
    pw.close_device_pool()
    log(f"value {value:.3f} depth maps/s, accuracy {acc['within_1pct_gt']:.4f}")

    # Per-kernel device time (one profiled photometric pass of view 0).
    views = wl.views(dev_imgs)
    pm = PatchMatchACMMCuda(make_options(scene, storage, False), wl.problem(0, views), stream=sptr)
    pm.SetTuning(tune["sweep_block_x"], tune["ref_tile_tma"], tune["threads_per_pixel"], tune["persistent"])
    pm.SetProfiling(True)
    pm.Run()
    prof = pm.Profile()
    pm.close()
    sweep_n, sweep_ms = prof.get("sweep", (0, 0.0))
    T = (2 * RADIUS // STEP + 1) ** 2
    taps_per_launch = (args.width * args.height / 2) * (args.views - 1) * HYP_PER_PIXEL * T
    sweep_avg_s = sweep_ms / max(sweep_n, 1) / 1000.0
    achieved_tflops = taps_per_launch * FLOP_PER_TAP / sweep_avg_s / 1e12
    fp32 = ctypes_rate(N, 0)
    tex = ctypes_rate(N, 1)
    peak_taps = min(fp32 / FLOP_PER_TAP, tex)
    full = (args.width, args.height, args.views) == (W, H, NSRC + 1)
    roof = {"bound": "texture-sampling", "achieved": achieved_tflops, "peak": peak_taps * FLOP_PER_TAP / 1e12,
            "unit": "TFLOP/s", "frac": (taps_per_launch / sweep_avg_s) / peak_taps,
            "traffic": SWEEP_DRAM_BYTES.get(args.storage) if full else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one sweep launch of this workload"
                              " (profiles/)",
            "kernel": (f"SweepKernelL<{RADIUS},{STEP},{12 if NSRC <= 12 else 16}>" if tune["threads_per_pixel"] == 1
                       else f"SweepKernel<{RADIUS},{STEP},{tune['threads_per_pixel']}>"),
            "taps_per_launch": taps_per_launch, "flop_per_tap": FLOP_PER_TAP, "avg_launch_ms": sweep_avg_s * 1000.0,
            "peak_source": (f"measured in this process: FP32 FMA {fp32 / 1e12:.1f} TFLOP/s, bilinear texture "
                            f"{tex / 1e9:.0f} Gsample/s; peak = min(FP32/25, texture) taps/s x 25 flop"),
            "kernel_share": {k: round(v[1] / sum(x[1] for x in prof.values()), 4) for k, v in prof.items()}}

    e2e = None
    if not args.no_e2e:
        # End to end through host buffers (pinned inputs; depth, normal and
        # confidence maps of both passes back to pinned host buffers).
        host_step = wl.step_host if args.mode == "engine" else (lambda: pw.step_host(sptr))
        host_step()
        torch.cuda.synchronize()
        barrier(world)
        e2e_steps = min(args.steps, 3)
        t = time.perf_counter()
        h2d = d2h = 0
        step_s = []
        for _ in range(e2e_steps):
            t_step = time.perf_counter()
            _, h2d, d2h, _ = host_step()
            step_s.append(time.perf_counter() - t_step)
        torch.cuda.synchronize()
        el = max_over_ranks(time.perf_counter() - t, world)
        e2e = {"value": e2e_steps * wl.V * world / el, "unit": "depth maps/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": e2e_steps, "step_s": [round(x, 3) for x in step_s]}
        log(f"e2e {e2e['value']:.3f} depth maps/s, host steps {', '.join(f'{x:.2f}' for x in step_s)} s")
        pw.close_host_pool()

    # The plain path: FP32 storage, one engine per reference view and pass.
    plain_wl = Workload(scene, STORE_F32, dev_imgs, host_imgs)
    p_steps = min(args.steps, 2)
    p_ms, p_launches, p_get, p_last, _ = timed_steps(engine_step_fn(plain_wl, sptr), p_steps, 1, stream, world)
    plain = {"value": p_steps * wl.V * world / (p_ms / 1000.0), "steps": p_steps, "launches": p_launches,
             "form": "engine (one smvs_create/smvs_run per reference view and pass), FP32 storage, R=5, S=1, default "
                     "launch shape", **accuracy_of(p_get, scene)}
    for o in p_last:
        o.close()
    log(f"plain {plain['value']:.3f} depth maps/s, accuracy {plain['within_1pct_gt']:.4f}")

    # The autotuner's window-step candidate: the batched form at S=2, accepted
    # when its ground-truth accuracy is within 0.5 points of the plain path's.
    pw2 = PoolWorkload(wl, block_x=tune["sweep_block_x"], ref_tile_tma=tune["ref_tile_tma"],
                       threads_per_pixel=tune["threads_per_pixel"], step=2, persistent=tune["persistent"])
    s_steps = min(args.steps, 4)
    s_ms, s_launches, s_get, s_last, _ = timed_steps(pool_step_fn(pw2, sptr), s_steps, 1, stream, world)
    s_acc = accuracy_of(s_get, scene)
    for o in s_last:
        o.close()
    pw2.close_device_pool()
    s_value = s_steps * wl.V * world / (s_ms / 1000.0)
    gap = 100.0 * (plain["within_1pct_gt"] - s_acc["within_1pct_gt"])
    autotuned = {"window_step": 2 if gap <= 0.5 else STEP, "candidate": {"window_step": 2, "value": s_value,
                                                                          "steps": s_steps, **s_acc},
                 "accuracy_gap_pt_vs_plain": gap, "accepted": gap <= 0.5,
                 "value": s_value if gap <= 0.5 else value,
                 "ratio_vs_plain": (s_value if gap <= 0.5 else value) / plain["value"],
                 "gate": "GT depth accuracy (within 1 %) within 0.5 points of the plain path's on this scene"}
    log(f"window step 2: {s_value:.3f} depth maps/s, accuracy {s_acc['within_1pct_gt']:.4f} (gap {gap:.2f} pt)")

    serving = None
    if args.serving_seconds > 0:
        serving = run_serving(args, wl, sptr, tune)

    ref_k = ncc = cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # Baseline legs (after every timed region): the reference's kernels on
        # this GPU, the FP64 cost check and the CPU transcription.
        try:
            ref_k = reference_kernels_leg(scene, ours_view0)
        except Exception as exc:  # reported, not fatal
            ref_k = {"unavailable": f"{type(exc).__name__}: {exc}"}
        ncc = ncc_fp64_leg(scene, storage, tune, sptr)
        maps = syn.noisy_maps(scene, seed=100)
        cpu = cpu_baseline(scene, maps, CPU_BAND_ROWS)
    if rank == 0:
        accuracy = dict(acc)
        accuracy["ncc_cost_err_fp64"] = ncc
        if ref_k and "ours_vs_reference_view0" in ref_k:
            accuracy["vs_reference_kernels"] = ref_k["ours_vs_reference_view0"]
        line = {"metric": METRIC, "value": value, "unit": "depth maps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"heightfield scene, {wl.V} views {args.width}x{args.height}, each view "
                                       f"photometric + geometric PatchMatch (R={RADIUS}, S={STEP}, {ITERS} "
                                       f"iterations), {args.storage} image storage, {args.mode} form",
                           "global_batch": wl.V * world, "parallelism": f"views sharded, {world} replica(s)",
                           "l2": "inputs larger than L2 (11 x 1600x1200 images + maps per step)"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "serving": serving,
                "clocks": clock_info, "autotune": tune, "accuracy": accuracy, "plain": plain,
                "autotuned_window": autotuned, "reference_kernels": ref_k}
        # The metric's second throughput unit: image megapixels x source
        # views x iterations x passes per second (one depth map = 2 passes).
        mpvi = args.width * args.height / 1e6 * (wl.V - 1) * ITERS * 2
        line["mpix_views_iters_per_s"] = {"value": value * mpvi, "plain": plain["value"] * mpvi,
                                          "autotuned_window": autotuned["value"] * mpvi,
                                          "per_depth_map": mpvi}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_serving(args, wl, sptr, tune) -> dict:
    """Poisson arrivals of photometric depth-map jobs (random reference view of
    the scene, the other views as sources), served (a) by the continuous-
    batching pool with every view resident and (b) by the plain path, one
    engine per job in arrival order (FP32 storage, default launch shape).
    p50/p99 completion latency (completion minus arrival) and throughput of
    each, on the same arrival times."""
    import torch
    from sensemap_b200 import STORE_F32
    from sensemap_b200 import serving as srv
    from sensemap_b200.patch_match import PatchMatchACMMCuda, Problem, View
    from sensemap_b200.pool import DepthMapPool
    sc = wl.scene
    n_jobs = max(4, int(args.serving_rate * args.serving_seconds))
    arrivals = srv.poisson_arrivals(args.serving_rate, n_jobs, seed=1)
    rng = np.random.default_rng(2)
    refs = [int(rng.integers(0, wl.V)) for _ in range(n_jobs)]
    specs = []
    for k, r in enumerate(refs):
        o = make_options(sc, wl.storage, False)
        o.random_seed = 5000 + k
        specs.append(srv.JobSpec(o, r, [i for i in range(wl.V) if i != r]))
    slots = 8
    pool = DepthMapPool(memory_budget_bytes=32 << 30, max_active_jobs=slots, image_storage=wl.storage, stream=sptr,
                        sweep_block_x=tune["sweep_block_x"], threads_per_pixel=tune["threads_per_pixel"],
                        persistent=tune["persistent"])
    for i, v in enumerate(sc.views):
        pool.add_view(i, View(wl.dev[i], v.K, v.R, v.T))
    acc = []

    def done(k, jid):
        if len(acc) < 8:
            acc.append(syn_depth_accuracy(pool.get_map(jid, 0), sc.views[specs[k].ref_view].depth_gt))
        pool.release(jid)

    res = srv.serve(pool, specs, arrivals, on_done=done)
    st = pool.stats()
    pool.close()
    res.pop("latencies")
    res.update({"arrival_rate_jobs_s": args.serving_rate, "slots": slots,
                "job": f"photometric pass, 1 ref + {wl.V - 1} src, {sc.views[0].image.shape[1]}x"
                       f"{sc.views[0].image.shape[0]}, {ITERS} iterations",
                "within_1pct_gt_first_jobs": float(np.mean(acc)) if acc else None,
                "graphs_built": st["graphs_built"], "pool_steps": st["steps"]})

    # The plain path under the same arrivals: one job at a time.
    views = [View(wl.dev[i], v.K, v.R, v.T) for i, v in enumerate(sc.views)]
    lat = np.zeros(n_jobs)
    t0 = time.perf_counter()
    for k, r in enumerate(refs):
        now = time.perf_counter() - t0
        if arrivals[k] > now:
            time.sleep(arrivals[k] - now)
        o = make_options(sc, STORE_F32, False)
        o.random_seed = 5000 + k
        with PatchMatchACMMCuda(o, Problem(r, [i for i in range(wl.V) if i != r], views), stream=sptr) as pm:
            pm.Run()
            pm.Synchronize()
        lat[k] = time.perf_counter() - t0 - arrivals[k]
    wall = time.perf_counter() - t0
    torch.cuda.synchronize()
    res["plain"] = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                    "mean_s": float(lat.mean()), "throughput_jobs_s": n_jobs / wall,
                    "form": "one engine per job in arrival order, FP32 storage"}
    return res


def syn_depth_accuracy(depth, gt):
    from sensemap_b200 import synthetic as syn
    return syn.depth_accuracy(depth, gt)


def run_single(args, wl, sptr):
    """One photometric pass of view 0 per step, nothing else (profiling)."""
    import torch
    from sensemap_b200.patch_match import PatchMatchACMMCuda
    views = wl.views(wl.dev)
    opt = make_options(wl.scene, wl.storage, False, step=args.single_step)
    per_kernel = {}
    for i in range(args.warmup + args.steps):
        with PatchMatchACMMCuda(opt, wl.problem(0, views), stream=sptr) as pm:
            pm.SetProfiling(i >= args.warmup)
            pm.Run()
            pm.Synchronize()
            if i >= args.warmup:
                for k, (n, ms) in pm.Profile().items():
                    per_kernel.setdefault(k, []).append(ms / max(n, 1))
                depth = pm.GetDepthMap()
    torch.cuda.synchronize()
    log("single-pass profiling run done")
    if per_kernel:
        # Per-kernel device time of the pass (CUDA events around each launch),
        # the best step's average launch, and the map's ground-truth accuracy.
        from sensemap_b200 import synthetic as syn
        print(json.dumps({"single_pass": {
            "workload": f"photometric pass of view 0, {args.width}x{args.height}, N={args.views - 1}, R={RADIUS}, "
                        f"S={args.single_step}, {ITERS} iterations, {args.storage} storage, default launch shape",
            "ms_per_launch": {k: round(min(v), 3) for k, v in per_kernel.items()},
            "within_1pct_gt": syn.depth_accuracy(depth, wl.scene.views[0].depth_gt)}}), flush=True)


# ---------------------------------------------------------------------------
# Cross-view filter workload
# ---------------------------------------------------------------------------
CF_METRIC = "cross-filtered depth maps/s (1.6MP,10 src)"


def cross_filter_set(args, rank, device):
    """The bench scene's views with noisy ground-truth depth/normal maps (what
    the PatchMatch passes hand over) and one problem per view against the
    other views."""
    from sensemap_b200 import synthetic as syn
    scene = syn.heightfield_scene(seed=rank, width=args.width, height=args.height, num_src=args.views - 1,
                                  device=device)
    maps = syn.noisy_maps(scene, seed=100 + rank)
    problems = [(r, [s for s in range(len(scene.views)) if s != r]) for r in range(len(scene.views))]
    return scene, maps, problems


def cross_filter_bytes(shapes, problems, per_ref, per_src):
    """Algorithmic bytes of one launch: every problem reads its reference maps
    and writes its output once (per_ref B/px) and reads each source's maps once
    (per_src B/px)."""
    total = 0
    for r, srcs in problems:
        total += per_ref * shapes[r][0] * shapes[r][1]
        total += sum(per_src * shapes[q][0] * shapes[q][1] for q in srcs)
    return total


def cpu_cross_filter(scene, maps, problems, steps=1) -> dict:
    """The oracle (OpenMP restatement of CrossFilterKernel/DeduplicFilterKernel)
    over the whole set: Run + DedupRun, filtered depth maps/s."""
    import oracle.oracle as orc
    from sensemap_b200.patch_match import PatchMatchOptions
    views = [orc.FilterView(v.K, v.R, v.T, d, n, ref_flag=True) for v, (d, n) in zip(scene.views, maps)]
    opt = PatchMatchOptions()
    t = time.perf_counter()
    for _ in range(steps):
        refined = orc.cross_filter_run(opt, views, problems)
        orc.cross_filter_dedup(opt, views, problems, refined)
    dt = (time.perf_counter() - t) / steps
    return {"value": len(problems) / dt, "unit": "depth maps/s", "cores": orc.num_threads(), "kind": "port",
            "sample": f"oracle Run + DedupRun over the whole {len(views)}-view set, {steps} pass(es), {dt:.2f} s each"}


def run_cross_filter_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import torch
    from oracle import build as oracle_build
    oracle_build.build()
    scene, maps, problems = cross_filter_set(args, 0, "cuda" if torch.cuda.is_available() else "cpu")
    samples, cb = [], None
    steps = min(args.steps, 5)  # each step is a full CPU pass (about a second)
    for i in range(min(args.warmup, 3) + steps):
        cb = cpu_cross_filter(scene, maps, problems)
        if i >= min(args.warmup, 3):
            samples.append(cb["value"])
    cb["sample"] += f"; median of {steps} timed passes"
    value = statistics.median(samples)
    line = {"metric": CF_METRIC, "value": value, "unit": "depth maps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * len(problems) / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"cross filter + dedup, {args.views} views {args.width}x{args.height}, each view "
                                   f"against the other {args.views - 1}", "global_batch": len(problems),
                       "parallelism": "cpu-openmp"},
            "cpu_baseline": {**cb, "value": value},
            "e2e": {"value": value, "unit": "depth maps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_cross_filter(args):
    import torch
    world, rank, local = dist_setup()
    from sensemap_b200 import build as engine_build
    from sensemap_b200.cross_filter import CrossFilterCuda
    from sensemap_b200.patch_match import PatchMatchOptions, Problem, View
    engine_build.build()
    scene, maps, problems = cross_filter_set(args, rank, "cuda")
    V = len(scene.views)
    shapes = [d.shape for d, _ in maps]
    dev = [(torch.from_numpy(d).cuda(), torch.from_numpy(n).cuda()) for d, n in maps]
    host = [(torch.from_numpy(d).pin_memory(), torch.from_numpy(n).pin_memory()) for d, n in maps]

    def api_args(pairs):
        ims = [View(None, v.K, v.R, v.T, depth=d, normal=n) for v, (d, n) in zip(scene.views, pairs)]
        probs = [Problem(r, [], ims, src_image_extend_idxs=s) for r, s in problems]
        return probs, list(range(V)), [True] * V

    opt = PatchMatchOptions()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    dev_args, host_args = api_args(dev), api_args(host)

    def step(args_, fetch, profile=False):
        cf = CrossFilterCuda(opt, *args_, stream=sptr)
        if profile:
            cf.SetProfiling(True)
        cf.Run()
        out = [cf.GetRefineDepthMap(r) for r, _ in problems] if fetch else None
        cf.DedupRun()
        if fetch:
            out += [cf.GetDeduplicDepthMap(k) for k in range(V)]
        return cf, out

    for _ in range(args.warmup):
        cf, _ = step(dev_args, False)
        cf.close()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        cf, _ = step(dev_args, False)
        launches += cf.LaunchCount()
        cf.close()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clock_info = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    value = args.steps * V * world / (ms / 1000.0)

    # Kernel times (CUDA events on the filter's stream) for the roofline.
    cf, _ = step(dev_args, False, profile=True)
    prof = cf.Profile()
    refined = {r: cf.GetRefineDepthMap(r) for r, _ in problems}
    cf.close()
    run_n, run_ms = prof.get("cross_filter", (1, float("nan")))
    ded_n, ded_ms = prof.get("dedup", (1, float("nan")))
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    run_bytes = cross_filter_bytes(shapes, problems, 12, 8)
    ded_bytes = cross_filter_bytes(shapes, problems, 16, 8)
    run_gbs = run_bytes / (run_ms / run_n / 1000.0) / 1e9
    roof = {"bound": "hbm", "achieved": run_gbs, "peak": hbm, "unit": "GB/s", "frac": run_gbs / hbm,
            "traffic": None, "kernel": "CrossFilterRunKernel", "bytes_per_launch": run_bytes,
            "avg_launch_ms": run_ms / run_n,
            "bytes_model": "per problem: reference depth + normal code read, refined map written (12 B/px); "
                           "each source's depth + normal code read once (8 B/px)",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s",
            "dedup": {"launches": ded_n, "avg_launch_ms": ded_ms / ded_n,
                      "achieved_gbs": ded_bytes / (ded_ms / 1000.0) / 1e9, "bytes_per_step": ded_bytes},
            "kernel_ms": {k: round(v[1], 3) for k, v in prof.items()}}

    e2e = None
    if not args.no_e2e:
        cf, _ = step(host_args, True)
        cf.close()
        torch.cuda.synchronize()
        barrier(world)
        e2e_steps = min(args.steps, 10)
        t = time.perf_counter()
        for _ in range(e2e_steps):
            cf, out = step(host_args, True)
            cf.close()
        torch.cuda.synchronize()
        el = max_over_ranks(time.perf_counter() - t, world)
        h2d = sum(d.numel() * 4 + n.numel() * 4 for d, n in host)
        d2h = sum(o.nbytes for o in out)
        e2e = {"value": e2e_steps * V * world / el, "unit": "depth maps/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": e2e_steps}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_cross_filter(scene, maps, problems)
    kept = float(np.mean([(refined[r] > 0).mean() for r in refined]))
    def kept_accuracy(d, gt):
        m = (d > 0) & (gt > 0)
        return float(np.mean(np.abs(d[m] - gt[m]) <= 0.01 * gt[m])) if m.any() else 0.0

    acc = float(np.mean([kept_accuracy(refined[r], scene.views[r].depth_gt) for r in refined]))
    if rank == 0:
        line = {"metric": CF_METRIC, "value": value, "unit": "depth maps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"cross filter + dedup (CrossFilterCuda::Run + DedupRun), {V} views "
                                       f"{args.width}x{args.height}, each view against the other {V - 1}; noisy "
                                       f"ground-truth depth/normal maps of the heightfield scene",
                           "global_batch": V * world, "parallelism": f"view sets sharded, {world} replica(s)",
                           "l2": f"inputs larger than L2 ({V} x {args.width}x{args.height} depth + normal maps)"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clock_info,
                "filter": {"refined_kept_fraction": kept, "kept_within_1pct_gt": acc}}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


FU_METRIC = "fused depth maps/s (1.6MP, 11 views)"


def fusion_set(args, rank, device):
    """The bench scene's views with noisy ground-truth depth/normal maps (what
    the PatchMatch passes hand over), an RGB bitmap per view and, as each
    view's overlapping images, every other view nearest first."""
    from sensemap_b200 import synthetic as syn
    scene = syn.heightfield_scene(seed=rank, width=args.width, height=args.height, num_src=args.views - 1,
                                  device=device)
    ims, ov = syn.fusion_inputs(scene, seed=200 + rank)
    return scene, ims, ov


def cpu_fusion(ims, ov) -> dict:
    """The oracle's fusion loop over the whole set with the reference's
    concurrent row slices on every host core (how the reference runs
    FuseImage), and the same seed after seed on one core: fused depth maps/s."""
    import oracle.oracle as orc
    from sensemap_b200.fusion import FusionOptions
    cores = os.cpu_count() or 1
    t = time.perf_counter()
    out = orc.fusion_run(FusionOptions(), ims, ov, masks=False, threads=cores)
    dt = time.perf_counter() - t
    t = time.perf_counter()
    one = orc.fusion_run(FusionOptions(), ims, ov, masks=False)
    dt1 = time.perf_counter() - t
    return {"value": len(out["order"]) / dt, "unit": "depth maps/s", "cores": cores, "kind": "port",
            "single_thread": len(one["order"]) / dt1,
            "sample": f"oracle fusion of the whole {len(ims)}-view set, one pass with {cores} concurrent row "
                      f"slices ({dt:.2f} s, {len(out['points'])} points) and one pass seed after seed on one "
                      f"core ({dt1:.2f} s, {len(one['points'])} points)"}


def run_fusion_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import torch
    from oracle import build as oracle_build
    oracle_build.build()
    _, ims, ov = fusion_set(args, 0, "cuda" if torch.cuda.is_available() else "cpu")
    samples, cb = [], None
    steps = min(args.steps, 2)  # each step is a full CPU pass (several seconds)
    for i in range(min(args.warmup, 1) + steps):
        cb = cpu_fusion(ims, ov)
        if i >= min(args.warmup, 1):
            samples.append(cb["value"])
    value = statistics.median(samples)
    line = {"metric": FU_METRIC, "value": value, "unit": "depth maps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * len(ims) / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"fusion (StereoFusion image loop), {args.views} views {args.width}x{args.height}",
                       "global_batch": len(ims), "parallelism": "cpu, concurrent row slices on every core"},
            "cpu_baseline": {**cb, "value": value, "sample": cb["sample"] + f"; median of {steps} timed passes"},
            "e2e": {"value": value, "unit": "depth maps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_fusion(args):
    import torch
    world, rank, local = dist_setup()
    from sensemap_b200 import build as engine_build
    from sensemap_b200.fusion import FusionImage, FusionOptions, StereoFusion
    engine_build.build()
    scene, ims, ov = fusion_set(args, rank, "cuda")
    V = len(ims)

    def placed(fn):
        return [FusionImage(K=i.K, R=i.R, T=i.T, depth=fn(i.depth), normal=fn(i.normal), color=fn(i.color),
                            is_rig=i.is_rig) for i in ims]

    dev = placed(lambda a: torch.from_numpy(a).cuda())
    host = placed(lambda a: torch.from_numpy(a).pin_memory())
    opts = FusionOptions()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def step(images, fetch, profile=False):
        f = StereoFusion(opts, images, ov, stream=sptr)
        if profile:
            f.SetProfiling(True)
        f.Run()
        out = None
        if fetch:
            pts = f.GetFusedPoints()
            off, vis = f.VisibilityCSR()
            out = (pts, off, vis)
        return f, out

    for _ in range(args.warmup):
        f, _ = step(dev, False)
        f.close()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        f, _ = step(dev, False)
        launches += f.LaunchCount()
        f.close()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clock_info = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    value = args.steps * V * world / (ms / 1000.0)

    f, out = step(dev, True, profile=True)
    prof = f.Profile()
    chains, shears = f.DependencyChains(with_shear=True)
    per_image = f.ImageProfile()
    replay_times = f.ReplayTimes()
    npts = len(out[0])
    # The clean-up passes the reference's Run applies after the image loop
    # (RemoveDuplicatePoints by default, RemoveOutliers on request), on this
    # cloud, each timed on its own (each waits for its result).
    torch.cuda.synchronize()
    t = time.perf_counter()
    dup = f.RemoveDuplicatePoints()
    dup_s = time.perf_counter() - t
    t = time.perf_counter()
    outl = f.RemoveOutliers(nb_neighbors=6, max_spacing_factor=6.0)
    out_s = time.perf_counter() - t
    cleanup = {"points_fused": npts, "duplicates_removed": dup, "duplicate_pass_ms": 1000.0 * dup_s,
               "outliers_removed": outl, "outlier_pass_ms": 1000.0 * out_s,
               "outlier_pass": "exact 6-nearest-neighbour spacing on the GPU, score histogram on the host"}
    f.close()
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    px = sum(int(i.depth.shape[0]) * int(i.depth.shape[1]) for i in ims)
    # Closure launches read each traversable image's depth, point and normal
    # maps and masks (29 B/px); summed over the images in fusion order, the
    # k-th image's launch can reach the V - k images not fused yet.
    clo_n, clo_ms = prof.get("closure", (1, float("nan")))
    clo_bytes = sum(29 * px * (V - k) // V for k in range(V))
    clo_gbs = clo_bytes / (clo_ms / 1000.0) / 1e9
    roof = {"bound": "hbm", "achieved": clo_gbs, "peak": hbm, "unit": "GB/s", "frac": clo_gbs / hbm,
            "traffic": None, "kernel": "ClosureKernel", "bytes_per_launch": clo_bytes / max(clo_n, 1),
            "avg_launch_ms": clo_ms / max(clo_n, 1),
            "bytes_model": "per image fused: depth + point + normal maps and masks of every image not fused yet "
                           "read once (29 B/px)",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s",
            "kernel_ms": {k: round(v[1], 3) for k, v in prof.items()},
            "kernel_launches": {k: v[0] for k, v in prof.items()}}
    e2e = None
    if not args.no_e2e:
        f, _ = step(host, True)
        f.close()
        torch.cuda.synchronize()
        barrier(world)
        e2e_steps = min(args.steps, 5)
        t = time.perf_counter()
        for _ in range(e2e_steps):
            f, o = step(host, True)
            f.close()
        torch.cuda.synchronize()
        el = max_over_ranks(time.perf_counter() - t, world)
        h2d = sum(i.depth.numel() * 4 + i.normal.numel() * 4 + i.color.numel() for i in host)
        d2h = sum(a.nbytes for a in o)
        e2e = {"value": e2e_steps * V * world / el, "unit": "depth maps/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": e2e_steps}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_fusion(ims, ov)
    if rank == 0:
        line = {"metric": FU_METRIC, "value": value, "unit": "depth maps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"fusion (StereoFusion image loop, default options), {V} views "
                                       f"{args.width}x{args.height}, every other view overlapping; noisy "
                                       f"ground-truth depth/normal maps of the heightfield scene",
                           "global_batch": V * world, "parallelism": f"view sets sharded, {world} replica(s)",
                           "l2": f"inputs larger than L2 ({V} x {args.width}x{args.height} depth, normal and "
                                 f"color maps)"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clock_info,
                "fusion": {"points": npts, "replay_chain_steps": chains, "ticket_shear": shears, "image_ms": per_image,
                           "replay_wait_post_us_seeds": replay_times,
                           "replay_us_per_chain_step": round(1000.0 * prof["replay"][1] / max(sum(chains), 1), 3)},
                "cleanup": cleanup}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Large single view: 6000x4000 + 20 sources, 3-level pyramid
# ---------------------------------------------------------------------------
LARGE_METRIC = "seconds per depth map (24MP, 20 src, 3-level pyramid)"


def large_scene(seed=0, width=6000, height=4000, focal=6000.0, altitude=100.0):
    """The aerial terrain with buildings; a nadir reference over the centre and
    20 nadir sources on a 5 x 5 grid around it (corners and centre left out)
    spaced for 80 % overlap."""
    from sensemap_b200 import synthetic as syn
    terrain = syn.aerial_terrain(seed=seed, extent=(400.0, 400.0), num_boxes=120, texel=0.05)
    K = syn.intrinsics(focal, width, height)
    R = syn.nadir_rotation()
    sx = 0.2 * width * altitude / focal
    sy = 0.2 * height * altitude / focal
    cams = [(K, R, -R @ np.array([0.0, 0.0, altitude]), "nadir")]
    for j in range(-2, 3):
        for i in range(-2, 3):
            if (i, j) == (0, 0) or (abs(i) == 2 and abs(j) == 2):
                continue
            cams.append((K, R, -R @ np.array([i * sx, j * sy, altitude]), "nadir"))
    return terrain, cams


def run_large(args):
    """The large single view: one 24 MP reference view with 20 source views of the aerial
    scene, coarse-to-fine over 3 pyramid levels (photometric + geometric
    passes of every view at the coarsest level, then geometric passes of the
    reference at each finer level), FP16 storage against plain FP32: seconds,
    device memory and ground-truth accuracy."""
    import torch
    from dataclasses import replace
    from sensemap_b200 import STORE_F16, STORE_F32
    from sensemap_b200 import build as engine_build
    from sensemap_b200 import synthetic as syn
    from sensemap_b200.patch_match import PatchMatchOptions, View
    from sensemap_b200.pyramid import PyramidPatchMatch
    engine_build.build()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    terrain, cams = large_scene()
    dviews = syn.aerial_views(terrain, cams, seed=7, normals=False)
    _, _, gt_normal = syn.render_aerial(terrain, *cams[0][:3], dviews[0].image.shape[1], dviews[0].image.shape[0])
    log(f"large: {len(dviews)} views {dviews[0].image.shape[1]}x{dviews[0].image.shape[0]} rendered in "
        f"{time.perf_counter() - t0:.1f} s")
    dmin = min(syn.depth_range_of(v)[0] for v in dviews)
    dmax = max(syn.depth_range_of(v)[1] for v in dviews)
    V = len(dviews)
    views = [View(v.image, v.K, v.R, v.T) for v in dviews]
    problems = [(r, [i for i in range(V) if i != r]) for r in range(V)]
    gt = dviews[0].depth_gt.cpu().numpy()
    gtn = gt_normal.cpu().numpy()
    results = {}
    for name, storage in (("f32", STORE_F32), ("f16", STORE_F16)):
        opt = PatchMatchOptions(depth_min=dmin, depth_max=dmax, window_radius=RADIUS, window_step=STEP,
                                sigma_spatial=RADIUS, num_iterations=ITERS, geom_consistency_regularizer=0.1,
                                image_storage=storage)
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info()
        t = time.perf_counter()
        res = PyramidPatchMatch(opt, views, problems, levels=3, refine=[0]).Run()
        torch.cuda.synchronize()
        el = time.perf_counter() - t
        d = res.depth[0].cpu().numpy()
        n = res.normal[0].cpu().numpy()
        results[name] = {"seconds": el, "level_seconds": [round(x, 3) for x in res.level_seconds],
                         "passes": res.passes,
                         "peak_device_bytes_above_inputs": int(res.peak_device_bytes - (before[1] - before[0])),
                         "within_1pct_gt": syn.depth_accuracy(d, gt),
                         "within_10deg_normal": syn.normal_accuracy(n, gtn, mask=gt > 0)}
        log(f"large {name}: {el:.2f} s, accuracy {results[name]['within_1pct_gt']:.4f}, "
            f"memory {results[name]['peak_device_bytes_above_inputs'] / 2**30:.2f} GiB")
    line = {"metric": LARGE_METRIC, "value": results["f16"]["seconds"], "unit": "s", "n_gpus": 1, "steps": 1,
            "warmup": 0, "ms_per_step": 1000.0 * results["f16"]["seconds"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"aerial terrain with buildings, reference {dviews[0].image.shape[1]}x"
                                   f"{dviews[0].image.shape[0]} + {V - 1} sources, 3 pyramid levels (1/4: photometric "
                                   f"+ geometric pass of every view, {ITERS} iterations; 1/2 and 1: geometric pass of "
                                   f"the reference, 3 iterations), R={RADIUS}, S={STEP}",
                       "parallelism": "one GPU"},
            "forms": results,
            "accuracy_gap_pt_f16_vs_f32": 100.0 * (results["f32"]["within_1pct_gt"] - results["f16"]["within_1pct_gt"])}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Batched: 64 references of uneven size on a 200-camera ring
# ---------------------------------------------------------------------------
BATCH_METRIC = "depth maps/s (64 refs of 0.5-6 MP, 5-20 src, one batch)"


def _device_problem_views(dviews):
    from sensemap_b200.patch_match import View
    return [View(v.image, v.K, v.R, v.T) for v in dviews]


def _job_options(dmin, dmax, storage, step=STEP, seed=0):
    from sensemap_b200.patch_match import PatchMatchOptions
    return PatchMatchOptions(depth_min=dmin, depth_max=dmax, window_radius=RADIUS, window_step=step,
                             sigma_spatial=RADIUS, num_iterations=ITERS, geom_consistency=False,
                             init_depth_random=True, image_storage=storage, random_seed=seed)


def run_batched(args):
    """The batched ring: a 200-camera ring (radius 20 m, heights 2-6 m) around the
    heightfield; 64 reference views of three sizes (800x600, 1600x1200,
    3000x2000) with 5-20 nearest ring cameras as sources, one photometric pass
    each: the whole set in one batched pool (every view resident once, one
    launch per checkerboard kernel for all jobs, each iteration a CUDA graph)
    against the plain path (one engine per job, FP32 storage)."""
    import torch
    from sensemap_b200 import STORE_F16, STORE_F32
    from sensemap_b200 import build as engine_build
    from sensemap_b200 import synthetic as syn
    from sensemap_b200.patch_match import PatchMatchACMMCuda, Problem, autotune
    from sensemap_b200.pool import DepthMapPool
    engine_build.build()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    terrain = syn.ring_terrain(seed=0)
    cams = syn.ring_cameras(200)
    dviews = syn.aerial_views(terrain, cams, seed=3)
    log(f"batched: {len(dviews)} ring views rendered in {time.perf_counter() - t0:.1f} s")
    gen = np.random.default_rng(5)
    refs = sorted(gen.choice(len(dviews), size=64, replace=False).tolist())
    jobs = []
    for r in refs:
        k = int(gen.integers(5, 21))
        order = sorted((i for i in range(len(dviews)) if i != r),
                       key=lambda i: (min(abs(i - r), len(dviews) - abs(i - r)), i))
        jobs.append((r, order[:k]))
    ranges = {r: syn.depth_range_of(dviews[r]) for r, _ in jobs}
    views = _device_problem_views(dviews)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    r0, s0 = jobs[0]
    tune = autotune(_job_options(*ranges[r0], STORE_F16), Problem(r0, s0, views), stream=sptr, repeats=2)

    def pool_pass(storage, step):
        pool = DepthMapPool(memory_budget_bytes=120 << 30, max_active_jobs=len(jobs), image_storage=storage,
                            sweep_block_x=tune["sweep_block_x"], threads_per_pixel=tune["threads_per_pixel"],
                            persistent=tune["persistent"], stream=sptr)
        for i, v in enumerate(views):
            pool.add_view(i, v)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ids = [pool.submit(_job_options(*ranges[r], storage, step, seed=r), r, srcs) for r, srcs in jobs]
        pool.run_until_done(ids)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        acc = [syn.depth_accuracy(pool.get_map(j, 0), dviews[r].depth_gt.cpu().numpy()) for j, (r, _) in
               zip(ids, jobs)]
        st = pool.stats()
        pool.close()
        return ms, acc, st

    pool_pass(STORE_F16, STEP)  # warm-up (graph capture, scratch, texture caches)
    ms16, acc16, st16 = pool_pass(STORE_F16, STEP)
    ms2, acc2, _ = pool_pass(STORE_F16, 2)
    # The plain path: one engine per job, FP32 storage, default launch shape.
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    plain_acc = []
    for r, srcs in jobs:
        with PatchMatchACMMCuda(_job_options(*ranges[r], STORE_F32, seed=r), Problem(r, srcs, views),
                                stream=sptr) as pm:
            pm.Run()
            plain_acc.append(syn.depth_accuracy(pm.GetDepthMap(), dviews[r].depth_gt.cpu().numpy()))
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_plain = ev0.elapsed_time(ev1)
    n = len(jobs)
    mp = sum(dviews[r].image.numel() for r, _ in jobs) / 1e6
    plain_value = n / (ms_plain / 1000.0)
    gap2 = 100.0 * (float(np.mean(plain_acc)) - float(np.mean(acc2)))
    line = {"metric": BATCH_METRIC, "value": n / (ms16 / 1000.0), "unit": "depth maps/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": ms16, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"200-camera ring around the heightfield, {n} references "
                                   f"({sum(1 for r, _ in jobs if dviews[r].image.shape[1] == 800)} x 800x600, "
                                   f"{sum(1 for r, _ in jobs if dviews[r].image.shape[1] == 1600)} x 1600x1200, "
                                   f"{sum(1 for r, _ in jobs if dviews[r].image.shape[1] == 3000)} x 3000x2000; "
                                   f"{mp:.0f} MP in all), 5-20 nearest sources, photometric pass (R={RADIUS}, "
                                   f"S={STEP}, {ITERS} iterations), FP16 storage, every job in one batch",
                       "parallelism": "one GPU"},
            "batched": {"value": n / (ms16 / 1000.0), "within_1pct_gt": float(np.mean(acc16)),
                        "graphs_built": st16["graphs_built"], "launches": st16["launches"], "autotune": tune},
            "plain": {"value": plain_value, "within_1pct_gt": float(np.mean(plain_acc)),
                      "form": "one engine per job, FP32 storage, default launch shape"},
            "ratio_vs_plain": (n / (ms16 / 1000.0)) / plain_value,
            "autotuned_window": {"window_step": 2, "value": n / (ms2 / 1000.0),
                                 "within_1pct_gt": float(np.mean(acc2)), "accuracy_gap_pt_vs_plain": gap2,
                                 "accepted": gap2 <= 0.5, "ratio_vs_plain": (n / (ms2 / 1000.0)) / plain_value}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Serving: Poisson job streams over a 400-camera aerial survey
# ---------------------------------------------------------------------------
SERVE_METRIC = "p50/p99 depth-map job latency (s) at Poisson arrival rates, 400-camera aerial survey"


def run_serving_aerial(args):
    """Aerial serving: an aerial survey of 400 cameras (20 x 20 stations at 100 m,
    80 % overlap, nadir and 45-degree obliques) over terrain with buildings,
    2000x1500 images kept in pinned host memory (8-bit); depth-map jobs (one
    photometric pass of a reference with its 8-16 nearest cameras of similar
    direction) arrive as Poisson streams. The pool admits them continuously,
    uploads views from host memory on first use and keeps them resident under
    a 120 GB budget (least recently used first out). Latency = completion
    minus arrival; the plain path (one engine per job in arrival order, FP32
    storage) serves the same stream at the lower rates."""
    import torch
    from sensemap_b200 import STORE_F16, STORE_F32
    from sensemap_b200 import build as engine_build
    from sensemap_b200 import serving as srv
    from sensemap_b200 import synthetic as syn
    from sensemap_b200.patch_match import PatchMatchACMMCuda, Problem, View, autotune
    from sensemap_b200.pool import DepthMapPool
    engine_build.build()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    terrain = syn.aerial_terrain(seed=1)
    cams = syn.aerial_grid_cameras()
    dviews = syn.aerial_views(terrain, cams, seed=4)
    # Host copies (8-bit, pinned) are what the service receives; the device
    # renders are dropped once copied, except the ground truth.
    host = [v.image.to(torch.uint8).cpu().pin_memory() for v in dviews]
    gts = [v.depth_gt for v in dviews]
    for v in dviews:
        v.image = None
    torch.cuda.empty_cache()
    log(f"serving: {len(dviews)} aerial views rendered in {time.perf_counter() - t0:.1f} s")
    rates = [float(x) for x in args.serving_rates.split(",")]
    jobs_per_rate = args.serving_jobs
    gen = np.random.default_rng(9)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def job_spec(k, storage, step):
        r = int(gen.integers(0, len(dviews)))
        srcs = syn.nearest_sources(dviews, r, int(gen.integers(8, 17)))
        d = gts[r]
        valid = d[d > 0]
        o = _job_options(float(valid.min()) * 0.9, float(valid.max()) * 1.1, storage, step, seed=10000 + k)
        return srv.JobSpec(o, r, srcs)

    def view_of(i):
        v = dviews[i]
        return View(host[i], v.K, v.R, v.T)

    r0 = 0
    probe = job_spec(0, STORE_F16, STEP)
    tune_views = [view_of(i) if i in [probe.ref_view] + probe.src_views else None for i in range(len(dviews))]
    tune = autotune(probe.options, Problem(probe.ref_view, probe.src_views, tune_views), stream=sptr, repeats=2)
    results = []
    for step in (STEP, 2):
        for rate in rates:
            specs = [job_spec(k, STORE_F16, step) for k in range(jobs_per_rate)]
            arrivals = srv.poisson_arrivals(rate, jobs_per_rate, seed=int(rate * 100) + step)
            pool = DepthMapPool(memory_budget_bytes=120 << 30, max_active_jobs=16, image_storage=STORE_F16,
                                sweep_block_x=tune["sweep_block_x"], threads_per_pixel=tune["threads_per_pixel"],
                                persistent=tune["persistent"], stream=sptr)
            acc = []

            def ensure(spec, pool=pool):
                for i in [spec.ref_view] + list(spec.src_views):
                    if not pool.has_view(i):
                        pool.add_view(i, view_of(i))

            def done(k, jid, pool=pool, specs=specs, acc=acc):
                if len(acc) < 16:
                    acc.append(syn.depth_accuracy(pool.get_map(jid, 0), gts[specs[k].ref_view].cpu().numpy()))
                pool.release(jid)

            res = srv.serve(pool, specs, arrivals, on_done=done, before_submit=ensure)
            st = pool.stats()
            pool.close()
            res.pop("latencies")
            res.update({"form": "pool", "window_step": step, "arrival_rate_jobs_s": rate,
                        "within_1pct_gt_first_jobs": float(np.mean(acc)), "evictions": st["evictions"],
                        "graphs_built": st["graphs_built"], "views_resident_at_end": st["views_resident"]})
            log(f"serving pool S={step} rate {rate}: p50 {res['p50_s']:.3f} p99 {res['p99_s']:.3f} "
                f"thr {res['throughput_jobs_s']:.2f} jobs/s")
            results.append(res)
    # The plain path at the lower rates.
    for rate in rates[:2]:
        specs = [job_spec(k, STORE_F32, STEP) for k in range(jobs_per_rate)]
        arrivals = srv.poisson_arrivals(rate, jobs_per_rate, seed=int(rate * 100) + 7)
        lat = np.zeros(len(specs))
        acc = []
        t0 = time.perf_counter()
        for k, spec in enumerate(specs):
            now = time.perf_counter() - t0
            if arrivals[k] > now:
                time.sleep(arrivals[k] - now)
            vs = [view_of(i) if i in [spec.ref_view] + spec.src_views else None for i in range(len(dviews))]
            with PatchMatchACMMCuda(spec.options, Problem(spec.ref_view, spec.src_views, vs), stream=sptr) as pm:
                pm.Run()
                d = pm.GetDepthMap()
            lat[k] = time.perf_counter() - t0 - arrivals[k]
            if len(acc) < 16:
                acc.append(syn.depth_accuracy(d, gts[spec.ref_view].cpu().numpy()))
        wall = time.perf_counter() - t0
        results.append({"form": "plain", "window_step": STEP, "arrival_rate_jobs_s": rate, "jobs": len(specs),
                        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                        "mean_s": float(lat.mean()), "throughput_jobs_s": len(specs) / wall,
                        "within_1pct_gt_first_jobs": float(np.mean(acc))})
        log(f"serving plain rate {rate}: p50 {results[-1]['p50_s']:.3f} p99 {results[-1]['p99_s']:.3f}")
    main_res = [r for r in results if r["form"] == "pool" and r["window_step"] == STEP]
    line = {"metric": SERVE_METRIC, "value": main_res[0]["p99_s"], "unit": "s", "n_gpus": 1, "steps": len(results),
            "warmup": 0, "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"aerial survey: {len(dviews)} cameras 2000x1500 (20 x 20 stations, 100 m, 80 % "
                                   f"overlap, nadir + 4 x 45-degree obliques) over terrain with "
                                   f"{len(terrain.boxes)} buildings; jobs = photometric pass (R={RADIUS}, "
                                   f"{ITERS} iterations) of a random reference with 8-16 nearest sources; "
                                   f"{jobs_per_rate} Poisson jobs per rate; 120 GB view budget, LRU",
                       "parallelism": "one GPU"},
            "autotune": tune, "runs": results}
    print(json.dumps(line), flush=True)


def ctypes_rate(N, kind):
    import ctypes as C
    r = C.c_double()
    N.check(N.lib().smvs_test_calibrate(kind, 0.5, C.byref(r)))
    return r.value


if __name__ == "__main__":
    main()
