"""Resident views, batched jobs and continuous admission (the C ABI's smvs_pool).

``DepthMapPool`` keeps views in HBM under a byte budget, queues depth-map jobs
(a reference view, its source views and PatchMatchOptions) and advances every
admitted job one PatchMatch iteration per ``step()`` in batched launches.
Jobs that arrive while others run are admitted as slots and memory free up;
each job's maps are the same as when it runs alone.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .patch_match import PatchMatchOptions, View, _addr, _is_cuda_tensor


class DepthMapPool:
    def __init__(self, memory_budget_bytes: int = 16 << 30, max_active_jobs: int = 64, image_storage: int = N.STORE_U8,
                 sweep_block_x: int = 32, use_graphs: bool = True, gpu_index: int = -1, stream=None,
                 ref_tile_tma: bool = True, threads_per_pixel: int = 1, persistent: bool = False):
        o = N.smvs_pool_options()
        N.check(N.lib().smvs_pool_options_default(C.byref(o)))
        o.memory_budget_bytes = int(memory_budget_bytes)
        o.max_active_jobs = int(max_active_jobs)
        o.image_storage = int(image_storage)
        o.sweep_block_x = int(sweep_block_x)
        o.use_graphs = int(use_graphs)
        o.gpu_index = int(gpu_index)
        o.ref_tile_tma = int(ref_tile_tma)
        o.sweep_threads_per_pixel = int(threads_per_pixel)
        o.sweep_persistent = int(persistent)
        h = C.c_void_p()
        N.check(N.lib().smvs_pool_create(C.byref(o), C.c_void_p(int(stream)) if stream is not None else None,
                                         C.byref(h)))
        self._h = h
        self._shapes = {}   # view id -> (H, W)
        self._jobs = {}     # job id -> (H, W, N)

    def add_view(self, view_id: int, view: View) -> None:
        img = view.image
        if _is_cuda_tensor(img):
            fmt = N.PIX_U8 if str(img.dtype) == "torch.uint8" else N.PIX_F32
            if fmt == N.PIX_F32 and str(img.dtype) != "torch.float32":
                img = img.float()
        else:
            img = np.asarray(img)
            fmt = N.PIX_U8 if img.dtype == np.uint8 else N.PIX_F32
            if fmt == N.PIX_F32:
                img = np.ascontiguousarray(img, dtype=np.float32)
        ptr, keep, dev = _addr(img)
        cv = N.smvs_view()
        cv.width, cv.height, cv.pixel_format, cv.row_stride = view.width, view.height, fmt, 0
        cv.pixels = ptr
        cv.K[:] = [float(a) for a in np.asarray(view.K, np.float64).reshape(9)]
        cv.R[:] = [float(a) for a in np.asarray(view.R, np.float64).reshape(9)]
        cv.T[:] = [float(a) for a in np.asarray(view.T, np.float64).reshape(3)]
        cv.scale = 1.0
        N.check(N.lib().smvs_pool_add_view(self._h, int(view_id), C.byref(cv), N.MEM_DEVICE if dev else N.MEM_HOST))
        self._shapes[int(view_id)] = (view.height, view.width)
        del keep

    def has_view(self, view_id: int) -> bool:
        r = C.c_int()
        N.check(N.lib().smvs_pool_has_view(self._h, int(view_id), C.byref(r)))
        return bool(r.value)

    def set_view_maps(self, view_id: int, depth, normal=None) -> None:
        dp, dk, ddev = _addr(depth if _is_cuda_tensor(depth) else np.asarray(depth, np.float32))
        np_, nk, _ = _addr(None if normal is None else (normal if _is_cuda_tensor(normal)
                                                        else np.asarray(normal, np.float32)))
        N.check(N.lib().smvs_pool_set_view_maps(self._h, int(view_id), dp, np_, N.MEM_DEVICE if ddev else N.MEM_HOST))
        del dk, nk

    def submit(self, options: PatchMatchOptions, ref_view: int, src_views) -> int:
        srcs = (C.c_int64 * len(src_views))(*[int(s) for s in src_views])
        jid = C.c_int64()
        N.check(N.lib().smvs_pool_submit(self._h, C.byref(options.to_c()), int(ref_view), srcs, len(src_views),
                                         C.byref(jid)))
        H, W = self._shapes[int(ref_view)]
        self._jobs[jid.value] = (H, W, len(src_views))
        return jid.value

    def step(self) -> dict:
        s = N.smvs_pool_stats()
        N.check(N.lib().smvs_pool_step(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in N.smvs_pool_stats._fields_}

    def stats(self) -> dict:
        s = N.smvs_pool_stats()
        N.check(N.lib().smvs_pool_stats_get(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in N.smvs_pool_stats._fields_}

    def state(self, job: int):
        st, lat = C.c_int(), C.c_double()
        N.check(N.lib().smvs_pool_job_state(self._h, int(job), C.byref(st), C.byref(lat)))
        return st.value, lat.value

    def wait(self, job: int, timeout_s: float) -> int:
        """Step until the job is done or failed (smvs_pool_wait); raises
        SmvsError(SMVS_ETIMEDOUT) after timeout_s seconds. Returns its state."""
        st = C.c_int()
        N.check(N.lib().smvs_pool_wait(self._h, int(job), float(timeout_s), C.byref(st)))
        return st.value

    def run_until_done(self, jobs, max_steps: int = 100000) -> None:
        """Step until every job in `jobs` is done; a failed job raises at once."""
        for _ in range(max_steps):
            states = [self.state(j)[0] for j in jobs]
            if any(st == N.JOB_FAILED for st in states):
                raise RuntimeError(f"job {jobs[states.index(N.JOB_FAILED)]} failed")
            if all(st == N.JOB_DONE for st in states):
                return
            self.step()
        raise RuntimeError("jobs did not finish")

    def get_map(self, job: int, which: int, out=None):
        """A done job's map (smvs_pool_get_map). `out`, if given, receives it: a
        contiguous numpy array or torch tensor (pinned host memory copies at
        full DMA rate; a CUDA tensor gets a device copy) of the map's size."""
        H, W, Nn = self._jobs[job]
        shape, dtype = {N.MAP_DEPTH: ((H, W), np.float32), N.MAP_NORMAL: ((3, H, W), np.float32),
                        N.MAP_CONF: ((H, W), np.float32), N.MAP_COST: ((Nn, H, W), np.float32),
                        N.MAP_VIEW_SEL: ((H, W), np.uint32)}[which]
        if out is None:
            out = np.empty(shape, dtype)
        nbytes = int(np.prod(shape)) * 4
        if isinstance(out, np.ndarray):
            if not out.flags.c_contiguous or not out.flags.writeable or out.nbytes != nbytes:
                raise ValueError(f"out must be a writable contiguous array of {nbytes} bytes")
            ptr = out.ctypes.data
        else:  # torch tensor
            if not out.is_contiguous() or out.numel() * out.element_size() != nbytes:
                raise ValueError(f"out must be a contiguous tensor of {nbytes} bytes")
            ptr = out.data_ptr()
        N.check(N.lib().smvs_pool_get_map(self._h, int(job), int(which), C.c_void_p(ptr)))
        return out

    def maps(self, job: int) -> dict:
        return {"depth": self.get_map(job, N.MAP_DEPTH), "normal": self.get_map(job, N.MAP_NORMAL),
                "conf": self.get_map(job, N.MAP_CONF), "cost": self.get_map(job, N.MAP_COST),
                "view_sel": self.get_map(job, N.MAP_VIEW_SEL)}

    def keep_maps(self, job: int) -> None:
        N.check(N.lib().smvs_pool_keep_maps(self._h, int(job)))

    def release(self, job: int) -> None:
        N.check(N.lib().smvs_pool_release(self._h, int(job)))
        self._jobs.pop(job, None)

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().smvs_pool_destroy(self._h)
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
