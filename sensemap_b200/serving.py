"""Continuous-batching serving loop over a DepthMapPool.

Depth-map jobs arrive as a Poisson process; each loop turn submits the jobs
that have arrived, advances every admitted job one PatchMatch iteration in
one batched step, and records the completion latency (completion minus
arrival) of the jobs that finished. Jobs arriving while others are on the GPU
join the batch as soon as a slot and memory are free.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class JobSpec:
    options: object          # PatchMatchOptions
    ref_view: int
    src_views: list


def poisson_arrivals(rate_per_s: float, count: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=count))


def serve(pool, specs, arrivals, on_done=None, time_fn=time.perf_counter, before_submit=None) -> dict:
    """Run `specs[i]` arriving at `arrivals[i]` seconds; returns latency stats.
    `on_done(i, job_id)` is called for each finished job (e.g. to read maps);
    `before_submit(spec)` before a job is submitted (e.g. to make its views
    resident). A job that fails raises RuntimeError (the other jobs stay in the
    pool)."""
    t0 = time_fn()
    pending = 0
    i = 0
    live = {}                 # job id -> spec index
    latency = np.zeros(len(specs))
    steps = 0
    while i < len(specs) or live:
        now = time_fn() - t0
        while i < len(specs) and arrivals[i] <= now:
            s = specs[i]
            if before_submit is not None:
                before_submit(s)
            live[pool.submit(s.options, s.ref_view, s.src_views)] = i
            i += 1
        if not live:
            # Idle: wait for the next arrival.
            time.sleep(max(0.0, min(0.002, arrivals[i] - (time_fn() - t0))))
            continue
        pool.step()
        steps += 1
        now = time_fn() - t0
        for jid in list(live):
            st, _ = pool.state(jid)
            if st == N.JOB_DONE:
                k = live.pop(jid)
                latency[k] = now - arrivals[k]
                if on_done is not None:
                    on_done(k, jid)
            elif st == N.JOB_FAILED:
                raise RuntimeError(f"serving: job {jid} (request {live[jid]}) failed")
    total = time_fn() - t0
    return {"jobs": len(specs), "wall_s": total, "throughput_jobs_s": len(specs) / total,
            "p50_s": float(np.percentile(latency, 50)), "p99_s": float(np.percentile(latency, 99)),
            "mean_s": float(latency.mean()), "max_s": float(latency.max()), "steps": steps, "latencies": latency}
