"""The serving loop (sensemap_b200.serving.serve) against a fake pool and a
fake clock, on the CPU: jobs are submitted when they arrive, every step
advances all admitted jobs, each job's latency is its completion time minus
its arrival time, and a failed job stops the loop with an error instead of
being waited for forever."""
import numpy as np
import pytest

from sensemap_b200 import _native as N
from sensemap_b200.serving import JobSpec, poisson_arrivals, serve


class FakeClock:
    """Advances by `tick` seconds on every reading."""

    def __init__(self, tick=0.01):
        self.t, self.tick = 0.0, tick

    def __call__(self):
        self.t += self.tick
        return self.t


class FakePool:
    """Each job needs `iters` steps; a job listed in `fail` fails instead."""

    def __init__(self, iters=3, fail=()):
        self.iters, self.fail = iters, set(fail)
        self.left, self.submitted, self.steps = {}, [], 0

    def submit(self, options, ref, srcs):
        jid = len(self.submitted) + 1
        self.submitted.append((jid, ref, self.steps))
        self.left[jid] = self.iters
        return jid

    def step(self):
        self.steps += 1
        for jid in self.left:
            self.left[jid] = max(0, self.left[jid] - 1)

    def state(self, jid):
        if jid in self.fail and self.left[jid] == 0:
            return N.JOB_FAILED, 0.0
        return (N.JOB_DONE if self.left[jid] == 0 else N.JOB_ACTIVE), 0.0


def test_poisson_arrivals_are_increasing_with_the_requested_rate():
    a = poisson_arrivals(5.0, 4000, seed=3)
    assert np.all(np.diff(a) > 0)
    assert abs(4000 / a[-1] - 5.0) < 0.3


def test_serve_admits_jobs_as_they_arrive_and_reports_latency():
    specs = [JobSpec(None, r, [r + 1]) for r in range(6)]
    arrivals = np.array([0.0, 0.0, 0.05, 0.3, 0.31, 0.9])
    pool, done = FakePool(iters=3), []
    out = serve(pool, specs, arrivals, on_done=lambda k, jid: done.append(k), time_fn=FakeClock())
    assert out["jobs"] == 6 and sorted(done) == list(range(6))
    # Submission order follows arrival order, and later arrivals join while
    # earlier jobs are still running (continuous admission).
    assert [ref for _, ref, _ in pool.submitted] == list(range(6))
    assert pool.submitted[2][2] < pool.iters  # job 2 joined before jobs 0-1 finished
    lat = out["latencies"]
    assert np.all(lat > 0)
    assert out["p50_s"] == pytest.approx(float(np.percentile(lat, 50)))
    assert out["p99_s"] == pytest.approx(float(np.percentile(lat, 99)))
    assert out["max_s"] == pytest.approx(float(lat.max()))


def test_serve_raises_on_a_failed_job():
    specs = [JobSpec(None, r, [r + 1]) for r in range(3)]
    with pytest.raises(RuntimeError, match="failed"):
        serve(FakePool(iters=2, fail={2}), specs, np.zeros(3), time_fn=FakeClock())


def test_pool_run_until_done_raises_on_a_failed_job():
    """DepthMapPool.run_until_done with its native calls replaced: it steps until
    every job is done and stops at once when one fails."""
    from sensemap_b200.pool import DepthMapPool
    pool = object.__new__(DepthMapPool)  # no native pool behind it
    states = {1: N.JOB_ACTIVE, 2: N.JOB_ACTIVE}
    steps = [0]

    def step():
        steps[0] += 1
        if steps[0] == 2:
            states[1], states[2] = N.JOB_DONE, N.JOB_FAILED

    pool.state = lambda j: (states[j], 0.0)
    pool.step = step
    with pytest.raises(RuntimeError, match="job 2 failed"):
        pool.run_until_done([1, 2])
    assert steps[0] == 2
    states[2] = N.JOB_DONE
    pool.run_until_done([1, 2])  # both done: returns without stepping
    assert steps[0] == 2
