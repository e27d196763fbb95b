"""Batched jobs and continuous admission (smvs_pool) against the single-job
engine: identical maps for every job, alone or in any mix, with views of
different sizes and source counts in one batch."""
import numpy as np
import pytest

from sensemap_b200 import _native as N
from sensemap_b200 import synthetic as syn
from sensemap_b200.patch_match import PatchMatchACMMCuda, View
from sensemap_b200.pool import DepthMapPool
from tests.helpers import photometric_options, problem_from_scene, small_planes

pytestmark = pytest.mark.gpu


def engine_maps(opt, prob):
    with PatchMatchACMMCuda(opt, prob) as pm:
        pm.Run()
        return {"depth": pm.GetDepthMap(), "normal": pm.GetNormalMap(), "conf": pm.GetConfMap(),
                "cost": pm.GetCostMap(), "view_sel": pm.GetViewSelMap()}


def assert_same(a, b):
    for k in ("depth", "normal", "conf", "cost", "view_sel"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.fixture(scope="module")
def scenes():
    return [small_planes(seed=41), syn.heightfield_scene(seed=42, width=112, height=84, focal=90.0, num_src=3)]


def add_scene(pool, scene, base):
    for i, v in enumerate(scene.views):
        pool.add_view(base + i, View(v.image, v.K, v.R, v.T))


@pytest.mark.parametrize("persistent,cap", [(False, 0), (True, 0), (True, 5)])
def test_batched_jobs_match_single_engine(scenes, persistent, cap):
    """Persistent launches too: with a cap of 5 blocks each block loops over
    the tiles of every job of the batch (jobs of two image sizes, 4 and 5
    iterations, so the batch changes while they run)."""
    jobs = []
    N.check(N.lib().smvs_test_persistent_grid(cap))
    try:
        with DepthMapPool(max_active_jobs=8, persistent=persistent) as pool:
            for si, sc in enumerate(scenes):
                add_scene(pool, sc, 100 * si)
                for r in (0, 1):
                    opt = photometric_options(sc, iters=4 + r, random_seed=10 * si + r)
                    srcs = [100 * si + i for i in range(len(sc.views)) if i != r]
                    jobs.append((pool.submit(opt, 100 * si + r, srcs), sc, r, opt))
            pool.run_until_done([j[0] for j in jobs])
            st = pool.stats()
            assert st["graphs_built"] >= 1 and st["done"] == len(jobs)
            for jid, sc, r, opt in jobs:
                assert_same(pool.maps(jid), engine_maps(opt, problem_from_scene(sc, ref=r)))
    finally:
        N.check(N.lib().smvs_test_persistent_grid(0))


def test_job_alone_equals_job_in_mix(scenes):
    sc = scenes[0]
    opt = photometric_options(sc, iters=6, random_seed=5)
    srcs = [i for i in range(1, len(sc.views))]
    with DepthMapPool(max_active_jobs=4) as pool:
        add_scene(pool, sc, 0)
        alone = pool.submit(opt, 0, srcs)
        pool.run_until_done([alone])
        ref_maps = pool.maps(alone)
    with DepthMapPool(max_active_jobs=2) as pool:
        add_scene(pool, sc, 0)
        add_scene(pool, scenes[1], 100)
        others = [pool.submit(photometric_options(scenes[1], iters=4, random_seed=9), 100, [101, 102, 103])]
        pool.step()
        pool.step()
        mixed = pool.submit(opt, 0, srcs)          # arrives while another job is on the GPU
        others.append(pool.submit(photometric_options(sc, iters=3, random_seed=3), 1, [0, 2, 3, 4]))  # queued: 2 slots
        pool.run_until_done([mixed] + others)
        assert_same(pool.maps(mixed), ref_maps)


def test_wait_steps_until_done_or_times_out(scenes):
    """smvs_pool_wait steps the pool for one job: with no time it reports
    SMVS_ETIMEDOUT and the job keeps its place; given time it returns the job
    done, with the maps of a job run to completion by explicit steps."""
    sc = scenes[0]
    opt = photometric_options(sc, iters=4, random_seed=6)
    srcs = [i for i in range(1, len(sc.views))]
    with DepthMapPool(max_active_jobs=2) as pool:
        add_scene(pool, sc, 0)
        job = pool.submit(opt, 0, srcs)
        with pytest.raises(N.SmvsError) as ei:
            pool.wait(job, 0.0)
        assert ei.value.status == N.SMVS_ETIMEDOUT
        assert pool.wait(job, 60.0) == N.JOB_DONE
        waited = pool.maps(job)
    with DepthMapPool(max_active_jobs=2) as pool:
        add_scene(pool, sc, 0)
        job = pool.submit(opt, 0, srcs)
        pool.run_until_done([job])
        assert_same(waited, pool.maps(job))


def test_geometric_pass_through_pool_matches_engine(scenes):
    sc = scenes[0]
    n = len(sc.views)
    with DepthMapPool(max_active_jobs=n) as pool:
        add_scene(pool, sc, 0)
        photo = [pool.submit(photometric_options(sc, iters=4, random_seed=i), i, [j for j in range(n) if j != i])
                 for i in range(n)]
        pool.run_until_done(photo)
        maps = [pool.maps(j) for j in photo]
        for j in photo:
            pool.keep_maps(j)
        gopt = photometric_options(sc, iters=3, geom_consistency=True, init_depth_random=False,
                                   geom_consistency_regularizer=0.1, random_seed=77)
        geo = pool.submit(gopt, sc.ref_index, [j for j in range(n) if j != sc.ref_index])
        pool.run_until_done([geo])
        got = pool.maps(geo)
    prob = problem_from_scene(sc, depth_maps=[m["depth"] for m in maps], normal_maps=[m["normal"] for m in maps])
    assert_same(got, engine_maps(gopt, prob))


def test_budget_evicts_unreferenced_views_and_rejects_oversized_jobs(scenes):
    sc = scenes[0]
    H, W = sc.views[0].image.shape
    per_view = W * H * 5
    with DepthMapPool(memory_budget_bytes=per_view * 7 + 4096 * 7, max_active_jobs=2) as pool:
        add_scene(pool, sc, 0)                       # 5 views fit
        add_scene(pool, scenes[1], 100)              # evicts least recently used views
        assert pool.stats()["evictions"] > 0
        assert not pool.has_view(0)
        add_scene(pool, sc, 0)
        jid = pool.submit(photometric_options(sc, iters=2), 0, [1, 2, 3, 4])
        with pytest.raises(N.SmvsError) as ei:       # its state does not fit the budget
            pool.step()
        assert ei.value.status == N.SMVS_ENOMEM
        pool.release(jid)


def test_ring_of_uneven_views_batched():
    """The batched configuration in small: a ring of cameras of three sizes
    around the heightfield, reference views with 3-12 nearest sources, all
    jobs admitted into one pool (one launch per kernel per window/view bucket)
    and each result identical to the single-job engine."""
    sc, jobs = syn.ring_scene(seed=2, num_cameras=20, scale=0.1, num_refs=6, min_src=3, max_src=12, device="cuda")
    assert len({v.image.shape for v in sc.views}) > 1
    assert len({len(s) for _, s in jobs}) > 1
    results = []
    with DepthMapPool(max_active_jobs=len(jobs)) as pool:
        add_scene(pool, sc, 0)
        for k, (r, srcs) in enumerate(jobs):
            opt = photometric_options(sc, iters=4, random_seed=300 + k)
            results.append((pool.submit(opt, r, srcs), r, srcs, opt))
        pool.run_until_done([j[0] for j in results])
        for jid, r, srcs, opt in results:
            assert_same(pool.maps(jid), engine_maps(opt, problem_from_scene(sc, ref=r, src=srcs)))


def test_get_map_into_caller_buffers(scenes):
    """Maps read into a pinned host tensor, a CUDA tensor and a numpy array
    equal the getter's own array; a buffer of the wrong size is rejected."""
    import torch
    sc = scenes[0]
    with DepthMapPool(max_active_jobs=2) as pool:
        add_scene(pool, sc, 0)
        job = pool.submit(photometric_options(sc, iters=2, random_seed=8), 0, [1, 2, 3, 4])
        pool.run_until_done([job])
        want = pool.get_map(job, N.MAP_NORMAL)
        pinned = pool.get_map(job, N.MAP_NORMAL, out=torch.empty(want.shape, dtype=torch.float32).pin_memory())
        cuda = pool.get_map(job, N.MAP_NORMAL, out=torch.empty(want.shape, dtype=torch.float32, device="cuda"))
        arr = pool.get_map(job, N.MAP_NORMAL, out=np.empty(want.shape, np.float32))
        np.testing.assert_array_equal(pinned.numpy(), want)
        np.testing.assert_array_equal(cuda.cpu().numpy(), want)
        np.testing.assert_array_equal(arr, want)
        with pytest.raises(ValueError):
            pool.get_map(job, N.MAP_NORMAL, out=np.empty(want.shape[1:], np.float32))
