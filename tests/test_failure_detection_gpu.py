"""Failure detection on the GPU in the allowed form: a bounded device wait is
made to run out (a copy or a release that never comes), the kernel returns
with an error status, the API reports SMVS_ETIMEDOUT, and the context stays
usable for the next run. Nothing faults or hangs: every wait has a limit.

Replaces the reference's failure handling, which exits the process
(CudaSafeCall / CudaSyncAndCheck, src/util/cudacc.cc:30-64)."""
import ctypes as C

import numpy as np
import pytest

from sensemap_b200 import _native as N
from sensemap_b200.patch_match import PatchMatchACMMCuda
from tests.helpers import photometric_options, problem_from_scene, small_planes

pytestmark = pytest.mark.gpu


def test_tile_wait_that_runs_out_reports_timeout_and_context_survives():
    scene = small_planes(seed=41, w=200, h=120)  # rows of 800 bytes: tiles go through TMA
    opt = photometric_options(scene, iters=2)
    with PatchMatchACMMCuda(opt, problem_from_scene(scene)) as pm:
        pm.SetTuning(32, True, 1)
        # The tile copy is never issued; each block gives up after 64 polls.
        N.check(N.lib().smvs_test_tile_waits(pm._h, 64, 1))
        pm.Run()
        with pytest.raises(N.SmvsError) as err:
            pm.GetDepthMap()
        assert err.value.status == N.SMVS_ETIMEDOUT
        assert pm.Tuning()["ref_tile_tma"]
    # The same problem runs normally afterwards on the same context.
    with PatchMatchACMMCuda(opt, problem_from_scene(scene)) as pm:
        pm.Run()
        d = pm.GetDepthMap()
    assert np.isfinite(d).all() and (d > 0).mean() > 0.9


def test_fusion_wait_that_runs_out_reports_timeout_and_context_survives():
    from sensemap_b200 import synthetic as syn
    from sensemap_b200.fusion import FusionOptions, StereoFusion
    scene = syn.heightfield_scene(seed=3, width=160, height=120, focal=120.0, num_src=4)
    ims, ov = syn.fusion_inputs(scene, seed=5)
    # No seed releases its successors; every wait for a predecessor gives up
    # after 50 ms.
    N.check(N.lib().smvs_test_fusion_waits(0.05, -2))
    try:
        f = StereoFusion(FusionOptions(), ims, ov)
        with pytest.raises(N.SmvsError) as err:
            f.Run()
        assert err.value.status == N.SMVS_ETIMEDOUT
        f.close()
    finally:
        N.check(N.lib().smvs_test_fusion_waits(0.0, -1))
    f = StereoFusion(FusionOptions(), ims, ov)
    f.Run()
    assert len(f.GetFusedPoints()) > 0
    f.close()
