"""The failure path of the kernels' bounded waits, exercised without a fault.

The fitter waits on its bulk copies with a time limit; when a limit runs out
the kernel records a status word, leaves, and bmfr_plan_check_device reports
BMFR_E_TIMEOUT.  Here a diagnostic kernel waits with the same bounded wait
on a barrier that nothing completes (a 20 ms limit): the host must see the
timeout, the status must clear, and the same plan must then denoise frames
exactly as before.
"""
import numpy as np
import pytest

import bmfr_b200 as B
from oracle.oracle import Oracle, OraclePipeline

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_the_plan_recovers(cuda):
    W, H = 64, 64
    sc = B.Scene(4, W, H, 8)
    plan = B.Plan(W, H, position_limit_squared=sc.position_limit_squared,
                  normal_limit_squared=sc.normal_limit_squared)
    plan.check_device()                        # clean to begin with
    plan.probe_bounded_wait(20000)
    with pytest.raises(B.BmfrError) as e:
        plan.check_device()
    assert e.value.status == B._native.BMFR_E_TIMEOUT
    plan.check_device()                        # the status was cleared

    ref = OraclePipeline(Oracle(W, H, sc.position_limit_squared, sc.normal_limit_squared))
    for f in range(2):
        d = sc.render(f)
        plan.upload_frame(d["albedo"], d["normals"], d["positions"], d["noisy"])
        plan.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        got = plan.download_result()
        want = ref.step(d["albedo"], d["normals"], d["positions"], d["noisy"], sc.prev_camera(f),
                        sc.pixel_offset(f))
        err = np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-2)
        assert err.max() <= 1e-4, f"frame {f} after the timeout: {err.max():.3e}"
    plan.check_device()
    plan.close()


def test_probe_rejects_bad_limits(cuda):
    plan = B.Plan(64, 64)
    for bad in (0, 2_000_000):
        with pytest.raises(B.BmfrError):
            plan.probe_bounded_wait(bad)
    plan.close()
