"""Failure detection on the GPU without a GPU fault.

The bounded device-side wait (the mbarrier poll the stencil kernels use
for their TMA copies) is made to run out by waiting on a barrier that
nothing arrives at: the kernel records the timeout bit and returns, the
host reads LBM_ERR_TIMEOUT, and the context stays usable for real work.
"""
import numpy as np
import pytest

from uq_b200 import native as N
from uq_b200 import workloads as W
from uq_b200.solver import Batch

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_device_stays_usable(cuda_device):
    L = N.lib()
    assert L.lbm_selftest_bounded_wait(1) == N.LBM_OK
    assert L.lbm_selftest_bounded_wait(0) == N.LBM_ERR_TIMEOUT
    assert b"ran out" in L.lbm_last_error()
    # the context still runs a real step afterwards
    case = W.couette(nx=32, ny=24, steps=3, seed=2)
    b = Batch([case], precision="f64")
    b.step(3)
    assert int(b.status()[0]) == N.LBM_OK
    assert np.all(np.isfinite(b.macro(0)["rho"]))
    b.close()
    assert L.lbm_selftest_bounded_wait(1) == N.LBM_OK
