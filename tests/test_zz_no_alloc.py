"""The allocation-free step (lbm_step_noalloc) against the regular handle.

Callers that cannot call cudaMalloc -- applications that own all device
memory through their own pools, or code running where allocating would be
wrong -- use lbm_step_noalloc: it takes the caller's device f and h arrays
and keeps every scratch buffer in a fixed array the library reserves per
GPU.  This file is collected last so that a failure here leaves every other
test already run.
"""
import ctypes as C

import numpy as np
import pytest

from uq_b200 import native as N
from uq_b200 import workloads as W
from uq_b200.solver import Solver, _CaseBuffers

pytestmark = pytest.mark.gpu


def _noalloc(case, d_f, d_h, n_steps):
    bufs = _CaseBuffers(case)
    ctype = np.ascontiguousarray(case["cellType"][case["bnd"]], dtype=np.int32).reshape(-1)
    nx, ny = case["bnd"].shape
    return N.lib().lbm_step_noalloc(C.byref(bufs.cfg), nx, ny, ctype.ctypes.data_as(C.POINTER(C.c_int)),
                                    C.c_void_p(d_f.data_ptr()), C.c_void_p(d_h.data_ptr()), int(n_steps), None)


@pytest.mark.parametrize("builder", ["couette", "mirror_walls"])
def test_noalloc_matches_handle_on_consecutive_calls(cuda_device, builder):
    import torch

    if builder == "couette":
        case = W.couette(nx=48, ny=40, steps=10, seed=7)
    else:
        case = W.random_state(37, 29, seed=3, bc="mirror", solid_frac=0.1, steps=10, du=0.02, drho=0.02, dT=0.02)
    ref = Solver(case, "f64")
    f0, h0 = ref.dist()
    d_f = torch.from_numpy(f0.reshape(-1).copy()).cuda()
    d_h = torch.from_numpy(h0.reshape(-1).copy()).cuda()
    for n in (5, 4):  # two calls in a row: the shared scratch keeps the last call's contents
        code_na = _noalloc(case, d_f, d_h, n)
        code, _ = ref.step(n)
        assert code_na == code == N.LBM_OK, (code_na, code, N.lib().lbm_last_error())
        f, h = ref.dist()
        got_f = d_f.cpu().numpy().reshape(f.shape)
        got_h = d_h.cpu().numpy().reshape(h.shape)
        assert np.max(np.abs(got_f - f)) <= 1e-12 * np.max(np.abs(f))
        assert np.max(np.abs(got_h - h)) <= 1e-12 * np.max(np.abs(h))


def test_noalloc_rejects_domains_beyond_its_scratch(cuda_device):
    import torch

    case = W.couette(nx=200, ny=100, steps=1, seed=1)  # 100 * roundup(200, 32) > 16384
    d = torch.zeros(200 * 100 * 13, dtype=torch.float64, device="cuda")
    assert _noalloc(case, d, d.clone(), 1) == N.LBM_ERR_INVALID
    assert "scratch" in N.lib().lbm_last_error().decode()
