"""The allocation-free step (lbm_step_noalloc) against the regular handle.

Some callers cannot call cudaMalloc: applications that keep every byte of
device memory in their own pools or arenas, or whose device-memory budget is
already spoken for, so that an allocation made by a library they call would
fail or break their accounting.  lbm_step_noalloc takes the caller's device
f and h arrays and keeps every scratch buffer in a fixed array the library
reserves per GPU.  Each check compares it with a regular handle (lbm_create,
which allocates) on the same case, over two calls in a row, because the
shared scratch keeps the last call's contents.  This file is collected last
so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from uq_b200 import native as N
from uq_b200 import workloads as W
from uq_b200.solver import Solver, _CaseBuffers

pytestmark = pytest.mark.gpu


def _noalloc(case, d_f, d_h, n_steps, stream=None):
    bufs = _CaseBuffers(case)
    ctype = np.ascontiguousarray(case["cellType"][case["bnd"]], dtype=np.int32).reshape(-1)
    nx, ny = case["bnd"].shape
    return N.lib().lbm_step_noalloc(C.byref(bufs.cfg), nx, ny, ctype.ctypes.data_as(C.POINTER(C.c_int)),
                                    C.c_void_p(d_f.data_ptr()), C.c_void_p(d_h.data_ptr()), int(n_steps),
                                    None if stream is None else C.c_void_p(stream))


def _check_against_handle(case, calls=(5, 4), stream=None):
    import torch

    ref = Solver(case, "f64")
    f0, h0 = ref.dist()
    d_f = torch.from_numpy(f0.reshape(-1).copy()).cuda()
    d_h = torch.from_numpy(h0.reshape(-1).copy()).cuda()
    for n in calls:
        code_na = _noalloc(case, d_f, d_h, n, stream)
        code, _ = ref.step(n)
        assert code_na == code == N.LBM_OK, (code_na, code, N.lib().lbm_last_error())
        f, h = ref.dist()
        got_f = d_f.cpu().numpy().reshape(f.shape)
        got_h = d_h.cpu().numpy().reshape(h.shape)
        assert np.max(np.abs(got_f - f)) <= 1e-12 * np.max(np.abs(f))
        assert np.max(np.abs(got_h - h)) <= 1e-12 * np.max(np.abs(h))
    ref.close()


@pytest.mark.parametrize("builder", ["couette", "mirror_walls"])
def test_noalloc_matches_handle_on_consecutive_calls(cuda_device, builder):
    if builder == "couette":
        case = W.couette(nx=48, ny=40, steps=10, seed=7)
    else:
        case = W.random_state(37, 29, seed=3, bc="mirror", solid_frac=0.1, steps=10, du=0.02, drho=0.02, dT=0.02)
    _check_against_handle(case)


@pytest.mark.parametrize("rk", [0, 1, 2, 3])
@pytest.mark.parametrize("fm", [0, 1])
def test_noalloc_every_stepper_and_flux_scheme(cuda_device, rk, fm):
    """RKMETHOD 0 (RK1), 1 (RK3), 2 (EULER), 3 (EULER_EQ) with NND and WENO5:
    the two-phase and three-phase steps and both reconstructions."""
    case = W.random_state(33, 21, seed=11 + rk + 4 * fm, bc="mixed", fmethod=fm, rkmethod=rk, solid_frac=0.08,
                          steps=10, du=0.02, drho=0.02, dT=0.02)
    _check_against_handle(case, calls=(3, 2))


def test_noalloc_on_a_caller_stream(cuda_device):
    import torch

    s = torch.cuda.Stream()
    case = W.couette(nx=40, ny=24, steps=10, seed=5, fmethod=0)
    _check_against_handle(case, stream=s.cuda_stream)


def test_noalloc_small_then_larger_domain(cuda_device):
    """A larger domain right after a smaller one: the tile list, node flags
    and tensor maps in the shared scratch are rebuilt for each call."""
    _check_against_handle(W.couette(nx=20, ny=12, steps=10, seed=8), calls=(3,))
    _check_against_handle(W.couette(nx=120, ny=100, steps=10, seed=9), calls=(3,))
    _check_against_handle(W.couette(nx=20, ny=12, steps=10, seed=10), calls=(2,))


def test_noalloc_rejects_domains_beyond_its_scratch(cuda_device):
    import torch

    case = W.couette(nx=200, ny=100, steps=1, seed=1)  # 100 * roundup(200, 32) > 16384
    d = torch.zeros(200 * 100 * 13, dtype=torch.float64, device="cuda")
    assert _noalloc(case, d, d.clone(), 1) == N.LBM_ERR_INVALID
    assert "scratch" in N.lib().lbm_last_error().decode()
