"""The C-ABI library loads and exports every symbol include/uq_lbm.h
declares; without a GPU, creating a handle fails loudly (no CPU path)."""
import ctypes
import os
import re

import numpy as np

from uq_b200 import native, workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            src = open(os.path.join(inc, fn)).read()
            names |= set(re.findall(r"^LBM_API[^(]*?\b(lbm_\w+)\s*\(", src, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(native.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers the same set
    assert names <= set(native.SIGNATURES), names - set(native.SIGNATURES)


def test_create_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        return
    from uq_b200.solver import Solver

    case = W.couette(nx=8, ny=8, steps=1)
    try:
        Solver(case)
    except native.LbmError as e:
        assert e.code == native.LBM_ERR_CUDA
        assert "CUDA" in str(e) or "device" in str(e)
    else:
        raise AssertionError("lbm_create succeeded without a CUDA device")


def test_invalid_config_is_rejected():
    import torch

    if torch.cuda.is_available():
        return
    L = native.lib()
    cfg = native.LbmConfig()
    ini = native.LbmInit()
    h = ctypes.c_void_p()
    assert L.lbm_create(ctypes.byref(cfg), ctypes.byref(ini), 0, ctypes.byref(h)) == native.LBM_ERR_INVALID
    assert not h.value


def test_server_and_selftest_without_gpu_fail_loudly():
    import torch

    if torch.cuda.is_available():
        return
    from uq_b200.solver import Server

    try:
        Server(precision="f32")
    except native.LbmError as e:
        assert e.code == native.LBM_ERR_CUDA
    else:
        raise AssertionError("lbm_server_create succeeded without a CUDA device")
    assert native.lib().lbm_selftest_bounded_wait(0) == native.LBM_ERR_CUDA


def test_oversized_sample_is_rejected_before_reading_arrays():
    """Ny * roundup(Nx, 32) above 2^26 nodes is refused (32-bit plane
    offsets in the kernels); the check comes before any per-node array is
    read, so the small arrays of this case are never indexed."""
    from uq_b200.solver import _CaseBuffers

    bufs = _CaseBuffers(W.couette(nx=8, ny=8, steps=1))
    bufs.ini.Nx, bufs.ini.Ny = 1 << 25, 3
    h = ctypes.c_void_p()
    L = native.lib()
    assert L.lbm_create(ctypes.byref(bufs.cfg), ctypes.byref(bufs.ini), 1, ctypes.byref(h)) == native.LBM_ERR_INVALID
    assert b"too large" in L.lbm_last_error()
    assert not h.value


def test_noalloc_rejects_bad_cell_types_before_device_work():
    """lbm_step_noalloc checks the host cellType array first (0 fluid,
    1 permanent, 2 solid), so no GPU is needed to see the refusal."""
    L = native.lib()
    case = W.couette(nx=8, ny=8, steps=1)
    from uq_b200.solver import _CaseBuffers

    bufs = _CaseBuffers(case)
    ctype = np.zeros(8 * 8, dtype=np.int32)
    ctype[9] = 3
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the check comes first
    code = L.lbm_step_noalloc(ctypes.byref(bufs.cfg), 8, 8, ctype.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              fake, fake, 1, None)
    assert code == native.LBM_ERR_INVALID
    assert b"cellType" in L.lbm_last_error()
