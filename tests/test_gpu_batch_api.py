"""Batch entry points beyond stepping: restart from macroscopic fields,
per-phase profiling, launch counts."""
import numpy as np
import pytest

from uq_b200 import workloads as W
from uq_b200.solver import Batch

pytestmark = pytest.mark.gpu


def test_set_macro_equals_fresh_initialisation(cuda_device):
    cases = [W.couette(nx=40, ny=30, steps=4, seed=1), W.couette(nx=64, ny=64, steps=4, seed=2)]
    for prec in ("f64", "f32"):
        a = Batch(cases, prec)
        f0, h0 = a.dist(1)
        a.step(3)
        c = cases[1]
        ids = c["bnd"]
        a.set_macro(1, c["density"][ids], c["velocityX"][ids], c["velocityY"][ids], c["temp"][ids])
        f1, h1 = a.dist(1)
        assert np.array_equal(f0, f1) and np.array_equal(h0, h1), prec


def test_profile_and_launch_count(cuda_device):
    b = Batch([W.couette(nx=64, ny=48, steps=4, seed=1)], "f32")
    ms = b.profile(2)
    assert ms.shape == (6,) and (ms[:5] >= 0).all() and ms[2] > 0
    # 2 x 6 tiles of 32 x 8: the four middle rows are simple (the tiles at
    # the periodic x edges read the ghost columns); the top and bottom rows
    # touch the walls.
    # Pointwise, ghost columns of buffer 2, walls, stencil 1 (simple and
    # general kernels), walls, stencil 2 (both), + residual
    assert b.launches_per_step(False) == 8
    assert b.launches_per_step(True) == 9


def test_tile_shape_does_not_change_results(cuda_device):
    cases = [W.couette(nx=70, ny=52, steps=4, seed=1), W.random_state(33, 41, seed=2, bc="mirror", solid_frac=0.1,
                                                                      du=0.02, drho=0.02, dT=0.02, steps=4)]
    ref = Batch(cases, "f32", tile=(32, 8))
    ref.step(4)
    for tile in ((16, 16), (8, 32), (64, 4)):
        b = Batch(cases, "f32", tile=tile)
        b.step(4)
        for k in range(len(cases)):
            assert np.array_equal(b.dist(k)[0], ref.dist(k)[0]), tile


def test_autotune_keeps_state_and_results(cuda_device):
    cases = [W.couette(nx=96, ny=80, steps=6, seed=3), W.couette(nx=64, ny=64, steps=6, seed=4, u_w=0.15)]
    a = Batch(cases, "f32")
    b = Batch(cases, "f32")
    a.step(2)
    b.step(2)
    f_before = b.dist(0)[0]
    chosen, table = b.autotune([(16, 16), (32, 8)], steps=1)
    assert chosen in ((16, 16), (32, 8)) and set(table) == {(16, 16), (32, 8)}
    assert np.array_equal(b.dist(0)[0], f_before)
    a.step(3)
    b.step(3)
    for k in range(2):
        assert np.array_equal(a.dist(k)[0], b.dist(k)[0])


def test_wrap_tiles_match_oracle(cuda_device):
    """Tiles at periodic edges whose halo holds only plain fluid run the
    simple-tile code: across an x edge the staged box reads the sample's
    ghost columns, across a y edge (wrap tiles) the periodic images are
    copied into it.  Periodic in x (Couette) and in both axes (a random
    state), FP64 against the oracle and FP32 within the mixed-path
    tolerance."""
    from oracle import oracle as O

    cases = [W.couette(nx=64, ny=48, steps=6, seed=5),
             W.random_state(64, 48, seed=6, bc="periodic", du=0.01, drho=0.01, dT=0.01, steps=6)]
    b = Batch(cases, "f64")
    # simple, wrap (the random state's tiles at its y edges) and general
    # (Couette's wall rows) runs in each stencil phase, and buffer 2's
    # ghost columns
    assert b.launches_per_step(False) == 10
    b.step(6)
    b32 = Batch(cases, "f32")
    b32.step(6)
    for k, c in enumerate(cases):
        o = O.Oracle(c)
        o.step(6)
        f, h = b.dist(k)
        fo, ho = o.dist()
        assert np.linalg.norm(f - fo) / np.linalg.norm(fo) < 1e-11, k
        assert np.linalg.norm(h - ho) / np.linalg.norm(ho) < 1e-11, k
        m, mo = b32.macro(k), o.macro()
        for q in ("rho", "T"):
            assert np.linalg.norm(m[q] - mo[q]) / np.linalg.norm(mo[q]) < 1e-5, (k, q)


def test_bulk_field_io_equals_per_sample_calls(cuda_device):
    """lbm_batch_set_macro_all / lbm_batch_get_macro_all (every sample's
    fields in one copy per field) give the bits of the per-sample calls."""
    cases = [W.couette(nx=40, ny=30, steps=4, seed=1), W.couette(nx=64, ny=64, steps=4, seed=2),
             W.riemann(nx=48, ny=32, steps=4)]
    for prec in ("f64", "f32"):
        a, b = Batch(cases, prec), Batch(cases, prec)
        a.step(3)
        b.step(3)
        per = [a.macro(k) for k in range(len(cases))]
        bulk = b.macro_all()
        for k in range(len(cases)):
            for q in ("rho", "ux", "uy", "T", "p"):
                assert np.array_equal(per[k][q], bulk[k][q]), (prec, k, q)
        # restart every sample from other fields, in bulk and one by one
        fields = [dict(rho=m["rho"] * 1.001, ux=m["uy"], uy=m["ux"], T=m["T"]) for m in per]
        for k, f in enumerate(fields):
            a.set_macro(k, f["rho"], f["ux"], f["uy"], f["T"])
        b.set_macro_all(fields)
        a.step(2)
        b.step(2)
        for k in range(len(cases)):
            fa, ha = a.dist(k)
            fb, hb = b.dist(k)
            assert np.array_equal(fa, fb) and np.array_equal(ha, hb), (prec, k)
