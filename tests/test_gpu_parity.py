"""CUDA path (through the C ABI) against the reference golden vectors and
the FP64 oracle.  Short horizons are compared pointwise; the Couette
configuration amplifies rounding differences ~1e5-fold per 50 steps, so
long runs are compared on invariants (see test_oracle_golden.py)."""
import numpy as np
import pytest

from golden_util import load, rel_l2, rel_max
from oracle import oracle as O
from uq_b200 import native
from uq_b200 import workloads as W
from uq_b200.solver import Batch, Solver

pytestmark = pytest.mark.gpu


def _gpu_run(case, meta, precision="f64"):
    s = Solver(case, precision)
    ms = meta.get("max_steps")
    stop, trace = s.run(-1 if ms is None else ms)
    return s, stop, trace


def test_fp64_random_states_match_reference(cuda_device):
    worst = 0.0
    for case, meta, g in load("random_states.npz"):
        s, stop, _ = _gpu_run(case, meta)
        f, h = s.dist()
        assert s.step_count == int(g["step"])
        e = max(rel_max(f, g["f"]), rel_max(h, g["h"]))
        worst = max(worst, e)
        assert e < 1e-11, (meta["kwargs"], e)
    print("worst rel max error over random-state cases: %.2e" % worst)


def test_fp64_initial_equilibria_match_reference(cuda_device):
    [(case, meta, g)] = load("equilibrium_init.npz")
    s = Solver(case)
    f, h = s.dist()
    assert rel_max(f, g["f"]) < 1e-14 and rel_max(h, g["h"]) < 1e-14
    m = s.macro()
    for k in ("rho", "ux", "uy", "T", "p"):
        assert rel_max(m[k], g[k]) < 1e-13, k


def test_fp64_short_horizon_matches_oracle(cuda_device):
    for fm in (0, 1):
        for rk in (0, 1, 2, 3):
            case = W.couette(nx=24, ny=20, steps=12, fmethod=fm, rkmethod=rk, seed=9)
            s = Solver(case)
            code, _ = s.step(12)
            o = O.Oracle(case)
            failed, _ = o.step(12)
            if rk == 2:  # explicit EULER diverges here: the failing step
                continue  # itself depends on rounding
            assert (code == native.LBM_ERR_EQUILIBRIUM) == bool(failed)
            f, h = s.dist()
            fo, ho = o.dist()
            assert rel_l2(f, fo) < 1e-11 and rel_l2(h, ho) < 1e-11, (fm, rk, rel_l2(f, fo))


def test_fp64_couette16_matches_reference(cuda_device):
    for case, meta, g in load("couette16.npz"):
        s, stop, _ = _gpu_run(case, meta)
        m = s.macro()
        kw = meta["kwargs"]
        tol = 1e-9 if (kw["fmethod"], kw["rkmethod"]) == (1, 1) else 1e-5
        for k in ("rho", "T"):
            assert rel_l2(m[k], g[k]) < tol, (kw, k, rel_l2(m[k], g[k]))


def test_fp64_driver_matches_reference(cuda_device):
    for case, meta, g in load("driver_residual.npz"):
        s, stop, trace = _gpu_run(case, meta)
        assert s.step_count == int(g["step"])
        assert stop == int(g["stop"]) or (meta["max_steps"] is not None and stop == 0)
        ref = g["residual_trace"][:60]
        np.testing.assert_allclose(trace[:len(ref)], ref, rtol=1e-5, atol=1e-14)


def test_fp64_riemann_matches_reference(cuda_device):
    for case, meta, g in load("riemann32.npz"):
        s, stop, _ = _gpu_run(case, meta)
        m = s.macro()
        for k in ("rho", "T"):
            assert rel_l2(m[k], g[k]) < 1e-8, (meta["kwargs"], k, rel_l2(m[k], g[k]))


def test_fp64_full_couette_invariants(cuda_device):
    [(case, meta, g)] = load("couette_64x128_2000.npz")
    s, stop, _ = _gpu_run(case, meta)
    assert s.step_count == 2000 and stop == 2
    m = s.macro()

    def agg(mm):
        rho, ux, uy, T = (mm[k][:, 1:-1] for k in ("rho", "ux", "uy", "T"))
        return rho.sum(), (rho * (ux ** 2 + uy ** 2 + 5.0 * T) / 2).sum(), T.mean()

    mass, energy, Tm = agg(m)
    gmass, genergy, gTm = agg(g)
    assert abs(mass - gmass) / gmass < 1e-11
    assert abs(energy - genergy) / genergy < 1e-3
    assert abs(Tm - gTm) / gTm < 1e-3


def test_fp32_short_horizon_within_tolerance(cuda_device):
    """Mixed path vs the FP64 oracle over 10 steps, a horizon where the
    configuration's rounding amplification (~1e5 per 50 steps) leaves the
    FP32 perturbation below the tolerance: L2(rho, u, T) <= 1e-5."""
    case = W.couette(nx=64, ny=64, steps=10, u_w=0.15, tau=0.03, Pr=0.8, seed=2)
    s = Solver(case, "f32")
    s.step(10)
    o = O.Oracle(case)
    o.step(10)
    m, mo = s.macro(), o.macro()
    assert rel_l2(m["rho"], mo["rho"]) < 1e-5
    assert rel_l2(m["T"], mo["T"]) < 1e-5
    assert rel_l2(np.stack([m["ux"], m["uy"]]), np.stack([mo["ux"], mo["uy"]])) < 1e-5


def test_nonuniform_grid_matches_oracle(cuda_device):
    case = W.flat_plate(nx=40, ny=24, steps=5, tau=2e-3)
    s = Solver(case)
    s.step(5)
    o = O.Oracle(case)
    o.step(5)
    assert abs(s.dt - o.dt) < 1e-15
    f, h = s.dist()
    fo, ho = o.dist()
    assert rel_l2(f, fo) < 1e-11 and rel_l2(h, ho) < 1e-11


def test_batch_equals_alone(cuda_device):
    """A sample advanced inside a batch of uneven grids and mixed methods is
    bit-identical to the same sample advanced alone."""
    cases = [W.couette(nx=40, ny=24, steps=5, seed=1),
             W.couette(nx=64, ny=33, steps=5, seed=2, rkmethod=0, fmethod=0),
             W.random_state(17, 29, seed=3, bc="mirror", solid_frac=0.1, steps=5),
             W.riemann(nx=48, ny=48, steps=5)]
    for prec in ("f64", "f32"):
        b = Batch(cases, precision=prec)
        b.step(5)
        assert list(b.status()) == [0] * len(cases)
        for k, c in enumerate(cases):
            s = Solver(c, prec)
            s.step(5)
            fb, hb = b.dist(k)
            fs, hs = s.dist()
            assert np.array_equal(fb, fs) and np.array_equal(hb, hs), (prec, k)


def test_checkpoint_roundtrip(cuda_device):
    case = W.couette(nx=32, ny=24, steps=10, seed=5)
    a = Solver(case)
    a.step(4)
    f, h = a.dist()
    b = Solver(case)
    b.set_dist(f, h)
    a.step(6)
    b.step(6)
    fa, ha = a.dist()
    fb, hb = b.dist()
    assert np.array_equal(fa, fb) and np.array_equal(ha, hb)


def test_status_reports_nonfinite_and_equilibrium(cuda_device):
    case = W.couette(nx=16, ny=16, steps=3, seed=1)
    for prec in ("f64", "f32"):
        s = Solver(case, prec)
        f, h = s.dist()
        f2 = f.copy()
        f2[5, 7, 3] = np.nan  # host-side corruption of one value
        s.set_dist(f2, h)
        code, _ = s.step(1)
        assert code == native.LBM_ERR_NONFINITE, prec
    # in a batch only the corrupted sample is flagged (FP32 finiteness sums)
    b = Batch([case, W.couette(nx=40, ny=24, steps=3, seed=2)], "f32")
    f, h = b.dist(0)
    f2 = f.copy()
    f2[5, 7, 3] = np.nan
    b.set_dist(0, f2, h)
    b.step(1)
    assert list(b.status()) == [native.LBM_ERR_NONFINITE, native.LBM_OK]
    # an enormous velocity breaks the equilibrium mass check, as in the reference
    big = W.random_state(8, 8, seed=1, du=0.0, steps=2)
    big["velocityX"][:] = 3e4
    s2 = Solver(big)
    code, _ = s2.step(1)
    o = O.Oracle(big)
    failed, _ = o.step(1)
    assert failed == 1 and code == native.LBM_ERR_EQUILIBRIUM


def test_periodic_edges_and_solids_across_tile_shapes(cuda_device):
    """Tiles on a periodic edge take the periodic images into their staged
    box, and boundary-aware stencils near solids and closed edges read the
    box: domains that mix simple and such tiles give the same bits in FP32
    for every tile shape, and match the FP64 oracle."""
    kw = dict(solid_frac=0.05, steps=4, du=0.02, drho=0.02, dT=0.02)
    cases = [W.random_state(70, 52, seed=7, bc="periodic", **kw),
             W.random_state(45, 38, seed=8, bc="mixed", **kw),
             W.random_state(50, 41, seed=9, bc="transmissive", **kw)]
    ref = Batch(cases, "f32", tile=(32, 8))
    ref.step(4)
    assert list(ref.status()) == [0] * len(cases)
    for tile in ((16, 16), (8, 32), (64, 4)):
        b = Batch(cases, "f32", tile=tile)
        b.step(4)
        for k in range(len(cases)):
            f, h = b.dist(k)
            fr, hr = ref.dist(k)
            assert np.array_equal(f, fr) and np.array_equal(h, hr), (tile, k)
    for c in cases:
        s = Solver(c, "f64")
        s.step(4)
        o = O.Oracle(c)
        o.step(4)
        f, h = s.dist()
        fo, ho = o.dist()
        assert rel_l2(f, fo) < 1e-11 and rel_l2(h, ho) < 1e-11, c.get("periodicX")
