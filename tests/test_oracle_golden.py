"""Pin the FP64 C restatement (oracle/lbm_oracle.c) against the golden
vectors that the unmodified reference solver produced."""
import numpy as np
import pytest

from golden_util import load, rel_l2, rel_max
from oracle import oracle as O


def _run(case, meta):
    o = O.Oracle(case)
    ms = meta.get("max_steps")
    stop, trace = o.run(-1 if ms is None else ms)
    return o, stop, trace


def test_random_states_two_steps():
    worst = 0.0
    for case, meta, g in load("random_states.npz"):
        o, stop, _ = _run(case, meta)
        f, h = o.dist()
        assert o.step_count == int(g["step"])
        e = max(rel_max(f, g["f"]), rel_max(h, g["h"]))
        worst = max(worst, e)
        assert e < 1e-12, (meta, e)
    assert worst > 0 or worst == 0


def test_equilibrium_known_answers():
    [(case, meta, g)] = load("equilibrium_init.npz")
    o = O.Oracle(case)
    f, h = o.dist()
    assert rel_max(f, g["f"]) < 1e-14
    assert rel_max(h, g["h"]) < 1e-14
    m = o.macro()
    for k in ("rho", "ux", "uy", "T", "p"):
        assert rel_max(m[k], g[k]) < 1e-13, k
    # sum_i f_eq = rho and sum_i h_eq = rho (|u|^2 + b R T) / 2 (cpuLBM.cpp:825-843)
    b = 2.0 / (case["gamma"] - 1.0)
    rho = case["density"][case["bnd"]]
    T = case["temp"][case["bnd"]]
    ux = case["velocityX"][case["bnd"]]
    uy = case["velocityY"][case["bnd"]]
    np.testing.assert_allclose(f.sum(-1), rho, rtol=1e-13)
    np.testing.assert_allclose(h.sum(-1), rho * (ux ** 2 + uy ** 2 + b * case["R"] * T) / 2, rtol=1e-13)


def test_equilibrium_direct_identities():
    rng = np.random.default_rng(3)
    for _ in range(50):
        rho, ux, uy, T = rng.uniform(0.2, 3), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.3, 2)
        R, Tc, K = rng.uniform(0.5, 300), rng.uniform(0.5, 3), rng.uniform(1, 5)
        f, h = O.equilibrium(rho, ux, uy, T, R, Tc, K)
        assert abs(f.sum() - rho) < 1e-12 * max(1, rho)
        assert abs(h.sum() - rho * (ux * ux + uy * uy + (K + 2) * R * T) / 2) < 1e-11 * max(1.0, abs(h).max())


def test_couette16_fifty_steps():
    # Over 50 steps rounding differences (the oracle evaluates the same
    # polynomials and WENO weights in its own operation order) are amplified
    # where NND's minmod or WENO's weights switch; the headline scheme
    # (WENO5 + RK3) stays within 1e-10.
    for case, meta, g in load("couette16.npz"):
        o, stop, _ = _run(case, meta)
        m = o.macro()
        f, h = o.dist()
        assert o.step_count == 50
        kw = meta["kwargs"]
        tol = 1e-10 if (kw["fmethod"], kw["rkmethod"]) == (1, 1) else 1e-6
        for k in ("rho", "T"):
            assert rel_l2(m[k], g[k]) < tol, (kw, k)
        assert rel_l2(np.hypot(m["ux"], m["uy"]), np.hypot(g["ux"], g["uy"])) < 100 * tol
        assert rel_l2(f, g["f"]) < tol and rel_l2(h, g["h"]) < tol


def test_driver_residual_and_stop():
    for case, meta, g in load("driver_residual.npz"):
        o, stop, trace = _run(case, meta)
        assert o.step_count == int(g["step"]), meta
        assert stop == int(g["stop"]) or (meta["max_steps"] is not None and stop == 0)
        # The residual is the RMS of one step's change of T, a small
        # difference of large numbers: rounding differences grow in it roughly
        # tenfold every dozen steps on this coarse grid, so the trace is
        # compared over its first 60 steps (normalisation included, steps 2-21).
        ref = g["residual_trace"][:60]
        np.testing.assert_allclose(trace[:len(ref)], ref, rtol=1e-5, atol=1e-14)


def test_riemann32():
    for case, meta, g in load("riemann32.npz"):
        o, stop, _ = _run(case, meta)
        m = o.macro()
        for k in ("rho", "T"):
            assert rel_l2(m[k], g[k]) < 1e-11, (meta["kwargs"], k)


@pytest.mark.slow
def test_couette_full_2000_steps():
    """The full Couette workload (64x128, WENO5, RK3, 2000 steps).

    This configuration amplifies rounding differences about 1e5-fold per 50
    steps (WENO5 with the two-flux IMEX update is weakly unstable here; the
    growth saturates at density fluctuations of ~1e-3), so two correct FP64
    implementations that differ only in operation order decorrelate at the
    fluctuation scale after ~200 steps.  After 2000 steps the comparison is
    therefore on what the dynamics cannot scramble: exact mass conservation,
    the total energy and the mean temperature, and the step/stop semantics.
    """
    [(case, meta, g)] = load("couette_64x128_2000.npz")
    o, stop, _ = _run(case, meta)
    m = o.macro()
    assert o.step_count == 2000 and stop == 2 == int(g["stop"])

    def agg(mm):
        rho, ux, uy, T = (mm[k][:, 1:-1] for k in ("rho", "ux", "uy", "T"))
        return rho.sum(), (rho * (ux ** 2 + uy ** 2 + 5.0 * T) / 2).sum(), T.mean()

    mass, energy, Tm = agg(m)
    gmass, genergy, gTm = agg(g)
    assert abs(mass - gmass) / gmass < 1e-11
    assert abs(energy - genergy) / genergy < 1e-3
    assert abs(Tm - gTm) / gTm < 1e-3


def _chaos():
    import json
    import os

    from golden_util import GOLDEN, case_digest
    from uq_b200 import workloads as W

    z = np.load(os.path.join(GOLDEN, "couette_chaos.npz"))
    case = W.build("couette", **json.loads(str(z["kwargs"])))
    assert case_digest(case) == str(z["digest"])
    return case, [int(s) for s in z["steps"]], z


def _l2_errors(m, r):
    du = np.sqrt((m["ux"] - r["ux"]) ** 2 + (m["uy"] - r["uy"]) ** 2)
    return np.array([rel_l2(m["rho"], r["rho"]), float(np.linalg.norm(du) / np.linalg.norm(np.hypot(r["ux"], r["uy"]))),
                     rel_l2(m["T"], r["T"])])


def test_reference_rounding_spread_grows_then_saturates():
    """The fixture's own record: a 1-ulp input change grows by orders of
    magnitude over 50 steps and saturates near the fluctuation scale."""
    _, steps, z = _chaos()
    for key in ("err_one_node", "err_all_nodes", "err_all_nodes_f32ulp"):
        e = z[key]
        assert e.shape == (len(steps), 3)
        assert np.all(e[2] > 1e3 * e[0]) or key == "err_all_nodes_f32ulp"
        assert np.all(e[-1] > 1e-4) and np.all(e[-1] < 1.0)


@pytest.mark.parametrize("upto", [200, pytest.param(2000, marks=pytest.mark.slow)])
def test_oracle_within_the_references_rounding_spread(upto):
    """A second FP64 implementation (the C restatement, its own operation
    order) stays within 10x the reference's 1-ulp spread at every checkpoint
    (measured: within 1.5x)."""
    case, steps, z = _chaos()
    o = O.Oracle(case)
    done = 0
    for j, n in enumerate(steps):
        if n > upto:
            break
        o.step(n - done)
        done = n
        if n < 2000:
            ref = {k: z["ref%d_%s" % (n, k)] for k in ("rho", "ux", "uy", "T")}
        else:
            [(_, _, ref)] = load("couette_64x128_2000.npz")
        e = _l2_errors(o.macro(), ref)
        spread = np.maximum(z["err_one_node"][j], z["err_all_nodes"][j])
        assert np.all(e <= 10.0 * spread), (n, e, spread)


@pytest.mark.slow
def test_oracle_riemann256_500_steps():
    import json
    import os

    from golden_util import GOLDEN, case_digest
    from uq_b200 import workloads as W

    z = np.load(os.path.join(GOLDEN, "riemann256_500.npz"))
    case = W.build("riemann", **json.loads(str(z["kwargs"])))
    assert case_digest(case) == str(z["digest"])
    o = O.Oracle(case)
    o.step(int(z["step"]))
    m = o.macro()
    for k in ("rho", "T"):
        assert rel_l2(m[k], z[k]) < 1e-8, (k, rel_l2(m[k], z[k]))
