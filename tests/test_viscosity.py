"""Temperature-dependent viscosity laws (VHS, Sutherland) of the OpenCL
generator (CODE/Python/simLB/codeCL.py:986-990), on the oracle (CPU).

The C++ solver has the constant law only, so the laws are pinned by their
formula and by these properties: VHS with exponent 0 is the constant law
bit for bit, and each law changes a flow whose temperature varies.
"""
import numpy as np

from oracle import oracle as O
from uq_b200 import workloads as W


def _case(**law):
    case = W.random_state(12, 10, seed=21, bc="mixed", dT=0.3, steps=6)
    case.update(law)
    return case


def _run(case, n=6):
    o = O.Oracle(case)
    o.step(n)
    return o.dist()


def test_vhs_with_exponent_zero_is_the_constant_law():
    f0, h0 = _run(_case())
    f1, h1 = _run(_case(mu_model=1, upsilon=-0.5))
    assert np.array_equal(f0, f1) and np.array_equal(h0, h1)


def test_laws_change_a_flow_with_varying_temperature():
    f0, _ = _run(_case())
    for law in (dict(mu_model=1, upsilon=0.25), dict(mu_model=2, S_v=0.4)):
        f1, _ = _run(_case(**law))
        d = np.max(np.abs(f1 - f0)) / np.max(np.abs(f0))
        assert 1e-8 < d < 1e-1, (law, d)
