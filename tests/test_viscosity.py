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


def test_laws_match_the_reference_generator():
    """The oracle's laws against the expressions the reference's own OpenCL
    generator emits (tests/golden/viscosity_laws.npz, made by running
    genOpenCL of CODE/Python/simLB/codeCL.py for a VHS and a Sutherland
    configuration and evaluating the `double mu = ...;` lines it writes).
    The GPU paths match the oracle for both laws (test_gpu_viscosity.py)."""
    import json
    import os

    from golden_util import GOLDEN

    z = np.load(os.path.join(GOLDEN, "viscosity_laws.npz"))
    laws = json.loads(str(z["laws"]))
    assert {law["model"] for law in laws} == {"VHS", "sutherland"}
    for j, law in enumerate(laws):
        model = 1 if law["model"] == "VHS" else 2
        c = law["constants"]
        mu = O.viscosity(model, c["mu_ref"], c["T_ref"], c.get("upsilon", 0.0), c.get("S_v", 0.0), z["T%d" % j])
        np.testing.assert_allclose(mu, z["mu%d" % j], rtol=1e-15, atol=0, err_msg=law["expression"])
