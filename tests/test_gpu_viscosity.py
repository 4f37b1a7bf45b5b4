"""Viscosity laws on the GPU against the oracle (FP64) and within the
mixed-precision tolerance (FP32)."""
import pytest

from oracle import oracle as O
from uq_b200 import workloads as W
from uq_b200.solver import Solver

from golden_util import rel_l2

pytestmark = pytest.mark.gpu

LAWS = [dict(mu_model=1, upsilon=0.25), dict(mu_model=2, S_v=0.4)]


def _cases(law):
    a = W.random_state(24, 20, seed=31, bc="mixed", dT=0.1, solid_frac=0.1, steps=12, du=0.02, drho=0.05)
    b = W.couette(nx=24, ny=20, steps=12, seed=9, T_w=1.2)
    for c in (a, b):
        c.update(law)
    return a, b


@pytest.mark.parametrize("law", LAWS, ids=["vhs", "sutherland"])
def test_fp64_laws_match_oracle(cuda_device, law):
    for case in _cases(law):
        s = Solver(case)
        s.step(12)
        o = O.Oracle(case)
        o.step(12)
        f, h = s.dist()
        fo, ho = o.dist()
        assert rel_l2(f, fo) < 1e-11 and rel_l2(h, ho) < 1e-11, (law, rel_l2(f, fo), rel_l2(h, ho))


@pytest.mark.parametrize("law", LAWS, ids=["vhs", "sutherland"])
def test_fp32_laws_within_tolerance(cuda_device, law):
    for case in _cases(law):
        case["steps"] = 10
        a, b = Solver(case, "f32"), Solver(case, "f64")
        a.step(10)
        b.step(10)
        ma, mb = a.macro(), b.macro()
        for k in ("rho", "T"):
            assert rel_l2(ma[k], mb[k]) <= 1e-5, (law, k, rel_l2(ma[k], mb[k]))
