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
    assert b.launches_per_step(False) == 5
    assert b.launches_per_step(True) == 6
