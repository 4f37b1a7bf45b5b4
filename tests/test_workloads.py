"""Host-side case builders and the reference-harness container format."""
import os
import tempfile

import numpy as np

from oracle import refrun
from uq_b200 import workloads as W


def test_builders_are_seeded():
    a = W.couette(nx=16, ny=8, seed=1)
    b = W.couette(nx=16, ny=8, seed=1)
    c = W.couette(nx=16, ny=8, seed=2)
    assert np.array_equal(a["density"], b["density"])
    assert not np.array_equal(a["density"], c["density"])
    assert a["bnd"].shape == (16, 8)
    assert set(a["cellType"][a["bnd"][:, 0]]) == {2} and set(a["cellType"][a["bnd"][:, -1]]) == {2}


def test_riemann_quadrants():
    c = W.riemann(nx=8, ny=6, steps=1)
    rho = c["density"][c["bnd"]]
    assert rho[7, 5] == 1.5 and rho[0, 5] == 0.5323 and rho[0, 0] == 0.138 and rho[7, 0] == 0.5323


def test_ensemble_draws():
    s = W.uq_ensemble(n=64, seed=7)
    assert len(s) == 64
    for d in s:
        assert 0.05 <= d["u_w"] <= 0.2 and 0.02 <= d["tau"] <= 0.1 and 0.6 <= d["Pr"] <= 1.0
        assert d["nx"] in (64, 128, 256, 512)


def test_container_roundtrip_and_flip():
    case = W.random_state(5, 4, seed=0, steps=1)
    vars_ = dict(refrun.case_to_vars(case))
    mat = vars_["bndArray"]
    # loadInput: BNDARRAY(x, y) = ptr[x*Ny + (Ny-1-y)] with ptr column-major (Ny, Nx)
    ptr = mat.reshape(-1, order="F")
    ny = mat.shape[0]
    for x in range(5):
        for y in range(4):
            assert ptr[x * ny + (ny - 1 - y)] == case["bnd"][x, y]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "c.lbmv")
        refrun.write_lbmv(p, list(vars_.items()))
        back = refrun.read_lbmv(p)
        assert np.array_equal(back["bndArray"], mat)
