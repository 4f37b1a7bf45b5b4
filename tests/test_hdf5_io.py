"""HDF5 output (ClassLBM.saveHDF5's datasets, LBM.py:516-567) written by the
C ABI, read back with a reader written from the file-format specification
(no HDF5 package is available here)."""
import numpy as np

import hdf5_min
from uq_b200 import native as N
from uq_b200.solver import write_hdf5_fields


def test_fields_roundtrip(tmp_path):
    rng = np.random.default_rng(5)
    nx, ny = 7, 5
    fields = {k: rng.standard_normal((nx, ny)) for k in ("rho", "ux", "uy", "T")}
    f, h = rng.standard_normal((nx, ny, 13)), rng.standard_normal((nx, ny, 13))
    dx = np.linspace(0.5, 1.5, nx)
    p = tmp_path / "step_10.hdf5"
    write_hdf5_fields(p, fields, t=2.5, gamma=1.4, R=287.0, T_ref=300.0, rho_ref=1.2, dx=dx, dy=0.25, f=f, h=h)
    d = hdf5_min.read(p)
    assert sorted(d) == sorted(["rho", "T", "ux", "uy", "t", "gamma", "R", "T_ref", "rho_ref", "dx", "dy", "Nx",
                                "Ny", "f", "h"])
    for k, v in fields.items():
        assert d[k].shape == (nx, ny) and np.array_equal(d[k], v), k
    assert np.array_equal(d["f"], f) and np.array_equal(d["h"], h)
    assert d["t"] == 2.5 and d["gamma"] == 1.4 and d["R"] == 287.0 and d["T_ref"] == 300.0 and d["rho_ref"] == 1.2
    assert np.array_equal(d["dx"], dx) and d["dy"] == 0.25
    assert d["Nx"] == nx and d["Ny"] == ny and d["Nx"].dtype == np.int64


def test_fields_without_distributions(tmp_path):
    nx, ny = 3, 4
    fields = {k: np.full((nx, ny), v) for k, v in (("rho", 1.0), ("ux", 0.1), ("uy", -0.1), ("T", 2.0))}
    p = tmp_path / "step_0.hdf5"
    write_hdf5_fields(p, fields)
    d = hdf5_min.read(p)
    assert "f" not in d and "h" not in d and len(d) == 13
    assert np.array_equal(d["T"], fields["T"]) and d["dx"] == 1.0


def test_bad_arguments_are_rejected(tmp_path):
    L = N.lib()
    z = np.zeros(4)
    d = z.ctypes.data_as(N._dp)
    assert L.lbm_hdf5_write_fields(str(tmp_path / "x.hdf5").encode(), 0, 2, d, d, d, d, 0.0, 1.4, 1.0, 1.0, 1.0, d,
                                   1, d, 1, None, None) == N.LBM_ERR_INVALID
    assert L.lbm_hdf5_write_fields(str(tmp_path / "no" / "x.hdf5").encode(), 2, 2, d, d, d, d, 0.0, 1.4, 1.0, 1.0,
                                   1.0, d, 1, d, 1, None, None) == N.LBM_ERR_INVALID
