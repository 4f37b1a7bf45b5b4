"""MAT-file input and output at the boundary (CPU: no GPU needed).

The reader must give the case that loadInput (cpuLBM.cpp:46-281) would
read from a Level-5 MAT file: same variable names, any numeric class as
double, compressed or not, bndArray's y axis flipped.  The writer must
produce createMAT's variables (cpuLBM.cpp:467-745) in a file that other
MAT readers (scipy here) read back.  The reference's own input file (a
Mach-2 boundary layer) is checked when the reference tree is present, and
its 2-step reference solution (a committed fixture) pins the oracle.
"""
import os

import numpy as np
import pytest

from uq_b200 import native as N
from uq_b200 import workloads as W
from uq_b200.solver import mat_case, read_mat_dist, write_mat_fields

from golden_util import GOLDEN, rel_max

sio = pytest.importorskip("scipy.io")

# the reference's own input file, read from the reference tree named by the
# UQ_REFERENCE_ROOT environment variable (the test is skipped without it)
_REF_ROOT = os.environ.get("UQ_REFERENCE_ROOT", "")
REF_INPUT = os.path.join(_REF_ROOT, "Items", "11.04.06-BoundaryLayer-Jacobs", "input.mat") if _REF_ROOT else ""
SCALARS = ("RKMETHOD", "FMETHOD", "CFL", "dtau", "tt_tref", "tt_time", "steps", "tol", "periodicX", "periodicY",
           "mirrorNorth", "mirrorSouth", "mirrorEast", "mirrorWest", "gamma", "R", "mu", "Pr", "dx", "dy", "Lx",
           "Ly", "rho_ref", "p_ref", "T_ref", "Tc_Tref")
TABLES = ("density", "pressure", "temp", "velocityX", "velocityY", "cellType")


def _as_mat_vars(case, integer_classes):
    """MAT variables of a case as loadInput expects them; with
    integer_classes, whole-valued numbers are stored as uint8/uint16 the way
    the reference's own input file stores them."""
    def enc(v):
        a = np.atleast_2d(np.asarray(v, dtype=np.float64))
        if integer_classes and np.all(a == np.round(a)) and a.min() >= 0:
            return a.astype(np.uint8 if a.max() < 256 else np.uint16)
        return a
    out = {k: enc(case[k]) for k in SCALARS}
    out["numProps"] = enc(case["numProps"])
    for k in TABLES:
        out[k] = enc(np.asarray(case[k]).reshape(1, -1))
    bnd = np.asarray(case["bnd"])
    out["bndArray"] = enc(bnd[:, ::-1].T)  # (Ny, Nx) with loadInput's y flip undone
    return out


def _case_equal(a, b):
    for k in SCALARS:
        assert float(a[k]) == float(b[k]), k
    assert int(a["numProps"]) == int(b["numProps"])
    for k in TABLES:
        assert np.array_equal(np.asarray(a[k], dtype=np.float64), np.asarray(b[k], dtype=np.float64)), k
    assert np.array_equal(np.asarray(a["bnd"]), np.asarray(b["bnd"]))


@pytest.mark.parametrize("compressed", [False, True])
@pytest.mark.parametrize("integer_classes", [False, True])
def test_reader_gives_the_case(tmp_path, compressed, integer_classes):
    case = W.couette(nx=23, ny=17, steps=40, seed=5)
    case["tt_time"] = 0.0
    p = tmp_path / "input.mat"
    sio.savemat(str(p), _as_mat_vars(case, integer_classes), do_compression=compressed)
    _case_equal(mat_case(p), case)


def test_writer_is_read_back(tmp_path):
    nx, ny = 9, 7
    rng = np.random.default_rng(3)
    fields = {k: rng.standard_normal((nx, ny)) for k in ("rho", "ux", "uy", "p", "T")}
    f, h = rng.standard_normal((nx, ny, 13)), rng.standard_normal((nx, ny, 13))
    ex, ey = np.arange(13.0), -np.arange(13.0)
    p = tmp_path / "out.mat"
    write_mat_fields(p, fields, t=0.25, dx=0.5, dy=0.125, f=f, h=h, ex=ex, ey=ey)
    m = sio.loadmat(str(p))
    for k in fields:  # {Ny, Nx} over [x*Ny + y]: element (y, x)
        assert m[k].shape == (ny, nx)
        assert np.array_equal(m[k], fields[k].T), k
    for k, v in (("f", f), ("h", h)):  # {13, Ny, Nx} over [(x*Ny + y)*13 + i]
        assert m[k].shape == (13, ny, nx)
        assert np.array_equal(m[k], np.transpose(v, (2, 1, 0))), k
    assert np.array_equal(m["ex"].ravel(), ex) and np.array_equal(m["ey"].ravel(), ey)
    assert (m["t"].item(), m["dx"].item(), m["dy"].item()) == (0.25, 0.5, 0.125)
    # without distributions only the fields and scalars are written
    write_mat_fields(p, fields)
    assert "f" not in sio.loadmat(str(p))


def test_bad_inputs_are_rejected(tmp_path):
    with pytest.raises(N.LbmError) as e:
        mat_case(tmp_path / "missing.mat")
    assert e.value.code == N.LBM_ERR_INVALID
    junk = tmp_path / "junk.mat"
    junk.write_bytes(b"not a mat file" * 20)
    with pytest.raises(N.LbmError) as e:
        mat_case(junk)
    assert e.value.code == N.LBM_ERR_INVALID
    case = W.couette(nx=8, ny=8, steps=1)
    v = _as_mat_vars(case, False)
    del v["bndArray"]
    p = tmp_path / "nobnd.mat"
    sio.savemat(str(p), v)
    with pytest.raises(N.LbmError) as e:
        mat_case(p)
    assert e.value.code == N.LBM_ERR_INVALID and b"bndArray" in N.lib().lbm_last_error()


def test_negative_dimensions_are_rejected(tmp_path):
    """A variable whose stored dimensions are negative is refused, not
    wrapped into a huge (or, multiplied, a small) element count."""
    import struct

    case = W.couette(nx=8, ny=8, steps=1)
    p = tmp_path / "negdims.mat"
    sio.savemat(str(p), _as_mat_vars(case, False), do_compression=False)
    raw = bytearray(p.read_bytes())
    at = raw.index(b"bndArray")  # name data; its 8-byte tag and the 2-int32 dims data come before it
    assert struct.unpack_from("<ii", raw, at - 16) == (8, 8)
    struct.pack_into("<ii", raw, at - 16, -1, -1)
    p.write_bytes(bytes(raw))
    with pytest.raises(N.LbmError) as e:
        mat_case(p)
    assert e.value.code == N.LBM_ERR_INVALID and b"negative" in N.lib().lbm_last_error()


def _fixture_case():
    z = np.load(os.path.join(GOLDEN, "mat_boundary_layer.npz"))
    case = {k[5:]: z[k] for k in z.files if k.startswith("case_")}
    for k in SCALARS + ("numProps",):
        case[k] = float(case[k])
    case["numProps"] = int(case["numProps"])
    case["bnd"] = case["bnd"].astype(np.int64)
    return case, {k[4:]: z[k] for k in z.files if k.startswith("out_")}


@pytest.mark.skipif(not REF_INPUT or not os.path.exists(REF_INPUT),
                    reason="set UQ_REFERENCE_ROOT to the reference tree to read its input.mat")
def test_reference_input_file():
    _case_equal(mat_case(REF_INPUT), _fixture_case()[0])


def test_oracle_on_the_reference_input():
    from oracle.oracle import Oracle

    case, ref = _fixture_case()
    o = Oracle(case)
    o.step(int(ref["step"]))
    m = o.macro()
    for k in ("rho", "ux", "uy", "T"):
        assert rel_max(m[k], ref[k]) <= 1e-11, (k, rel_max(m[k], ref[k]))


def test_checkpoint_distributions_round_trip(tmp_path):
    nx, ny = 11, 6
    rng = np.random.default_rng(4)
    fields = {k: rng.standard_normal((nx, ny)) for k in ("rho", "ux", "uy", "p", "T")}
    f, h = rng.standard_normal((nx, ny, 13)), rng.standard_normal((nx, ny, 13))
    p = tmp_path / "ckpt.mat"
    write_mat_fields(p, fields, t=1.75, f=f, h=h, ex=np.zeros(13), ey=np.zeros(13))
    f2, h2, t = read_mat_dist(p, nx, ny)
    assert np.array_equal(f2, f) and np.array_equal(h2, h) and t == 1.75
    with pytest.raises(N.LbmError) as e:  # wrong shape
        read_mat_dist(p, ny, nx)
    assert e.value.code == N.LBM_ERR_INVALID
    write_mat_fields(p, fields)  # no distributions in the file
    with pytest.raises(N.LbmError):
        read_mat_dist(p, nx, ny)
