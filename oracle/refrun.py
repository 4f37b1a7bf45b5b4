"""Run the reference C++ solver (built by ``make -C oracle`` into
``oracle/_ref/simlb_ref``) on a case and read back its state.

Test infrastructure only.  The binary is the unmodified reference
``CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp`` driven by its own ``runSimStep``
(``main.cpp:32-112``); see ``refshim/harness.cpp``.

A *case* is a dict holding the MAT variables that ``cpuLBM::loadInput``
reads (``cpuLBM.cpp:113-265``) plus ``bnd``, the property-id array in the
solver's internal order ``bnd[x, y]`` (``BNDARRAY(x,y)``, ``macros.h:8``).
``loadInput`` flips y when it reads ``bndArray`` (``cpuLBM.cpp:254-266``);
``case_to_vars`` applies the inverse flip so that the solver sees ``bnd``.
"""
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "simlb_ref")

SCALAR_KEYS = (
    "RKMETHOD", "FMETHOD", "CFL", "dtau", "PROCESSOR", "tt_tref", "tt_time", "steps", "tol",
    "periodicX", "periodicY", "mirrorNorth", "mirrorSouth", "mirrorEast", "mirrorWest",
    "gamma", "R", "mu", "Pr", "dx", "dy", "Lx", "Ly", "rho_ref", "p_ref", "T_ref", "Tc_Tref",
    "nPrintOut", "MAT", "numProps",
)
TABLE_KEYS = ("density", "pressure", "temp", "velocityX", "velocityY", "cellType")


def write_lbmv(path, variables):
    """Write ``[(name, ndarray)]`` in the LBMV1 container (first dim fastest)."""
    with open(path, "wb") as fp:
        fp.write(b"LBMV1\0\0\0")
        fp.write(struct.pack("<I", len(variables)))
        for name, arr in variables:
            arr = np.asarray(arr, dtype=np.float64)
            if arr.ndim == 0:
                arr = arr.reshape(1, 1)
            nb = name.encode()
            fp.write(struct.pack("<I", len(nb)))
            fp.write(nb)
            fp.write(struct.pack("<I", arr.ndim))
            fp.write(struct.pack("<%dQ" % arr.ndim, *arr.shape))
            fp.write(np.asfortranarray(arr).tobytes(order="F"))


def read_lbmv(path):
    out = {}
    with open(path, "rb") as fp:
        data = fp.read()
    assert data[:5] == b"LBMV1"
    (n,) = struct.unpack_from("<I", data, 8)
    off = 12
    for _ in range(n):
        (nl,) = struct.unpack_from("<I", data, off)
        off += 4
        name = data[off:off + nl].decode()
        off += nl
        (nd,) = struct.unpack_from("<I", data, off)
        off += 4
        dims = struct.unpack_from("<%dQ" % nd, data, off)
        off += 8 * nd
        cnt = int(np.prod(dims)) if nd else 1
        arr = np.frombuffer(data, dtype=np.float64, count=cnt, offset=off).copy()
        off += 8 * cnt
        out[name] = arr.reshape(dims, order="F") if nd > 1 else arr
    return out


def case_to_vars(case):
    """MAT variables in the order ``loadInput`` reads them."""
    variables = []
    for k in SCALAR_KEYS:
        variables.append((k, np.array([[float(case.get(k, 0))]])))
    for k in TABLE_KEYS:
        variables.append((k, np.asarray(case[k], dtype=np.float64).reshape(1, -1)))
    bnd = np.asarray(case["bnd"])
    nx, ny = bnd.shape
    # loadInput: BNDARRAY(x, y) = ptr[x*Ny + (Ny-1-y)], ptr column-major (Ny, Nx)
    mat = np.empty((ny, nx), dtype=np.float64)
    mat[ny - 1 - np.arange(ny)[:, None], np.arange(nx)[None, :]] = bnd.T
    variables.append(("bndArray", mat))
    return variables


def available():
    return os.path.isfile(REF_BIN) and os.access(REF_BIN, os.X_OK)


def run_reference(case, max_steps=None, workdir=None, timeout=None):
    """Run the reference to its stop condition (or ``max_steps`` steps).

    Returns a dict with ``rho, ux, uy, T, p`` as ``[Nx, Ny]`` arrays,
    ``f, h`` as ``[Nx, Ny, 13]`` (the reference AoS layout), the step count,
    ``dt``, ``stop``, ``residual``, the per-step residual/stop traces and the
    seconds spent in the timed step loop.
    """
    if not available():
        raise RuntimeError("reference oracle binary missing: run `make -C oracle`")
    tmp = None
    if workdir is None:
        tmp = tempfile.TemporaryDirectory(prefix="simlb_ref_")
        workdir = tmp.name
    try:
        inp = os.path.join(workdir, "case.lbmv")
        outp = os.path.join(workdir, "out.lbmv")
        write_lbmv(inp, case_to_vars(case))
        args = [REF_BIN, inp, outp]
        if max_steps is not None:
            args.append(str(int(max_steps)))
        subprocess.run(args, cwd=workdir, check=True, timeout=timeout,
                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
        raw = read_lbmv(outp)
    finally:
        if tmp is not None:
            tmp.cleanup()
    sc = raw["scalars"]
    nx, ny = int(sc[0]), int(sc[1])
    res = {k: raw[k].reshape(nx, ny) for k in ("rho", "ux", "uy", "T", "p")}
    res["f"] = raw["f"].reshape(nx, ny, 13)
    res["h"] = raw["h"].reshape(nx, ny, 13)
    res.update(step=int(sc[2]), nsteps=int(sc[3]), dt=float(sc[4]), stop=int(sc[5]),
               residual=float(sc[6]), seconds=float(sc[7]),
               residual_trace=raw["residual_trace"], stop_trace=raw["stop_trace"],
               e=raw["e"].reshape(2, 13).T.copy())
    return res
