"""Generate the golden fixtures in this directory from the reference solver.

Every fixture is produced by the UNMODIFIED reference C++ solver
(CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp) built by ``make -C oracle`` into
``oracle/_ref/simlb_ref``; the reference has no test vectors of its own.
Each fixture records the case builder and its arguments
(``uq_b200.workloads.build``) so tests rebuild the identical input, plus a
checksum of that input to catch builder drift.

    python tests/golden/make_golden.py          # regenerate all fixtures
    python tests/golden/make_golden.py mat      # only the MAT-input fixture

Needs the reference tree (only in the development container); the fixtures
themselves are committed and need nothing at test time.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refrun  # noqa: E402
from uq_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def case_digest(case):
    h = hashlib.sha256()
    for k in sorted(case):
        v = case[k]
        if k in ("mu_model", "upsilon", "S_v") and not np.any(np.asarray(v)):
            continue  # the constant viscosity law: as before these keys existed
        h.update(k.encode())
        h.update(np.ascontiguousarray(np.asarray(v, dtype=np.float64)).tobytes())
    return h.hexdigest()[:16]


def run(builder, kwargs, max_steps=None, keep=("rho", "ux", "uy", "T", "p", "f", "h")):
    case = W.build(builder, **kwargs)
    r = refrun.run_reference(case, max_steps=max_steps)
    out = {k: r[k] for k in keep}
    out.update(step=r["step"], stop=r["stop"], dt=r["dt"], residual=r["residual"],
               residual_trace=r["residual_trace"])
    meta = dict(builder=builder, kwargs=kwargs, max_steps=max_steps, digest=case_digest(case))
    return meta, out


def save(name, entries):
    """entries: list of (meta, arrays) -> one npz with keys c<k>_<field>."""
    arrays = {"meta": np.array(json.dumps([m for m, _ in entries]))}
    for k, (_, arr) in enumerate(entries):
        for field, v in arr.items():
            arrays["c%d_%s" % (k, field)] = np.asarray(v)
    np.savez_compressed(os.path.join(OUT, name), **arrays)
    print(name, len(entries), "cases")


# the reference tree: UQ_REFERENCE_ROOT, else where this container mounts it
REF_ROOT = os.environ.get("UQ_REFERENCE_ROOT", "/root/reference")
MAT_INPUT = os.path.join(REF_ROOT, "Items", "11.04.06-BoundaryLayer-Jacobs", "input.mat")


def mat_input():
    """The reference's own input file (a Mach-2 boundary layer, 1001 x 101,
    R = 287, Tc_Tref = 2.5) read by the library's MAT reader and by scipy
    (they must agree), then 2 steps of the reference binary on it."""
    import scipy.io as sio

    from uq_b200.solver import mat_case

    case = mat_case(MAT_INPUT)
    raw = sio.loadmat(MAT_INPUT)
    for k, v in raw.items():
        if k.startswith("__") or k in ("bndArray",) or k not in case:
            continue
        assert np.allclose(np.ravel(case[k])[: np.size(v)], np.ravel(v).astype(np.float64)), k
    bnd = np.asarray(raw["bndArray"], dtype=np.int64)  # (Ny, Nx), y flipped by loadInput
    assert np.array_equal(case["bnd"], bnd[::-1, :].T)
    # nPrintOut / MAT are driver output switches, not part of the case
    r = refrun.run_reference(dict(case, nPrintOut=1 << 30, MAT=0), max_steps=2)
    arrays = {"case_" + k: np.asarray(v) for k, v in case.items() if k != "bnd"}
    arrays["case_bnd"] = case["bnd"].astype(np.uint8)
    for k in ("rho", "ux", "uy", "T"):
        arrays["out_" + k] = r[k]
    arrays["out_step"] = np.asarray(r["step"])
    arrays["out_dt"] = np.asarray(r["dt"])
    np.savez_compressed(os.path.join(OUT, "mat_boundary_layer.npz"), **arrays)
    print("mat_boundary_layer.npz", case["bnd"].shape, "steps", r["step"])


def main():
    if not refrun.available():
        sys.exit("reference binary missing: make -C oracle")
    if sys.argv[1:] == ["mat"]:
        mat_input()
        return

    # (i) two steps from seeded random states: every BC family x flux x stepper
    entries = []
    for bc in ("transmissive", "periodic", "mirror", "mixed"):
        for fm in (0, 1):
            for rk in (0, 1, 3):
                for sf in (0.0, 0.15):
                    entries.append(run("random_state", dict(nx=8, ny=8, seed=11 + len(entries), bc=bc,
                                                            fmethod=fm, rkmethod=rk, solid_frac=sf, steps=2),
                                       keep=("f", "h", "rho", "T")))
    for bc in ("transmissive", "mirror"):
        for fm in (0, 1):
            entries.append(run("random_state", dict(nx=8, ny=8, seed=11 + len(entries), bc=bc, fmethod=fm,
                                                    rkmethod=2, solid_frac=0.15, steps=1),
                               keep=("f", "h", "rho", "T")))
    save("random_states.npz", entries)

    # (iii) equilibrium known answers: the reference's initial state (0 steps)
    save("equilibrium_init.npz",
         [run("random_state", dict(nx=8, ny=8, seed=5, du=0.4, drho=0.5, dT=0.5, steps=1), max_steps=0,
              keep=("f", "h", "rho", "ux", "uy", "T", "p"))])

    # Couette on 16x16 with wall rows, 50 steps per scheme
    entries = [run("couette", dict(nx=16, ny=16, steps=50, fmethod=fm, rkmethod=rk, seed=3),
                   keep=("rho", "ux", "uy", "T", "f", "h"))
               for fm in (0, 1) for rk in (0, 1, 3)]
    save("couette16.npz", entries)

    # residual normalisation and tolerance stop of the driver (main.cpp:54-110)
    save("driver_residual.npz",
         [run("couette", dict(nx=16, ny=16, steps=60, seed=4, u_w=0.05, overrides=dict(tol=1e-9)),
              keep=("rho", "T")),
          run("couette", dict(nx=16, ny=16, steps=0, seed=4, u_w=0.05, overrides=dict(tol=2e-2)),
              max_steps=200, keep=("rho", "T"))])

    # Riemann problem on a reduced grid, both schemes
    save("riemann32.npz",
         [run("riemann", dict(nx=32, ny=32, steps=100), keep=("rho", "ux", "uy", "T")),
          run("riemann", dict(nx=32, ny=32, steps=60, fmethod=1, rkmethod=1), keep=("rho", "ux", "uy", "T"))])

    # (ii) the full Couette workload: 64x128, WENO5, RK3, 2000 steps
    save("couette_64x128_2000.npz",
         [run("couette", dict(nx=64, ny=128, steps=2000, seed=0), keep=("rho", "ux", "uy", "T"))])

    mat_input()


if __name__ == "__main__":
    main()
