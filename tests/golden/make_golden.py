"""Generate the golden fixtures in this directory from the reference solver.

Every fixture is produced by the UNMODIFIED reference C++ solver
(CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp) built by ``make -C oracle`` into
``oracle/_ref/simlb_ref``; the reference has no test vectors of its own.
Each fixture records the case builder and its arguments
(``uq_b200.workloads.build``) so tests rebuild the identical input, plus a
checksum of that input to catch builder drift.

    python tests/golden/make_golden.py          # regenerate all fixtures
    python tests/golden/make_golden.py mat      # only the MAT-input fixture
    python tests/golden/make_golden.py chaos    # only the 1-ulp perturbation fixture
    python tests/golden/make_golden.py riemann  # only the Riemann 256^2 fixture
    python tests/golden/make_golden.py ensemble # only the ensemble's 64^2 status fixture
    python tests/golden/make_golden.py spread   # only the single-precision spread fixture
    python tests/golden/make_golden.py viscosity  # the viscosity laws from the reference's OpenCL generator

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


CHAOS_STEPS = (10, 50, 200, 2000)


def _ref_fields(args):
    """One reference run (a picklable task for the process pool)."""
    case, steps = args
    r = refrun.run_reference(case, max_steps=steps)
    return {k: r[k] for k in ("rho", "ux", "uy", "T")}


def _l2_errors(a, b):
    """Relative L2 of rho, the u vector and T over all nodes: a against b."""
    d_u = np.sqrt((a["ux"] - b["ux"]) ** 2 + (a["uy"] - b["uy"]) ** 2)
    return [float(np.linalg.norm(a["rho"] - b["rho"]) / np.linalg.norm(b["rho"])),
            float(np.linalg.norm(d_u) / np.linalg.norm(np.hypot(b["ux"], b["uy"]))),
            float(np.linalg.norm(a["T"] - b["T"]) / np.linalg.norm(b["T"]))]


def chaos():
    """How far two FP64 runs of the Couette workload (64 x 128, WENO5, RK3)
    drift apart when their inputs differ by one unit in the last place.

    The reference runs the workload four times: as built, with one interior
    node's density raised by 1 ulp, with every interior node's density
    moved by 1 ulp up or down (seeded signs), and with every interior
    density moved by one single-precision ulp (relative 2^-24, the same
    signs).  The fixture keeps the
    unperturbed fields at 10, 50 and 200 steps (2000 steps are in
    couette_64x128_2000.npz) and the relative L2 distance of rho, u, T of
    each perturbed run from it at 10, 50, 200 and 2000 steps: the spread
    that rounding alone produces, against which other FP64 and FP32
    implementations are judged."""
    import concurrent.futures as cf
    import multiprocessing as mp

    kw = dict(nx=64, ny=128, steps=2000, seed=0)
    base = W.build("couette", **kw)
    one = W.build("couette", **kw)
    k_one = 2 + 64 * 63 + 17  # an interior node's property id: x = 32, y = 18 (ids 2 + x*(Ny-2) + y-1)
    one["density"] = one["density"].copy()
    one["density"][k_one] = np.nextafter(one["density"][k_one], np.inf)
    allp = W.build("couette", **kw)
    rng = np.random.default_rng(77)
    d = allp["density"].copy()
    sgn = rng.choice([-np.inf, np.inf], size=d.size - 2)
    d[2:] = np.nextafter(d[2:], sgn)
    allp["density"] = d
    # every interior density moved by one FP32 ulp (relative 2^-24, seeded
    # signs): the size of a rounding to single precision
    f32p = W.build("couette", **kw)
    d = f32p["density"].copy()
    d[2:] = d[2:] * (1.0 + np.sign(sgn) * 2.0 ** -24)
    f32p["density"] = d
    variants = [base, one, allp, f32p]
    tasks = [(c, s) for c in variants for s in CHAOS_STEPS]
    with cf.ProcessPoolExecutor(max_workers=min(len(tasks), os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_ref_fields, tasks))
    n = len(CHAOS_STEPS)
    ref = res[:n]
    arrays = {"steps": np.array(CHAOS_STEPS), "digest": np.array(case_digest(base)),
              "kwargs": np.array(json.dumps(kw)), "one_node_id": np.array(k_one),
              "perturb_seed": np.array(77)}
    arrays["err_one_node"] = np.array([_l2_errors(res[n + j], ref[j]) for j in range(n)])
    arrays["err_all_nodes"] = np.array([_l2_errors(res[2 * n + j], ref[j]) for j in range(n)])
    arrays["err_all_nodes_f32ulp"] = np.array([_l2_errors(res[3 * n + j], ref[j]) for j in range(n)])
    for j, s in enumerate(CHAOS_STEPS[:-1]):
        for k in ("rho", "ux", "uy", "T"):
            arrays["ref%d_%s" % (s, k)] = ref[j][k]
    g = np.load(os.path.join(OUT, "couette_64x128_2000.npz"))
    for k in ("rho", "ux", "uy", "T"):
        assert np.array_equal(g["c0_" + k], ref[-1][k]), k  # the committed 2000-step run, bit for bit
    np.savez_compressed(os.path.join(OUT, "couette_chaos.npz"), **arrays)
    print("couette_chaos.npz: L2 (rho, u, T) one node", arrays["err_one_node"].tolist())
    print("couette_chaos.npz: L2 (rho, u, T) all nodes", arrays["err_all_nodes"].tolist())
    print("couette_chaos.npz: L2 (rho, u, T) all nodes, FP32 ulp", arrays["err_all_nodes_f32ulp"].tolist())


def riemann_floor():
    """The Riemann workload on a reduced 256 x 256 grid (Lax-Liu 3, NND,
    RK1, tau 1e-3, CFL 0.2, 500 steps): the reference's FP64 fields after
    500 steps, against which the GPU's FP64 and FP32 paths are measured."""
    kw = dict(nx=256, ny=256, steps=500)
    case = W.build("riemann", **kw)
    r = refrun.run_reference(case, max_steps=500)
    arrays = {"digest": np.array(case_digest(case)), "kwargs": np.array(json.dumps(kw)),
              "step": np.array(r["step"])}
    for k in ("rho", "ux", "uy", "T"):
        arrays[k] = r[k]
    np.savez_compressed(os.path.join(OUT, "riemann256_500.npz"), **arrays)
    print("riemann256_500.npz steps", r["step"])


def _ref_status(args):
    """Reference run of one ensemble sample to `steps` steps: (stop flag,
    steps done, all fields finite); perturbed: every interior density moved
    by 1 ulp (seeded signs) first.  A run that the reference binary does not
    survive (it dies of a signal on some diverging states) is recorded as
    stop -1, step -1."""
    sample, steps, perturbed = args
    case = W.ensemble_case(sample)
    if perturbed:
        rng = np.random.default_rng(77)
        d = case["density"].copy()
        d[2:] = np.nextafter(d[2:], rng.choice([-np.inf, np.inf], size=d.size - 2))
        case["density"] = d
    import subprocess

    try:
        r = refrun.run_reference(case, max_steps=steps)
    except subprocess.CalledProcessError:
        return -1, -1, False
    finite = all(np.all(np.isfinite(r[k])) for k in ("rho", "ux", "uy", "T"))
    return int(r["stop"]), int(r["step"]), bool(finite)


def ensemble_status(side=64, steps=1000, seed=1234, n=512):
    """The UQ ensemble's samples of the given side (512 Couette samples,
    u_w ~ U(0.05, 0.2), tau ~ U(0.02, 0.1), Pr ~ U(0.6, 1.0), WENO5, RK3):
    what the reference's driver reports after `steps` steps for each --
    stop (1: runOne's hasFailed, the equilibrium check) and the step it
    stopped at -- and the same for a second reference run whose interior
    densities differ by 1 ulp (how much of that record rounding decides)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    samples = W.uq_ensemble(n=n, seed=seed)
    picks = [(k, d) for k, d in enumerate(samples) if d["nx"] == side]
    with cf.ProcessPoolExecutor(max_workers=os.cpu_count() or 1, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_ref_status, [(d, steps, False) for _, d in picks]))
        res_p = list(ex.map(_ref_status, [(d, steps, True) for _, d in picks]))
    arrays = {"index": np.array([k for k, _ in picks]), "side": np.array(side), "steps": np.array(steps),
              "seed": np.array(seed), "n": np.array(n),
              "u_w": np.array([d["u_w"] for _, d in picks]), "tau": np.array([d["tau"] for _, d in picks]),
              "Pr": np.array([d["Pr"] for _, d in picks]),
              "stop": np.array([r[0] for r in res]), "step": np.array([r[1] for r in res]),
              "finite": np.array([r[2] for r in res]),
              "stop_ulp": np.array([r[0] for r in res_p]), "step_ulp": np.array([r[1] for r in res_p])}
    np.savez_compressed(os.path.join(OUT, "ensemble%d_status.npz" % side), **arrays)
    fail, fail_p = arrays["stop"] != 2, arrays["stop_ulp"] != 2
    print("ensemble%d_status.npz: %d samples, %d did not complete (%d crashed); 1-ulp run %d (%d crashed), "
          "disagreeing on %d" % (side, len(picks), int(fail.sum()), int((arrays["stop"] == -1).sum()),
                                 int(fail_p.sum()), int((arrays["stop_ulp"] == -1).sum()), int((fail != fail_p).sum())))


def per_node_ids(case):
    """The same case with every node its own property id (same values), so
    that each node's inputs can be changed alone."""
    bnd = np.asarray(case["bnd"])
    out = dict(case)
    for k in ("density", "pressure", "temp", "velocityX", "velocityY", "cellType"):
        out[k] = np.asarray(case[k])[bnd.reshape(-1)]
    out["numProps"] = bnd.size
    out["bnd"] = np.arange(bnd.size, dtype=np.int64).reshape(bnd.shape)
    return out


def f32ulp_perturbed(case, seed=77):
    """Every non-solid node's density moved by one single-precision ulp
    (relative 2^-24), up or down with seeded signs."""
    c = per_node_ids(case)
    rng = np.random.default_rng(seed)
    d = np.asarray(c["density"], dtype=np.float64).copy()
    move = np.asarray(c["cellType"]) != 2
    d[move] *= 1.0 + rng.choice([-1.0, 1.0], size=int(move.sum())) * 2.0 ** -24
    c["density"] = d
    return c


def _ref_macro(args):
    case, steps = args
    r = refrun.run_reference(case, max_steps=steps)
    return {k: r[k] for k in ("rho", "ux", "uy", "T")}


def f32_spread():
    """How far the reference moves, on each short-horizon fixture case, when
    every node's density changes by one single-precision ulp: the relative
    L2 of rho, u, T of that run against the unperturbed one (the committed
    fixture's fields, which the per-node-id case reproduces bit for bit).
    Cases: couette16.npz (6 schemes, 50 steps), riemann32.npz (2 cases),
    riemann256_500.npz."""
    import concurrent.futures as cf
    import multiprocessing as mp

    jobs, refs, names = [], [], []
    for fname in ("couette16.npz", "riemann32.npz"):
        z = np.load(os.path.join(OUT, fname))
        metas = json.loads(str(z["meta"]))
        for k, meta in enumerate(metas):
            case = W.build(meta["builder"], **meta["kwargs"])
            steps = int(z["c%d_step" % k])
            jobs += [(per_node_ids(case), steps), (f32ulp_perturbed(case), steps)]
            refs.append({f: z["c%d_%s" % (k, f)] for f in ("rho", "ux", "uy", "T")})
            names.append("%s[%d]" % (fname, k))
    z = np.load(os.path.join(OUT, "riemann256_500.npz"))
    case = W.build("riemann", **json.loads(str(z["kwargs"])))
    jobs += [(per_node_ids(case), int(z["step"])), (f32ulp_perturbed(case), int(z["step"]))]
    refs.append({f: z[f] for f in ("rho", "ux", "uy", "T")})
    names.append("riemann256_500.npz")
    with cf.ProcessPoolExecutor(max_workers=os.cpu_count() or 1, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_ref_macro, jobs))
    errs = []
    for j, name in enumerate(names):
        same, pert = res[2 * j], res[2 * j + 1]
        for f in ("rho", "ux", "uy", "T"):
            assert np.array_equal(same[f], refs[j][f]), (name, f)  # per-node ids change nothing
        errs.append(_l2_errors(pert, refs[j]))
        print(name, "FP32-ulp spread (rho, u, T):", ["%.2e" % e for e in errs[-1]])
    np.savez_compressed(os.path.join(OUT, "f32_spread.npz"), names=np.array(names), err=np.array(errs),
                        perturb_seed=np.array(77))


VISCOSITY_LAWS = (dict(model="VHS", mu_ref=0.05, T_ref=1.0, upsilon=0.25),
                  dict(model="VHS", mu_ref=1.8e-5, T_ref=273.0, upsilon=0.31),
                  dict(model="sutherland", mu_ref=0.05, T_ref=1.0, S_v=0.4),
                  dict(model="sutherland", mu_ref=1.716e-5, T_ref=273.15, S_v=110.4))


def viscosity_laws():
    """The viscosity laws as the reference's own OpenCL generator writes them
    (CODE/Python/simLB/codeCL.py: genOpenCL, 60-69 and 986-990): the
    generator runs in a temporary directory (it writes kernel.cl there) for
    each law, every `double mu = ...;` line it emits is collected (all must
    be the same expression), and the expression is evaluated with the
    constants it emits over a grid of temperatures.  The fixture keeps the
    expressions and the values."""
    import importlib.util
    import math
    import re
    import tempfile

    spec = importlib.util.spec_from_file_location(
        "ref_codeCL", os.path.join(REF_ROOT, "CODE", "Python", "simLB", "codeCL.py"))
    codeCL = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(codeCL)
    ex = [0, 1, 0, -1, 0, 1, -1, -1, 1, 2, 0, -2, 0]
    ey = [0, 0, 1, 0, -1, 1, 1, -1, -1, 0, 2, 0, -2]
    inp = dict(Nx=8, Ny=8, Ni=13, FMETHOD=1, RKMETHOD=1, K=3.0, Pr=0.71, R=1.0, Tc=1.0, b=5.0, dt=0.25,
               isSolid=0, mirrorE=0, mirrorN=0, mirrorS=0, mirrorW=0, periodicX=1, periodicY=0)
    cwd = os.getcwd()
    arrays, exprs = {}, []
    for j, law in enumerate(VISCOSITY_LAWS):
        with tempfile.TemporaryDirectory(prefix="gencl_") as tmp:
            os.chdir(tmp)
            try:
                codeCL.genOpenCL(dict(inp), dict(law), ex, ey, [1.0] * inp["Nx"], [1.0] * inp["Ny"])
                src = open("kernel.cl").read()
            finally:
                os.chdir(cwd)
        consts = {m.group(1): float(m.group(2))
                  for m in re.finditer(r"__constant double (\w+) = ([-+0-9.eE]+);", src)}
        lines = sorted({m.group(1).strip() for m in re.finditer(r"double mu = (.+);", src)})
        # the laws use T (or T2, the same temperature, in one kernel)
        forms = sorted({ln.replace("T2", "T") for ln in lines})
        assert len(forms) == 1, forms
        T = np.linspace(0.2, 3.0, 57) * law["T_ref"]
        env = dict(consts, powr=math.pow)
        mu = np.array([eval(forms[0], {"__builtins__": {}}, dict(env, T=t)) for t in T])
        exprs.append(dict(law, expression=forms[0], constants=consts))
        arrays["T%d" % j] = T
        arrays["mu%d" % j] = mu
    arrays["laws"] = np.array(json.dumps(exprs))
    np.savez_compressed(os.path.join(OUT, "viscosity_laws.npz"), **arrays)
    for e in exprs:
        print("viscosity_laws.npz:", e["model"], e["expression"])


def main():
    if sys.argv[1:] == ["viscosity"]:  # needs only the reference's Python sources
        viscosity_laws()
        return
    if not refrun.available():
        sys.exit("reference binary missing: make -C oracle")
    if sys.argv[1:] == ["mat"]:
        mat_input()
        return
    if sys.argv[1:] == ["chaos"]:
        chaos()
        return
    if sys.argv[1:] == ["riemann"]:
        riemann_floor()
        return
    if sys.argv[1:] == ["ensemble"]:
        ensemble_status()
        return
    if sys.argv[1:] == ["spread"]:
        f32_spread()
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
    chaos()
    riemann_floor()
    ensemble_status()
    f32_spread()
    viscosity_laws()


if __name__ == "__main__":
    main()
