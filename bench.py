"""Benchmark: batched D2Q13 thermal LBM throughput (f+h MLUPS) on B200.

Workload (default): the UQ ensemble -- 512 Couette samples, square sides
drawn from {64,128,256,512}, u_w~U(0.05,0.2), tau~U(0.02,0.1),
Pr~U(0.6,1.0), WENO5 fluxes, RK3 (the reference's RKMETHOD 1), FP32 state
with FP64 moment sums.  One bench step = one time step of every sample
(1 LU = one node, f and h, all 13 velocities, all RK stages).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  Under torchrun each rank advances its own
ensemble (weak scaling, no data-path collective); timings are the max over
ranks.  ``--impl reference`` times the reference C++ solver (oracle/_ref,
built from the reference's unmodified sources) on the host cores instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG_F32 = 208  # algorithmic bytes per LU: f and h (26 values) read + written once, 4-byte state
B_ALG_F64 = 416
WORKLOAD = "uq_ensemble_couette_weno5_rk3"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--samples", type=int, default=512)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile", default="0,0")
    ap.add_argument("--serving-seconds", type=float, default=45.0,
                    help="Poisson arrival window of the serving run (0: skip it)")
    ap.add_argument("--no-probes", action="store_true",
                    help="only the timed ensemble run: no accuracy, plain-FP64, serving or CPU runs (profiling)")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the FP32-vs-FP64 ensemble comparison (the configuration's 1000; 0: skip it)")
    ap.add_argument("--long", action="store_true",
                    help="also run the flat-plate batch for its configured 20000 steps (about 3 minutes)")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fp:
            d = json.load(fp)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as fp:
            for line in fp:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# steps each reference process runs per bench step, by grid side: about
# 2.6e5 lattice updates (a few seconds of one core) for every side
REF_SIDE_STEPS = {64: 64, 128: 16, 256: 4, 512: 1}


def cpu_reference_arm(samples, n_procs):
    """The reference C++ solver (oracle/_ref, built from the reference's
    unmodified sources; else the FP64 C restatement) on the ensemble's own
    mix of grid sides.

    The reference has no threading, so n_procs independent processes run at
    once, one ensemble sample each, cycling through the sides 64, 128, 256,
    512 (REF_SIDE_STEPS steps each).  Each process reports the seconds of its
    own step loop, giving the cost of a lattice update per side with every
    core busy.  The ensemble's CPU throughput is then n_procs x its nodes
    over one pass of it at those per-side costs:
        MLUPS = n_procs * sum_s N_s / sum_s (N_s * t_LU(s)),
    N_s the ensemble's nodes on grids of side s."""
    from oracle import refrun
    from uq_b200 import workloads as W

    sides = sorted(REF_SIDE_STEPS)
    by_side = {sd: [d for d in samples if d["nx"] == sd] for sd in sides}
    nodes_by_side = {sd: sum(d["nx"] * d["ny"] for d in by_side[sd]) for sd in sides}
    total_nodes = sum(nodes_by_side.values())
    present = [sd for sd in sides if by_side[sd]]
    t_lu = {}
    if refrun.available():
        kind = "reference"
        picks = []
        for j in range(max(n_procs, len(present))):
            sd = present[j % len(present)]
            lst = by_side[sd]
            picks.append((sd, lst[(j // len(present)) % len(lst)]))
        tmp = tempfile.mkdtemp(prefix="refarm_")
        procs, work = [], []
        for k, (sd, d) in enumerate(picks):
            wd = os.path.join(tmp, "p%d" % k)
            os.makedirs(wd)
            steps = REF_SIDE_STEPS[sd]
            refrun.write_lbmv(os.path.join(wd, "case.lbmv"), refrun.case_to_vars(W.ensemble_case(dict(d, steps=steps))))
            work.append((sd, wd, d["nx"] * d["ny"] * steps))
        t0 = time.perf_counter()
        for sd, wd, _ in work:
            procs.append(subprocess.Popen([refrun.REF_BIN, "case.lbmv", "out.lbmv", str(REF_SIDE_STEPS[sd])], cwd=wd,
                                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
        for p in procs:
            p.wait()
        wall = time.perf_counter() - t0
        per = {sd: [] for sd in sides}
        for sd, wd, lu in work:
            secs = float(refrun.read_lbmv(os.path.join(wd, "out.lbmv"))["scalars"][7])
            per[sd].append(secs / lu)
        subprocess.run(["rm", "-rf", tmp])
        cores = len(picks)
        t_lu = {sd: float(np.mean(v)) for sd, v in per.items() if v}
    else:
        kind = "port"
        from oracle import oracle as O

        t0 = time.perf_counter()
        for sd in present:
            d = by_side[sd][0]
            steps = max(1, REF_SIDE_STEPS[sd] // 8)
            o = O.Oracle(W.ensemble_case(dict(d, steps=steps)))
            t1 = time.perf_counter()
            o.step(steps)
            t_lu[sd] = (time.perf_counter() - t1) / (d["nx"] * d["ny"] * steps)
        wall = time.perf_counter() - t0
        cores = 1
    pass_s = sum(nodes_by_side[sd] * t_lu[sd] for sd in present)
    mlups = cores * total_nodes / pass_s / 1e6
    detail = {"us_per_lu_by_side": {str(sd): 1e6 * t_lu[sd] for sd in present},
              "node_share_by_side": {str(sd): nodes_by_side[sd] / total_nodes for sd in present}}
    return mlups, cores, kind, wall, detail


def run_reference_impl(args, rank, world):
    if rank != 0:
        return
    from uq_b200 import workloads as W

    samples = W.uq_ensemble(n=args.samples, seed=args.seed)
    ncores = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference_arm(samples, ncores)
    vals, walls = [], []
    kind, detail = "reference", {}
    for _ in range(args.steps):
        v, cores, kind, wall, detail = cpu_reference_arm(samples, ncores)
        vals.append(v)
        walls.append(wall)
    value = float(np.mean(vals))
    sample = ("per bench step %d concurrent reference processes, one ensemble sample each, cycling through the "
              "sides 64/128/256/512 (%s steps); per-side cost per lattice update weighted by the ensemble's node "
              "share" % (cores, "/".join(str(REF_SIDE_STEPS[s]) for s in sorted(REF_SIDE_STEPS))))
    out = {
        "metric": "batched f+h MLUPS (UQ ensemble, WENO5 RK3)", "value": value, "unit": "MLUPS",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(walls)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "samples_per_gpu": args.samples, "sides": [64, 128, 256, 512],
                   "seed": args.seed, "reference_sample": sample},
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cores, "kind": kind, "sample": sample,
                         **detail},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def field_errors(m, r):
    """Relative L2 and max-norm differences of rho, |u| (vector difference)
    and T between two macro dicts (m against the reference r)."""
    out = {}
    for name in ("rho", "u", "T"):
        if name == "u":
            d = np.sqrt((m["ux"] - r["ux"]) ** 2 + (m["uy"] - r["uy"]) ** 2)
            ref = np.hypot(r["ux"], r["uy"])
        else:
            d = np.abs(m[name] - r[name])
            ref = np.abs(r[name])
        out[name] = (float(np.linalg.norm(d) / max(np.linalg.norm(ref), 1e-300)),
                     float(d.max() / max(ref.max(), 1e-300)))
    return out


def _timed_steps(b, n):
    """Device time (ms) of n steps of a batch, CUDA events on its stream."""
    import torch

    st = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    b.step(n)
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def ulp_perturbed(case, seed=77):
    """The same case with every interior node's density moved by one unit in
    the last place, up or down (seeded): the inputs of a second FP64 run that
    differs from the first only by rounding."""
    rng = np.random.default_rng(seed)
    d = np.asarray(case["density"], dtype=np.float64).copy()
    d[2:] = np.nextafter(d[2:], rng.choice([-np.inf, np.inf], size=d.size - 2))
    return dict(case, density=d)


def accuracy_probe(samples, steps=1000):
    """The mixed path against the FP64 path on every sample of the ensemble
    after `steps` steps (the configuration's full length), with the FP64
    floor beside it.

    Three batches run the ensemble: FP64, FP64 with every interior density
    moved by 1 ulp (ulp_perturbed), and FP32.  Reported per precision: how
    many samples finished with status 0; over the samples all three finished:
    the relative L2 of rho, |u|, T of FP32 against FP64 (max, median, count
    within 1e-5), the same for the perturbed FP64 run (the floor: how far two
    FP64 runs drift apart from rounding alone), and FP32's error in units of
    that floor.  The FP64 batch's time gives the batched FP64 MLUPS of the
    same ensemble and step count."""
    from uq_b200 import workloads as W
    from uq_b200.solver import Batch

    cases = [W.ensemble_case(d) for d in samples]

    def run(cs, prec):
        b = Batch(cs, prec)
        ms = _timed_steps(b, steps)
        mlups = b.nodes * steps / (ms * 1e3)
        st = b.status()
        macros = [b.macro(k) for k in range(len(cs))]
        b.close()
        return macros, st, mlups

    m64, st64, mlups64 = run(cases, "f64")
    mp, stp, _ = run([ulp_perturbed(c) for c in cases], "f64")
    floor = [field_errors(mp[k], m64[k]) for k in range(len(cases))]
    del mp
    m32, st32, mlups32 = run(cases, "f32")
    err = [field_errors(m32[k], m64[k]) for k in range(len(cases))]
    del m32, m64
    ok = [k for k in range(len(cases)) if st64[k] == 0 and stp[k] == 0 and st32[k] == 0]
    names = ("rho", "u", "T")

    def summary(e):
        v = {n: [e[k][n][0] for k in ok] for n in names}
        return ({n: float(np.max(v[n])) if ok else None for n in names},
                {n: float(np.median(v[n])) if ok else None for n in names})

    emax, emed = summary(err)
    fmax, fmed = summary(floor)
    ratio = [max(err[k][n][0] / max(floor[k][n][0], 1e-300) for n in names) for k in ok]
    sides = sorted({d["nx"] for d in samples})
    return {
        "steps": steps, "samples": len(cases),
        "status_ok": {"f32": int((st32 == 0).sum()), "f64": int((st64 == 0).sum()),
                      "f64_ulp_perturbed": int((stp == 0).sum())},
        "failed_by_side": {str(sd): {"f32": int(sum(1 for k, d in enumerate(samples) if d["nx"] == sd and st32[k])),
                                     "f64": int(sum(1 for k, d in enumerate(samples) if d["nx"] == sd and st64[k]))}
                           for sd in sides},
        "failed_same_samples": bool(np.array_equal(st32 != 0, st64 != 0)),
        "compared_samples": len(ok),
        "l2_rel_max": emax, "l2_rel_median": emed,
        "samples_within_1e-5": int(sum(all(err[k][n][0] <= 1e-5 for n in names) for k in ok)),
        "fp64_floor_l2_rel_max": fmax, "fp64_floor_l2_rel_median": fmed,
        "f32_over_floor": {"max": float(np.max(ratio)) if ratio else None,
                           "median": float(np.median(ratio)) if ratio else None},
        "batched_fp64_mlups": mlups64, "batched_fp32_mlups_untimed_steps": mlups32,
    }


def config_probes(seed=99, plate_steps=50):
    """The other full-size workloads.

    Riemann 2048 x 2048 (Lax-Liu 3, NND, RK1 -- the reference has no RK2 --,
    tau 1e-3, 500 steps): FP32 and FP64 timed on the device, then the FP32
    fields against the FP64 ones.  Flat plate, 16 samples of 2048 x 512 on
    the y-stretched grid with Ma ~ U(1.5, 2.5), tau ~ U(5e-4, 2e-3) (WENO5,
    RK3): FP32 timed over plate_steps steps (the configuration's length is
    20000; --long runs all of them) with the status of every sample after
    them, and FP32 against FP64 after 10 steps."""
    from uq_b200 import workloads as W
    from uq_b200.solver import Batch

    out = {}
    case = W.riemann(nx=2048, ny=2048, steps=500)
    res = {}
    for prec in ("f32", "f64"):
        b = Batch([case], prec)
        ms = _timed_steps(b, 500)
        res[prec] = (b.nodes * 500 / (ms * 1e3), int(b.status()[0]), b.macro(0))
        b.close()
    err = field_errors(res["f32"][2], res["f64"][2])
    out["riemann_2048_nnd_rk1_500"] = {
        "mlups_f32": res["f32"][0], "mlups_f64": res["f64"][0], "status_f32": res["f32"][1],
        "status_f64": res["f64"][1], "f32_vs_f64_l2": {k: v[0] for k, v in err.items()},
        "f32_vs_f64_linf": {k: v[1] for k, v in err.items()}}
    rng = np.random.default_rng(seed)
    draws = [(float(rng.uniform(1.5, 2.5)), float(rng.uniform(5e-4, 2e-3))) for _ in range(16)]
    plates = [W.flat_plate(mach=m, tau=t, steps=20000) for m, t in draws]
    b = Batch(plates, "f32")
    ms = _timed_steps(b, plate_steps)
    mlups = b.nodes * plate_steps / (ms * 1e3)
    st_end = b.status()
    b.close()
    long_run = {}
    if plate_steps >= 1000:
        # the configured length: which plates complete, in FP32 and in FP64
        b = Batch(plates, "f64")
        ms64 = _timed_steps(b, plate_steps)
        st64 = b.status()
        b.close()
        long_run = {"per_plate": [{"mach": m, "tau": t, "status_f32": int(a), "status_f64": int(c)}
                                  for (m, t), a, c in zip(draws, st_end, st64)],
                    "mlups_f64": sum(pl["bnd"].size for pl in plates) * plate_steps / (ms64 * 1e3)}
    b32, b64 = Batch(plates, "f32"), Batch(plates, "f64")
    b32.step(10)
    b64.step(10)
    worst = {"rho": 0.0, "u": 0.0, "T": 0.0}
    for k in range(len(plates)):
        e = field_errors(b32.macro(k), b64.macro(k))
        for name in worst:
            worst[name] = max(worst[name], e[name][0])
    b32.close()
    b64.close()
    out["flat_plate_16x2048x512_weno5_rk3"] = {
        "mlups_f32": mlups, "steps_timed": plate_steps, "status_ok_after_timed_steps": int((st_end == 0).sum()),
        **long_run,
        "f32_vs_f64_l2_max_10_steps": worst}
    return out


def plain_fp64_probe(samples, steps=10, n=32):
    """The plain FP64 path (one handle per sample, as a drop-in for runOne)
    on the first n samples: MLUPS, to compare with the batched path."""
    import torch

    from uq_b200 import workloads as W
    from uq_b200.solver import Solver

    picked = samples[:n]
    solvers = [Solver(W.ensemble_case(d), "f64") for d in picked]
    for s in solvers:
        s.step(2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in solvers:
        s.step(steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    lu = sum(d["nx"] * d["ny"] for d in picked) * steps
    for s in solvers:
        s.close()
    return lu / wall / 1e6


def rank_seed(seed, rank):
    """Each rank advances its own seeded ensemble; rank 0 is the 1-GPU run."""
    return seed + 7919 * rank


def reduce_over_ranks(x, dist, op, device):
    """x reduced over the ranks (dist None: one rank); op 'sum' or 'max'."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_mlups(total_nodes, steps, max_ms):
    """Whole-job MLUPS: all ranks' lattice updates over the slowest rank's time."""
    return total_nodes * steps / (max_ms * 1e3)


SERVE_SIDES = (32, 1024)      # square grid side ~ U{32..1024}
SERVE_STEPS = (200, 5000)     # step count ~ U{200..5000}


def _serving_requests(seconds, lam, seed):
    """Poisson(lam) arrivals over `seconds`: Couette or Riemann solves with
    random side, step count and RK method (RK1/RK3); Couette solves use
    WENO5 or NND, Riemann solves NND (with WENO5 the Riemann problem
    reaches the equilibrium failure check within 500-3000 steps at every
    CFL tried, in FP64 as in FP32)."""
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / lam)
        if t >= seconds:
            break
        kind = ["couette", "riemann"][int(rng.integers(0, 2))]
        fm = int(rng.integers(0, 2))
        reqs.append(dict(t=t, kind=kind, side=int(rng.integers(SERVE_SIDES[0], SERVE_SIDES[1] + 1)),
                         steps=int(rng.integers(SERVE_STEPS[0], SERVE_STEPS[1] + 1)),
                         fm=fm if kind == "couette" else 0, rk=int(rng.integers(0, 2)),
                         seed=int(rng.integers(1 << 30))))
    return reqs


def _serving_case(r, steps=None):
    from uq_b200 import workloads as W

    n = steps if steps is not None else r["steps"]
    # CFL numbers at which every method combination stays within the
    # equilibrium check for 5000 steps
    if r["kind"] == "couette":
        return W.couette(nx=r["side"], ny=r["side"], steps=n, seed=r["seed"], fmethod=r["fm"], rkmethod=r["rk"],
                         CFL=0.3)
    return W.riemann(nx=r["side"], ny=r["side"], steps=n, fmethod=r["fm"], rkmethod=r["rk"], CFL=0.05)


def _alone_fp64_rates(sides=(32, 128, 512, 1024), steps=10):
    """Plain FP64 path (one lbm_handle) MLUPS per (kind, rk, fm, side)."""
    import torch

    from uq_b200.solver import Solver

    rates = {}
    for kind in ("couette", "riemann"):
        for rk in (0, 1):
            for fm in ((0, 1) if kind == "couette" else (0,)):
                for side in sides:
                    s = Solver(_serving_case(dict(kind=kind, side=side, rk=rk, fm=fm, seed=1), steps + 2), "f64")
                    s.step(2)
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    s.step(steps)
                    torch.cuda.synchronize()
                    rates[(kind, rk, fm, side)] = side * side * steps / (time.perf_counter() - t0) / 1e6
                    s.close()
    return rates


def _alone_rate(rates, r, sides=(32, 128, 512, 1024)):
    """log-log interpolation of the plain FP64 rate in the grid side."""
    xs = np.log(np.array(sides, dtype=float))
    ys = np.log(np.array([rates[(r["kind"], r["rk"], r["fm"], s)] for s in sides]))
    return float(np.exp(np.interp(np.log(r["side"]), xs, ys)))


def serving_saturated(n_requests=48, seed=777):
    """The server's capacity: n_requests solves of the serving mix submitted
    together at t = 0, makespan from the first submit to the last result in
    host memory.  Against the same requests run one after another on the
    plain FP64 path (rates per kind/method/side, interpolated)."""
    from uq_b200.solver import Server

    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n_requests):
        kind = ["couette", "riemann"][int(rng.integers(0, 2))]
        fm = int(rng.integers(0, 2))
        reqs.append(dict(t=0.0, kind=kind, side=int(rng.integers(SERVE_SIDES[0], SERVE_SIDES[1] + 1)),
                         steps=int(rng.integers(SERVE_STEPS[0], SERVE_STEPS[1] + 1)),
                         fm=fm if kind == "couette" else 0, rk=int(rng.integers(0, 2)),
                         seed=int(rng.integers(1 << 30))))
    cases = [_serving_case(r) for r in reqs]
    srv = Server(precision="f32")
    warm = srv.submit(_serving_case(dict(kind="couette", side=64, steps=20, fm=1, rk=1, seed=3)))
    srv.wait(warm)
    srv.release(warm)
    st0 = srv.stats()
    t0 = time.perf_counter()
    ids = [srv.submit(c) for c in cases]
    codes = []
    for rid in ids:
        srv.wait(rid)
        code, _ = srv.result(rid)
        codes.append(int(code))
        srv.release(rid)
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lu = float(sum(r["side"] ** 2 * r["steps"] for r in reqs))
    rates = _alone_fp64_rates()
    alone = sum(r["side"] ** 2 * r["steps"] / (_alone_rate(rates, r) * 1e6) for r in reqs)
    d = {k: st[k] - st0[k] for k in ("steps", "repacks", "graph_captures", "boundary_seconds", "capture_seconds",
                                     "steps_eager", "steps_graph")}
    return {"requests": n_requests, "completed_ok": int(sum(1 for c in codes if c == 0)), "makespan_s": wall,
            "throughput_mlups": lu / wall / 1e6, "alone_fp64_sequential_mlups": lu / alone / 1e6,
            "speedup_vs_alone_fp64_sequential": alone / wall, "server": d}


def serving_probe(seconds, capacity_mlups, load=0.7, seed=4242):
    """Continuous-batching serving run: Poisson arrivals submitted in real
    time to one lbm_server (FP32), results collected as they finish.
    Latency = result in host memory - scheduled arrival.  The same requests
    run alone one after another on the plain FP64 path would take the sum of
    their alone times (rates measured per kind/method/side, interpolated)."""
    import threading

    from uq_b200.solver import Server

    sides = np.arange(SERVE_SIDES[0], SERVE_SIDES[1] + 1, dtype=float)
    mean_work = float(np.mean(sides ** 2)) * (SERVE_STEPS[0] + SERVE_STEPS[1]) / 2.0
    lam = load * capacity_mlups * 1e6 / mean_work
    reqs = _serving_requests(seconds, lam, seed)
    cases = [_serving_case(r) for r in reqs]
    srv = Server(precision="f32")
    warm = srv.submit(_serving_case(dict(kind="couette", side=64, steps=20, fm=1, rk=1, seed=3)))
    srv.wait(warm)
    srv.release(warm)
    ids, t_arrive, t_done, status = {}, {}, {}, {}
    errors = []
    t0 = time.perf_counter()

    def submitter():
        try:
            for k, (r, c) in enumerate(zip(reqs, cases)):
                dt = t0 + r["t"] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids[srv.submit(c)] = k
                t_arrive[k] = t0 + r["t"]
        except Exception as exc:  # reported below
            errors.append(repr(exc))

    th = threading.Thread(target=submitter)
    th.start()
    got = 0
    while got < len(reqs) and not errors:
        rid = srv.wait_any(timeout=600.0)
        if rid is None:
            errors.append("no request finished within 600 s")
            break
        code, _ = srv.result(rid)  # copy the fields to host memory
        t = time.perf_counter()
        while rid not in ids:  # the submitter records the id right after submit returns
            time.sleep(1e-4)
        t_done[ids[rid]] = t
        status[ids[rid]] = int(code)
        srv.release(rid)
        got += 1
    th.join()
    t_end = time.perf_counter()
    st = srv.stats()
    srv.close()
    lat = np.array([t_done[k] - t_arrive[k] for k in sorted(t_done)])
    lu = float(sum(r["side"] ** 2 * r["steps"] for r in reqs))
    rates = _alone_fp64_rates()
    alone = np.array([r["side"] ** 2 * r["steps"] / (_alone_rate(rates, r) * 1e6) for r in reqs])
    done_k = sorted(t_done)
    return {
        "requests": len(reqs), "completed_ok": int(sum(1 for v in status.values() if v == 0)),
        "arrival_rate_per_s": lam, "offered_load": load, "window_s": seconds,
        "mix": "couette (CFL 0.3, WENO5|NND) | riemann (CFL 0.05, NND), side~U{%d..%d}, steps~U{%d..%d}, "
               "RK1|RK3, FP32" % (SERVE_SIDES + SERVE_STEPS),
        "latency_s": {"p50": float(np.percentile(lat, 50)) if lat.size else None,
                      "p99": float(np.percentile(lat, 99)) if lat.size else None,
                      "max": float(lat.max()) if lat.size else None},
        "latency_over_alone_fp64": {
            "p50": float(np.percentile(lat / alone[done_k], 50)) if lat.size else None,
            "p99": float(np.percentile(lat / alone[done_k], 99)) if lat.size else None},
        "aggregate_mlups": lu / (t_end - t0) / 1e6,
        "busy_mlups": st["lattice_updates"] / max(st["busy_seconds"], 1e-9) / 1e6,
        "alone_fp64_sequential_mlups": lu / float(alone.sum()) / 1e6,
        "server": {k: st[k] for k in ("steps", "repacks", "compactions", "graph_captures", "arena_bytes",
                                      "boundary_seconds", "capture_seconds", "steps_eager", "steps_graph",
                                      "busy_seconds")},
        "errors": errors,
    }


def run_ours(args, rank, world, local_rank):
    import torch

    from uq_b200 import workloads as W
    from uq_b200.solver import Batch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    samples = W.uq_ensemble(n=args.samples, seed=rank_seed(args.seed, rank))
    cases = [W.ensemble_case(d) for d in samples]
    tx, ty = (int(v) for v in args.tile.split(","))
    b = Batch(cases, precision=args.precision, tile=(tx, ty))
    nodes = b.nodes
    st = torch.cuda.ExternalStream(b.stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_over_ranks(x, dist, "max", "cuda")

    total_nodes = reduce_over_ranks(nodes, dist, "sum", "cuda")

    b.step(args.warmup)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    b.step(args.steps)
    e1.record(st)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    ms_per_step = ms / args.steps
    status = b.status()
    value = aggregate_mlups(total_nodes, args.steps, ms)

    # per-phase device time (CUDA events on the batch's stream, no graph)
    phases = b.profile(3)
    names = ["pointwise", "walls2", "stencil1", "walls3", "stencil2", "residual"]
    dom = int(np.argmax(phases[:5]))
    peak, peak_kind = measured_peaks()
    b_alg = B_ALG_F32 if args.precision == "f32" else B_ALG_F64
    achieved = b_alg * nodes / (phases[dom] * 1e-3) / 1e9
    # bytes a phase must move per node, state-sized buffers read or written
    # once (26 values each): pointwise reads the state and writes buffer 2;
    # stencil phase 1 reads buffer 2 and the state, writes buffer 3 and the
    # state; stencil phase 2 reads buffer 3 and the state, writes the state
    es = 4 if args.precision == "f32" else 8
    phase_bytes = {"pointwise": 52 * es, "stencil1": 104 * es, "stencil2": 78 * es}
    phase_frac = {k: phase_bytes[k] * nodes / (phases[names.index(k)] * 1e-3) / 1e9 / peak
                  for k in phase_bytes if phases[names.index(k)] > 0}
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic_per_node.json")
    if os.path.exists(tp):
        with open(tp) as fp:
            tb = json.load(fp).get("%s_%s" % (args.precision, names[dom]))
        if tb:
            traffic = float(tb) * nodes

    # end to end through the C ABI: pinned host fields in (every sample's
    # fields, one copy per field), K steps, every sample's fields out
    n_s = len(cases)
    lattice = sum(c["bnd"].size for c in cases)
    host_in = torch.empty((4, lattice), dtype=torch.float64, pin_memory=True)
    host_out = torch.empty((5, lattice), dtype=torch.float64, pin_memory=True)
    off = 0
    for c in cases:
        ids = c["bnd"].reshape(-1)
        nn = ids.size
        for j, key in enumerate(("density", "velocityX", "velocityY", "temp")):
            host_in[j, off:off + nn] = torch.from_numpy(c[key][ids])
        off += nn
    h2d = host_in.numel() * 8
    d2h = host_out.numel() * 8
    b.macro_all_ptr(*[host_out[j].data_ptr() for j in range(5)])  # untimed: makes the bulk device buffer
    barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(st)
    b.set_macro_all_ptr(*[host_in[j].data_ptr() for j in range(4)])
    b.step(args.steps)
    b.macro_all_ptr(*[host_out[j].data_ptr() for j in range(5)])
    e3.record(st)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e2.elapsed_time(e3))
    e2e_value = aggregate_mlups(total_nodes, args.steps, e2e_ms)

    extra = {}
    if rank == 0 and not args.no_probes:
        if args.accuracy_steps > 0:
            extra["accuracy_vs_fp64"] = accuracy_probe(samples, args.accuracy_steps)
        try:
            extra["configs"] = config_probes(plate_steps=20000 if args.long else 50)
        except Exception as exc:  # reported, not fatal
            extra["configs"] = {"error": repr(exc)}
        try:
            extra["plain_fp64_mlups_32_samples"] = plain_fp64_probe(samples)
        except Exception as exc:  # reported, not fatal
            extra["plain_fp64_mlups_32_samples"] = "error: %s" % exc
        # the headline against both FP64 baselines: the same ensemble batched
        # in FP64 (same step count), and one plain FP64 handle per sample
        acc = extra.get("accuracy_vs_fp64") or {}
        plain = extra.get("plain_fp64_mlups_32_samples")
        extra["speedup"] = {
            "vs_batched_fp64": value / acc["batched_fp64_mlups"] if acc.get("batched_fp64_mlups") else None,
            "vs_plain_fp64": value / plain if isinstance(plain, float) and plain > 0 else None}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.no_probes:
        v, cores, kind, wall, detail = cpu_reference_arm(samples, os.cpu_count() or 1)
        cpu = {"value": v, "unit": "MLUPS", "cores": cores, "kind": kind,
               "sample": "%d concurrent reference processes, one ensemble sample each, cycling through the sides "
                         "64/128/256/512 (%s steps), per-side cost weighted by the ensemble's node share (%.1f s "
                         "wall)" % (cores, "/".join(str(REF_SIDE_STEPS[x]) for x in sorted(REF_SIDE_STEPS)), wall),
               **detail}

    launches = b.launches_per_step(False) * args.steps
    b.close()
    if rank == 0 and world == 1 and args.serving_seconds > 0 and not args.no_probes:
        try:
            extra["serving"] = serving_probe(args.serving_seconds, value)
        except Exception as exc:  # reported, not fatal
            extra["serving"] = {"error": repr(exc)}
        try:
            extra["serving_saturated"] = serving_saturated()
        except Exception as exc:  # reported, not fatal
            extra["serving_saturated"] = {"error": repr(exc)}

    if rank == 0:
        out = {
            "metric": "batched f+h MLUPS (UQ ensemble, WENO5 RK3)", "value": value, "unit": "MLUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "f32" else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "samples_per_gpu": n_s, "sides": [64, 128, 256, 512],
                       "nodes_per_step_per_gpu": nodes, "nodes_per_step_total": int(total_nodes),
                       "steps_per_solve": 1000,
                       "precision": "FP32 state/stencils/collision, FP64 moment sums" if args.precision == "f32"
                       else "FP64", "l2": "inputs larger than L2 (whole-ensemble state ~%.1f GB)" %
                       (nodes * 26 * 4 * (4 if args.precision == "f32" else 8) / 1e9),
                       "parallelism": "samples sharded per rank (dp%d)" % world, "seed": args.seed},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": "k_flux " + names[dom],
                         "peak_kind": peak_kind, "alg_bytes_per_lu": b_alg,
                         "frac_whole_step": b_alg * nodes / (ms_per_step * 1e-3) / 1e9 / peak,
                         "phase_ms": dict(zip(names, [float(x) for x in phases])),
                         "phase_compulsory_bytes_per_node": phase_bytes,
                         "phase_frac_of_peak_at_compulsory_bytes": phase_frac},
            "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": d2h / args.steps,
                    "what": "pinned host fields of every sample -> lbm_batch_set_macro_all, K steps, "
                            "lbm_batch_get_macro_all into pinned host buffers"},
            "gpu_launches": launches,
            "clocks": clk,
            "sample_status": {"ok": int((status == 0).sum()), "failed": int((status != 0).sum())},
            "cpu_baseline": cpu,
        }
        out.update(extra)
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference_impl(args, rank, world)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
