"""Case builders for the synthetic workloads (seeded numpy, FP64 inputs).

A *case* is a dict of the reference solver's configuration variables, with
the same names and meaning as the MAT variables read by
``cpuLBM::loadInput`` (``CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp:113-265``),
plus ``bnd``: the per-node property id in the solver's internal order
``bnd[x, y]`` (``BNDARRAY(x,y)``, ``macros.h:8``).  Property ids index the
tables ``density, pressure, temp, velocityX, velocityY, cellType``;
``cellType`` is 0 fluid, 1 permanent (fixed state), 2 solid
(``cpuLBM.cpp:1215,1486,1625``).  Optional ``dx_array``/``dy_array`` give
non-uniform cell widths (the OpenCL generator's form,
``CODE/Python/simLB/codeCL.py:100-114,611-618``).

Workloads (all synthetic, seeded):

* ``couette``: thermal Couette flow, periodic in x, solid wall rows at
  y=0 (at rest) and y=Ny-1 (moving at ``u_w``), per-node density noise.
* ``riemann``: four-quadrant 2D Riemann problem, transmissive boundaries,
  quadrant states from the table in ``CODE/Python/simLB/makeLaxLiu3.py:115-118``
  (column 0, the (1.5,1.5)/(0.5323,0.3)/(0.138,0.029)/(0.5323,0.3) case)
  placed as in ``makeLaxLiu3.py:79-89``, non-dimensional (R=1).
* ``flat_plate``: supersonic boundary layer on a y-stretched grid
  laid out as ``CODE/Python/simLB/makeBoundaryLayer.py:237-265``.
* ``uq_ensemble``: seeded Couette samples with drawn wall speed, relaxation
  time, Prandtl number and side.
"""
import numpy as np

BASE = dict(
    RKMETHOD=1, FMETHOD=1, CFL=0.5, dtau=0.0, PROCESSOR=0, tt_tref=0.0, tt_time=0.0,
    steps=0, tol=0.0, periodicX=0, periodicY=0, mirrorNorth=0, mirrorSouth=0,
    mirrorEast=0, mirrorWest=0, gamma=1.4, R=1.0, mu=0.05, Pr=0.71, dx=1.0, dy=1.0,
    Lx=0.0, Ly=0.0, rho_ref=1.0, p_ref=1.0, T_ref=1.0, Tc_Tref=1.0, nPrintOut=1 << 30, MAT=0,
    mu_model=0, upsilon=0.0, S_v=0.0,
)


def _finish(case, props, bnd):
    case["numProps"] = len(props["density"])
    for k in ("density", "pressure", "temp", "velocityX", "velocityY"):
        case[k] = np.asarray(props[k], dtype=np.float64)
    case["cellType"] = np.asarray(props["cellType"], dtype=np.int64)
    case["bnd"] = np.ascontiguousarray(bnd, dtype=np.int64)
    return case


def couette(nx=64, ny=128, u_w=0.1, tau=0.05, Pr=0.71, steps=2000, seed=0, noise=1e-4,
            fmethod=1, rkmethod=1, T_w=1.0, rho0=1.0, Tc_Tref=1.0, CFL=0.5):
    """Thermal Couette flow: x periodic, solid rows y=0 (u=0) and y=ny-1 (u=u_w).

    Every interior node gets its own property id so that the seeded density
    noise rho = rho0 * (1 + U(-noise, noise)) survives ``loadInput``.  The
    relaxation time enters the reference as mu = tau * p0 (tau_f = mu / p,
    ``cpuLBM.cpp:952``).
    """
    rng = np.random.default_rng(seed)
    p0 = rho0 * 1.0 * T_w
    case = dict(BASE, periodicX=1, mu=tau * p0, Pr=Pr, steps=steps, FMETHOD=fmethod,
                RKMETHOD=rkmethod, Tc_Tref=Tc_Tref, CFL=CFL, T_ref=T_w, rho_ref=rho0, p_ref=p0)
    nint = nx * (ny - 2)
    rho = rho0 * (1.0 + rng.uniform(-noise, noise, size=nint))
    props = dict(
        density=np.concatenate([[rho0, rho0], rho]),
        pressure=np.zeros(nint + 2),
        temp=np.full(nint + 2, T_w),
        velocityX=np.concatenate([[0.0, u_w], np.zeros(nint)]),
        velocityY=np.zeros(nint + 2),
        cellType=np.concatenate([[2, 2], np.zeros(nint, dtype=np.int64)]),
    )
    bnd = np.empty((nx, ny), dtype=np.int64)
    bnd[:, 0] = 0
    bnd[:, ny - 1] = 1
    bnd[:, 1:ny - 1] = 2 + np.arange(nint).reshape(nx, ny - 2)
    return _finish(case, props, bnd)


# makeLaxLiu3.py:115-118, column 0: rows are quadrants 0 (top right),
# 1 (top left), 2 (bottom left), 3 (bottom right).
RIEMANN_QUADRANTS = dict(
    rho=(1.5, 0.5323, 0.138, 0.5323),
    p=(1.5, 0.3, 0.029, 0.3),
    ux=(0.0, 1.206, 1.206, 0.0),
    uy=(0.0, 0.0, 1.206, 1.206),
)


def riemann(nx=2048, ny=2048, tau=1e-3, steps=500, fmethod=0, rkmethod=0, Tc_Tref=1.5, CFL=0.2):
    """Four-quadrant Riemann problem, transmissive (clamped) boundaries.

    Non-dimensional: R = 1, p_ref = 1, T = p / rho; mu = tau * p_ref.
    Quadrant placement follows ``makeLaxLiu3.py:79-89``; CFL 0.2 is the
    reference setup's own (``makeLaxLiu3.py:22``).  Tc_Tref = 1.5 keeps the
    D2Q13 equilibria positive for the coldest quadrant (T = 0.21): at
    Tc_Tref = 1 the scheme diverges within a few hundred steps.
    """
    q = RIEMANN_QUADRANTS
    case = dict(BASE, mu=tau * 1.0, steps=steps, FMETHOD=fmethod, RKMETHOD=rkmethod,
                Tc_Tref=Tc_Tref, CFL=CFL)
    props = dict(
        density=np.array(q["rho"]), pressure=np.array(q["p"]),
        temp=np.array(q["p"]) / np.array(q["rho"]),
        velocityX=np.array(q["ux"]), velocityY=np.array(q["uy"]),
        cellType=np.zeros(4, dtype=np.int64),
    )
    bnd = np.empty((nx, ny), dtype=np.int64)
    mx, my = nx // 2, ny // 2
    bnd[mx:, my:] = 0
    bnd[:mx, my:] = 1
    bnd[:mx, :my] = 2
    bnd[mx:, :my] = 3
    return _finish(case, props, bnd)


def flat_plate(nx=2048, ny=512, stretch=1.02, mach=2.0, tau=1e-3, steps=20000, dy0=None,
               fmethod=1, rkmethod=1, Tc_Tref=4.0, CFL=0.5):
    """Supersonic flat-plate boundary layer on a y-stretched grid.

    Layout as ``makeBoundaryLayer.py:237-265``: the inlet column x=0 and the
    top row are permanent (cellType 1) at the free-stream state, the wall row
    y=0 is solid at rest with T_wall = T_inf; dy grows by ``stretch`` per row
    away from the wall.  Non-dimensional, R = 1, T_inf = 1.
    """
    gamma = 1.4
    u_inf = mach * np.sqrt(gamma * 1.0)
    dx = 1.0
    if dy0 is None:
        dy0 = 0.25 * dx
    dy = dy0 * stretch ** np.arange(ny)
    case = dict(BASE, mu=tau * 1.0, steps=steps, FMETHOD=fmethod, RKMETHOD=rkmethod,
                Tc_Tref=Tc_Tref, CFL=CFL, dx=dx, dy=float(dy.min()))
    case["dx_array"] = np.full(nx, dx)
    case["dy_array"] = dy
    props = dict(
        density=np.array([1.0, 1.0, 1.0]), pressure=np.zeros(3), temp=np.ones(3),
        velocityX=np.array([u_inf, u_inf, 0.0]), velocityY=np.zeros(3),
        cellType=np.array([0, 1, 2]),
    )
    bnd = np.zeros((nx, ny), dtype=np.int64)
    bnd[0, :] = 1
    bnd[:, ny - 1] = 1
    bnd[:, 0] = 2
    return _finish(case, props, bnd)


def uq_ensemble(n=512, seed=1234, sides=(64, 128, 256, 512), steps=1000):
    """Seeded UQ ensemble of Couette samples: u_w~U(0.05,0.2), tau~U(0.02,0.1),
    Pr~U(0.6,1.0), side drawn uniformly from ``sides``."""
    rng = np.random.default_rng(seed)
    samples = []
    for k in range(n):
        u_w = rng.uniform(0.05, 0.2)
        tau = rng.uniform(0.02, 0.1)
        Pr = rng.uniform(0.6, 1.0)
        side = int(rng.choice(sides))
        samples.append(dict(u_w=u_w, tau=tau, Pr=Pr, nx=side, ny=side, steps=steps,
                            seed=seed * 100003 + k))
    return samples


def random_state(nx, ny, seed, bc="transmissive", fmethod=1, rkmethod=1, solid_frac=0.0, steps=1,
                 mu=0.05, Pr=0.71, du=0.1, drho=0.1, dT=0.1):
    """Seeded random near-equilibrium state: every node is its own property
    with rho in 1 +- drho, T in 1 +- dT, u in +-du; optionally a random
    fraction of solid (cellType 2, at rest) and half as many permanent
    (cellType 1) nodes.  ``bc`` is transmissive (clamped), periodic, mirror
    (all four sides) or mixed (periodic x, mirror north)."""
    rng = np.random.default_rng(seed)
    n = nx * ny
    case = dict(BASE, steps=steps, FMETHOD=fmethod, RKMETHOD=rkmethod, mu=mu, Pr=Pr)
    if bc == "periodic":
        case.update(periodicX=1, periodicY=1)
    elif bc == "mirror":
        case.update(mirrorNorth=1, mirrorSouth=1, mirrorEast=1, mirrorWest=1)
    elif bc == "mixed":
        case.update(periodicX=1, mirrorNorth=1)
    elif bc != "transmissive":
        raise ValueError(bc)
    rho = rng.uniform(1 - drho, 1 + drho, n)
    T = rng.uniform(1 - dT, 1 + dT, n)
    ux = rng.uniform(-du, du, n)
    uy = rng.uniform(-du, du, n)
    ct = np.zeros(n, dtype=np.int64)
    if solid_frac > 0:
        ct[rng.uniform(size=n) < solid_frac] = 2
        ct[rng.uniform(size=n) < solid_frac / 2] = 1
        ux[ct == 2] = 0.0
        uy[ct == 2] = 0.0
    props = dict(density=rho, pressure=np.zeros(n), temp=T, velocityX=ux, velocityY=uy, cellType=ct)
    return _finish(case, props, np.arange(n).reshape(nx, ny))


BUILDERS = dict(couette=couette, riemann=riemann, flat_plate=flat_plate, random_state=random_state)


def build(name, overrides=None, **kwargs):
    """Build a case by builder name, then apply ``overrides`` (extra or
    replaced configuration variables); used by the golden fixtures."""
    case = BUILDERS[name](**kwargs)
    if overrides:
        case.update(overrides)
    return case


def ensemble_case(sample):
    return couette(nx=sample["nx"], ny=sample["ny"], u_w=sample["u_w"], tau=sample["tau"],
                   Pr=sample["Pr"], steps=sample["steps"], seed=sample["seed"])
