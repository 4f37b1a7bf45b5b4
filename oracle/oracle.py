"""ctypes wrapper of the FP64 C restatement (``lbm_oracle.c``).

Test infrastructure only: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py, never by the product package.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liblbm_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrcConfig(C.Structure):
    _fields_ = [
        ("RKMETHOD", C.c_int), ("FMETHOD", C.c_int),
        ("CFL", C.c_double), ("dtau", C.c_double), ("tt_tref", C.c_double), ("tt_time", C.c_double),
        ("steps", C.c_int), ("tol", C.c_double),
        ("periodicX", C.c_int), ("periodicY", C.c_int), ("mirrorNorth", C.c_int),
        ("mirrorSouth", C.c_int), ("mirrorEast", C.c_int), ("mirrorWest", C.c_int),
        ("gamma", C.c_double), ("R", C.c_double), ("mu", C.c_double), ("Pr", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("Lx", C.c_double), ("Ly", C.c_double),
        ("rho_ref", C.c_double), ("p_ref", C.c_double), ("T_ref", C.c_double), ("Tc_Tref", C.c_double),
        ("dx_array", _dp), ("dy_array", _dp),
        ("mu_model", C.c_int), ("upsilon", C.c_double), ("S_v", C.c_double),
    ]


class OrcInit(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("numProps", C.c_int),
        ("bnd", _ip), ("cellType", _ip),
        ("density", _dp), ("pressure", _dp), ("temp", _dp), ("velocityX", _dp), ("velocityY", _dp),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            raise RuntimeError("oracle library missing: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcConfig), C.POINTER(OrcInit)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.orc_run.argtypes = [C.c_void_p, C.c_int, _dp]
        L.orc_get_macro.argtypes = [C.c_void_p] + [_dp] * 5
        L.orc_get_dist.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_set_dist.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_dt.restype = C.c_double
        L.orc_dt.argtypes = [C.c_void_p]
        L.orc_nsteps.argtypes = [C.c_void_p]
        L.orc_step_count.argtypes = [C.c_void_p]
        L.orc_residual.restype = C.c_double
        L.orc_residual.argtypes = [C.c_void_p]
        L.orc_equilibrium.argtypes = [C.c_double] * 7 + [_dp, _dp]
        L.orc_viscosity.restype = C.c_double
        L.orc_viscosity.argtypes = [C.c_int] + [C.c_double] * 5
        _lib = L
    return _lib


def viscosity(mu_model, mu_ref, T_ref, upsilon, S_v, T):
    """The oracle's viscosity law (0 constant, 1 VHS, 2 Sutherland) at each
    temperature of T."""
    L = lib()
    return np.array([L.orc_viscosity(int(mu_model), float(mu_ref), float(T_ref), float(upsilon), float(S_v),
                                     float(t)) for t in np.ravel(T)])


def _d(a):
    return a.ctypes.data_as(_dp)


class Oracle:
    """One FP64 CPU solver instance built from a case dict (uq_b200.workloads)."""

    def __init__(self, case):
        L = lib()
        self._keep = []
        cfg = OrcConfig()
        for name, _ in OrcConfig._fields_:
            if name in ("dx_array", "dy_array"):
                continue
            setattr(cfg, name, type(getattr(cfg, name))(case.get(name, 0)))
        for name in ("dx_array", "dy_array"):
            if case.get(name) is not None:
                arr = np.ascontiguousarray(case[name], dtype=np.float64)
                self._keep.append(arr)
                setattr(cfg, name, _d(arr))
        bnd = np.ascontiguousarray(case["bnd"], dtype=np.int32)
        self.nx, self.ny = bnd.shape
        ini = OrcInit()
        ini.Nx, ini.Ny, ini.numProps = self.nx, self.ny, int(case["numProps"])
        arrs = dict(bnd=bnd, cellType=np.ascontiguousarray(case["cellType"], dtype=np.int32))
        for k in ("density", "pressure", "temp", "velocityX", "velocityY"):
            arrs[k] = np.ascontiguousarray(case[k], dtype=np.float64)
        for k, a in arrs.items():
            self._keep.append(a)
            setattr(ini, k, a.ctypes.data_as(_ip if a.dtype == np.int32 else _dp))
        self._h = L.orc_create(C.byref(cfg), C.byref(ini))
        if not self._h:
            raise ValueError("orc_create rejected the case")

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dt(self):
        return lib().orc_dt(self._h)

    @property
    def nsteps(self):
        return lib().orc_nsteps(self._h)

    @property
    def step_count(self):
        return lib().orc_step_count(self._h)

    def step(self, n=1, residual=False):
        r = C.c_double(0)
        failed = lib().orc_step(self._h, int(n), 1 if residual else 0, C.byref(r))
        return failed, r.value

    def run(self, max_steps=-1):
        trace = np.zeros(max(int(max_steps), 0) if max_steps >= 0 else max(self.nsteps, 1) + 1)
        stop = lib().orc_run(self._h, int(max_steps), _d(trace))
        return stop, trace

    def macro(self):
        n = self.nx * self.ny
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "T", "p")}
        lib().orc_get_macro(self._h, *[_d(out[k]) for k in ("rho", "ux", "uy", "T", "p")])
        return {k: v.reshape(self.nx, self.ny) for k, v in out.items()}

    def dist(self):
        n = self.nx * self.ny * 13
        f, h = np.empty(n), np.empty(n)
        lib().orc_get_dist(self._h, _d(f), _d(h))
        return f.reshape(self.nx, self.ny, 13), h.reshape(self.nx, self.ny, 13)

    def set_dist(self, f, h):
        f = np.ascontiguousarray(f, dtype=np.float64)
        h = np.ascontiguousarray(h, dtype=np.float64)
        lib().orc_set_dist(self._h, _d(f), _d(h))


def equilibrium(rho, ux, uy, T, R, Tc, K):
    eqf, eqh = np.empty(13), np.empty(13)
    lib().orc_equilibrium(rho, ux, uy, T, R, Tc, K, _d(eqf), _d(eqh))
    return eqf, eqh
