"""Python host mirror of the reference's step API over the C ABI.

``Solver`` mirrors the C++ class ``cpuLBM``
(CODE/C++/VS2010/simLB/simLB/cpuLBM.h:16-175): it is built from a case (the
MAT variables of ``loadInput``, see ``uq_b200.workloads``), steps with
``runOne`` / ``run`` and exposes ``rho_G, u_G, T_G, p_G, f_G, h_G`` in the
reference's layouts (``macros.h:8-14``).  ``Batch`` advances many samples
in one launch sequence; ``Server`` runs solves submitted at any time as a
continuous batch.  All run only on the CUDA library; a missing library
raises.
"""
import ctypes as C

import numpy as np

from . import native as N

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


class _CaseBuffers:
    """Holds the numpy arrays a config/init struct points into."""

    def __init__(self, case):
        self.keep = []
        cfg = N.LbmConfig()
        for name, _ in N.LbmConfig._fields_:
            if name in ("dx_array", "dy_array"):
                continue
            setattr(cfg, name, type(getattr(cfg, name))(case.get(name, 0)))
        for name in ("dx_array", "dy_array"):
            if case.get(name) is not None:
                arr = np.ascontiguousarray(case[name], dtype=np.float64)
                self.keep.append(arr)
                setattr(cfg, name, _d(arr))
        bnd = np.ascontiguousarray(case["bnd"], dtype=np.int32)
        ini = N.LbmInit()
        ini.Nx, ini.Ny = bnd.shape
        ini.numProps = int(case["numProps"])
        arrs = dict(bndArray=bnd.reshape(-1), cellType=np.ascontiguousarray(case["cellType"], dtype=np.int32))
        for k in ("density", "pressure", "temp", "velocityX", "velocityY"):
            arrs[k] = np.ascontiguousarray(case[k], dtype=np.float64)
        for k, a in arrs.items():
            self.keep.append(a)
            setattr(ini, k, a.ctypes.data_as(_ip if a.dtype == np.int32 else _dp))
        self.cfg, self.ini = cfg, ini
        self.nx, self.ny = bnd.shape


def mat_case(path):
    """An input MAT file read by the library (loadInput's rules) as a case
    dict: the lbm_config fields, ``bnd`` [x, y] and the property tables."""
    L = N.lib()
    h = C.c_void_p()
    N.check(L.lbm_mat_read_case(str(path).encode(), C.byref(h)), "lbm_mat_read_case")
    try:
        cfg, ini = N.LbmConfig(), N.LbmInit()
        N.check(L.lbm_mat_case_get(h, C.byref(cfg), C.byref(ini)), "lbm_mat_case_get")
        case = {name: getattr(cfg, name) for name, _ in N.LbmConfig._fields_ if name not in ("dx_array", "dy_array")}
        nx, ny, npr = ini.Nx, ini.Ny, ini.numProps
        case["bnd"] = np.ctypeslib.as_array(ini.bndArray, shape=(nx * ny,)).reshape(nx, ny).copy()
        case["numProps"] = npr
        case["cellType"] = np.ctypeslib.as_array(ini.cellType, shape=(npr,)).copy()
        for k in ("density", "pressure", "temp", "velocityX", "velocityY"):
            case[k] = np.ctypeslib.as_array(getattr(ini, k), shape=(npr,)).copy()
        return case
    finally:
        L.lbm_mat_case_free(h)


def read_mat_dist(path, nx, ny):
    """(f, h, t) of a checkpoint MAT file; f, h as [x, y, 13]."""
    f, h, t = np.empty(nx * ny * 13), np.empty(nx * ny * 13), C.c_double()
    N.check(N.lib().lbm_mat_read_dist(str(path).encode(), nx, ny, _d(f), _d(h), C.byref(t)), "lbm_mat_read_dist")
    return f.reshape(nx, ny, 13), h.reshape(nx, ny, 13), t.value


def write_mat_fields(path, fields, t=0.0, dx=1.0, dy=1.0, f=None, h=None, ex=None, ey=None):
    """createMAT's file from host arrays: fields rho, ux, uy, p, T as
    [x, y] arrays; f, h [x, y, 13] and ex, ey [13] optional."""
    nx, ny = fields["rho"].shape
    arrs = [np.ascontiguousarray(fields[k], dtype=np.float64).reshape(-1) for k in ("rho", "ux", "uy", "p", "T")]
    dist = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (f, h, ex, ey)]
    ptr = [None if a is None else _d(a) for a in dist]
    N.check(N.lib().lbm_mat_write_fields(str(path).encode(), nx, ny, *[_d(a) for a in arrs], float(t), float(dx),
                                         float(dy), *ptr), "lbm_mat_write_fields")


def write_hdf5_fields(path, fields, t=0.0, gamma=1.4, R=1.0, T_ref=1.0, rho_ref=1.0, dx=1.0, dy=1.0, f=None,
                      h=None):
    """ClassLBM.saveHDF5's file (LBM.py:516-567) from host arrays: fields
    rho, T, ux, uy as [x, y] arrays; dx, dy scalars or per-cell arrays; f, h
    [x, y, 13] optional (both or neither)."""
    nx, ny = fields["rho"].shape
    arrs = [np.ascontiguousarray(fields[k], dtype=np.float64).reshape(-1) for k in ("rho", "ux", "uy", "T")]
    dxa = np.ascontiguousarray(np.atleast_1d(dx), dtype=np.float64)
    dya = np.ascontiguousarray(np.atleast_1d(dy), dtype=np.float64)
    dist = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (f, h)]
    ptr = [None if a is None else _d(a) for a in dist]
    N.check(N.lib().lbm_hdf5_write_fields(str(path).encode(), nx, ny, *[_d(a) for a in arrs], float(t), float(gamma),
                                          float(R), float(T_ref), float(rho_ref), _d(dxa), dxa.size, _d(dya),
                                          dya.size, *ptr), "lbm_hdf5_write_fields")


class Solver:
    """One solver instance (an ``lbm_handle``): the drop-in for cpuLBM."""

    @classmethod
    def from_mat(cls, path, precision="f64"):
        """new cpuLBM(files) on an input MAT file."""
        return cls(mat_case(path), precision)

    def write_mat(self, path, with_dist=False):
        """createMAT of the current state (rho, ux, uy, p, T, t, dx, dy; f,
        h, ex, ey with with_dist)."""
        N.check(N.lib().lbm_write_mat(self._h, str(path).encode(), 1 if with_dist else 0), "lbm_write_mat")

    def write_hdf5(self, path, with_dist=False):
        """ClassLBM.saveHDF5(all) of the current state: rho, T, ux, uy, t,
        gamma, R, T_ref, rho_ref, dx, dy, Nx, Ny (f, h with with_dist)."""
        N.check(N.lib().lbm_write_hdf5(self._h, str(path).encode(), 1 if with_dist else 0), "lbm_write_hdf5")

    def restore_mat(self, path):
        """Resume from a file write_mat(path, with_dist=True) made: f, h and
        the step count."""
        N.check(N.lib().lbm_restore_mat(self._h, str(path).encode()), "lbm_restore_mat")

    def __init__(self, case, precision="f64"):
        L = N.lib()
        self._bufs = _CaseBuffers(case)
        self.nx, self.ny = self._bufs.nx, self._bufs.ny
        h = C.c_void_p()
        N.check(L.lbm_create(C.byref(self._bufs.cfg), C.byref(self._bufs.ini), N.PREC[precision], C.byref(h)),
                "lbm_create")
        self._h = h
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            N.lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- stepping (cpuLBM::updateStepCount + runOne; main.cpp runSimStep)
    def runOne(self, res=0):
        """One step; returns 1 where the reference's runOne returns hasFailed."""
        code = N.lib().lbm_step(self._h, 1, 1 if res else 0, None)
        if code not in (N.LBM_OK, N.LBM_ERR_EQUILIBRIUM, N.LBM_ERR_NONFINITE):
            N.check(code, "lbm_step")
        return 1 if code == N.LBM_ERR_EQUILIBRIUM else 0

    def step(self, n=1, residual=False):
        """n steps; returns (lbm_status, residual)."""
        r = C.c_double(0)
        code = N.lib().lbm_step(self._h, int(n), 1 if residual else 0, C.byref(r))
        if code not in (N.LBM_OK, N.LBM_ERR_EQUILIBRIUM, N.LBM_ERR_NONFINITE):
            N.check(code, "lbm_step")
        return code, r.value

    def run(self, max_steps=-1, trace_len=None):
        """The reference driver loop; returns (stop, residual trace)."""
        if trace_len is None:
            trace_len = max_steps if max_steps >= 0 else max(self.info().nsteps, 1)
        trace = np.zeros(max(int(trace_len), 1))
        stop = C.c_int(0)
        code = N.lib().lbm_run(self._h, int(max_steps), C.byref(stop), _d(trace), int(trace_len))
        if code not in (N.LBM_OK, N.LBM_ERR_EQUILIBRIUM, N.LBM_ERR_NONFINITE):
            N.check(code, "lbm_run")
        return stop.value, trace

    # -- state
    def info(self):
        inf = N.LbmInfo()
        N.check(N.lib().lbm_get_info(self._h, C.byref(inf)), "lbm_get_info")
        return inf

    @property
    def dt(self):
        return self.info().dt

    @property
    def nsteps(self):
        return self.info().nsteps

    @property
    def step_count(self):
        return self.info().step

    def macro(self):
        n = self.nx * self.ny
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "T", "p")}
        N.check(N.lib().lbm_get_macro(self._h, *[_d(out[k]) for k in ("rho", "ux", "uy", "T", "p")]),
                "lbm_get_macro")
        return {k: v.reshape(self.nx, self.ny) for k, v in out.items()}

    def dist(self):
        n = self.nx * self.ny * 13
        f, h = np.empty(n), np.empty(n)
        N.check(N.lib().lbm_get_dist(self._h, _d(f), _d(h)), "lbm_get_dist")
        return f.reshape(self.nx, self.ny, 13), h.reshape(self.nx, self.ny, 13)

    def set_dist(self, f, h):
        f = np.ascontiguousarray(f, dtype=np.float64)
        h = np.ascontiguousarray(h, dtype=np.float64)
        N.check(N.lib().lbm_set_dist(self._h, _d(f), _d(h)), "lbm_set_dist")

    @property
    def rho_G(self):
        return self.macro()["rho"]

    @property
    def T_G(self):
        return self.macro()["T"]

    @property
    def p_G(self):
        return self.macro()["p"]

    @property
    def u_G(self):
        m = self.macro()
        return np.stack([m["ux"], m["uy"]], axis=-1)

    @property
    def f_G(self):
        return self.dist()[0]

    @property
    def h_G(self):
        return self.dist()[1]

    @property
    def stream(self):
        return N.lib().lbm_stream(self._h)


class Batch:
    """Many samples advanced together (an ``lbm_batch``)."""

    def __init__(self, cases, precision="f32", tile=(0, 0), use_graph=True):
        L = N.lib()
        self._bufs = [_CaseBuffers(c) for c in cases]
        n = len(cases)
        cfgs = (N.LbmConfig * n)(*[b.cfg for b in self._bufs])
        inis = (N.LbmInit * n)(*[b.ini for b in self._bufs])
        opt = N.LbmBatchOptions(N.PREC[precision], int(tile[0]), int(tile[1]), 1 if use_graph else 0)
        h = C.c_void_p()
        N.check(L.lbm_batch_create(n, cfgs, inis, C.byref(opt), C.byref(h)), "lbm_batch_create")
        self._h = h
        self.n = n
        self.shapes = [(b.nx, b.ny) for b in self._bufs]
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            N.lib().lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nodes(self):
        return N.lib().lbm_batch_nodes(self._h)

    @property
    def stream(self):
        return N.lib().lbm_batch_stream(self._h)

    def step(self, n=1, residual=False):
        N.check(N.lib().lbm_batch_step(self._h, int(n), 1 if residual else 0), "lbm_batch_step")

    def status(self):
        st = np.zeros(self.n, dtype=np.int32)
        N.check(N.lib().lbm_batch_status(self._h, st.ctypes.data_as(_ip)), "lbm_batch_status")
        return st

    def residuals(self):
        r = np.zeros(self.n)
        N.check(N.lib().lbm_batch_residuals(self._h, _d(r)), "lbm_batch_residuals")
        return r

    def macro(self, s):
        nx, ny = self.shapes[s]
        out = {k: np.empty(nx * ny) for k in ("rho", "ux", "uy", "T", "p")}
        N.check(N.lib().lbm_batch_get_macro(self._h, int(s), *[_d(out[k]) for k in ("rho", "ux", "uy", "T", "p")]),
                "lbm_batch_get_macro")
        return {k: v.reshape(nx, ny) for k, v in out.items()}

    def dist(self, s):
        nx, ny = self.shapes[s]
        f, h = np.empty(nx * ny * 13), np.empty(nx * ny * 13)
        N.check(N.lib().lbm_batch_get_dist(self._h, int(s), _d(f), _d(h)), "lbm_batch_get_dist")
        return f.reshape(nx, ny, 13), h.reshape(nx, ny, 13)

    def set_dist(self, s, f, h):
        f = np.ascontiguousarray(f, dtype=np.float64)
        h = np.ascontiguousarray(h, dtype=np.float64)
        N.check(N.lib().lbm_batch_set_dist(self._h, int(s), _d(f), _d(h)), "lbm_batch_set_dist")

    def set_macro_ptr(self, s, rho, ux, uy, T):
        """Equilibrium restart from host fields given as raw addresses (for
        pinned buffers); asynchronous on the batch's stream."""
        c = C.cast
        N.check(N.lib().lbm_batch_set_macro(self._h, int(s), c(rho, _dp), c(ux, _dp), c(uy, _dp), c(T, _dp)),
                "lbm_batch_set_macro")

    def macro_ptr(self, s, rho, ux, uy, T, p):
        """Macroscopic fields into host buffers given as raw addresses."""
        c = C.cast
        N.check(N.lib().lbm_batch_get_macro(self._h, int(s), c(rho, _dp), c(ux, _dp), c(uy, _dp), c(T, _dp),
                                            c(p, _dp)), "lbm_batch_get_macro")

    def set_macro_all_ptr(self, rho, ux, uy, T):
        """Every sample's fields at once from host buffers given as raw
        addresses (samples one after another, each [x*Ny + y]); asynchronous
        on the batch's stream."""
        c = C.cast
        N.check(N.lib().lbm_batch_set_macro_all(self._h, c(rho, _dp), c(ux, _dp), c(uy, _dp), c(T, _dp)),
                "lbm_batch_set_macro_all")

    def macro_all_ptr(self, rho, ux, uy, T, p):
        """Every sample's fields at once into host buffers given as raw
        addresses (same layout as set_macro_all_ptr)."""
        c = C.cast
        N.check(N.lib().lbm_batch_get_macro_all(self._h, c(rho, _dp), c(ux, _dp), c(uy, _dp), c(T, _dp), c(p, _dp)),
                "lbm_batch_get_macro_all")

    def macro_all(self):
        """[macro(s) for every sample], through one bulk copy."""
        n = sum(nx * ny for nx, ny in self.shapes)
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "T", "p")}
        N.check(N.lib().lbm_batch_get_macro_all(self._h, *[_d(out[k]) for k in ("rho", "ux", "uy", "T", "p")]),
                "lbm_batch_get_macro_all")
        res, off = [], 0
        for nx, ny in self.shapes:
            res.append({k: v[off:off + nx * ny].reshape(nx, ny) for k, v in out.items()})
            off += nx * ny
        return res

    def set_macro_all(self, fields):
        """fields: one dict (rho, ux, uy, T as [Nx, Ny]) per sample."""
        arrs = [np.ascontiguousarray(np.concatenate([np.asarray(f[k], dtype=np.float64).reshape(-1) for f in fields]))
                for k in ("rho", "ux", "uy", "T")]
        N.check(N.lib().lbm_batch_set_macro_all(self._h, *[_d(a) for a in arrs]), "lbm_batch_set_macro_all")
        self.status()  # synchronises: the host arrays may be released after return

    def set_macro(self, s, rho, ux, uy, T):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (rho, ux, uy, T)]
        N.check(N.lib().lbm_batch_set_macro(self._h, int(s), *[_d(a) for a in arrs]), "lbm_batch_set_macro")
        self.status()  # synchronises: the host arrays may be released after return

    def profile(self, n=3):
        ms = np.zeros(6)
        N.check(N.lib().lbm_batch_profile(self._h, int(n), _d(ms), 6), "lbm_batch_profile")
        return ms

    def autotune(self, candidates=None, steps=2):
        """Pick the fastest tile shape for this batch (state unchanged);
        returns ((tile_x, tile_y), {candidate: ms per step})."""
        if candidates is None:
            candidates = [(32, 8), (16, 16), (64, 4), (8, 32), (32, 4), (16, 8)]
        flat = np.array([v for c in candidates for v in c], dtype=np.int32)
        chosen = np.zeros(2, dtype=np.int32)
        ms = np.zeros(len(candidates))
        N.check(N.lib().lbm_batch_autotune(self._h, flat.ctypes.data_as(_ip), len(candidates), int(steps),
                                           chosen.ctypes.data_as(_ip), _d(ms)), "lbm_batch_autotune")
        return (int(chosen[0]), int(chosen[1])), {tuple(c): float(t) for c, t in zip(candidates, ms)}

    def launches_per_step(self, residual=False):
        return N.lib().lbm_batch_launches_per_step(self._h, 1 if residual else 0)


class Server:
    """A request server (an ``lbm_server``): solves submitted at any time run
    as one continuous batch on the GPU; results come back per request."""

    def __init__(self, precision="f32", tile=(0, 0), arena_bytes=0, hbm_fraction=0.0, max_resident=0,
                 max_queued=0, use_graph=True, status_poll_steps=0, fast_lane_steps=0):
        L = N.lib()
        opt = N.LbmServerOptions(N.PREC[precision], int(tile[0]), int(tile[1]), int(arena_bytes),
                                 float(hbm_fraction), int(max_resident), int(max_queued), 1 if use_graph else 0,
                                 int(status_poll_steps), int(fast_lane_steps))
        h = C.c_void_p()
        N.check(L.lbm_server_create(C.byref(opt), C.byref(h)), "lbm_server_create")
        self._h = h
        self.precision = precision
        self._shapes = {}

    def close(self):
        if getattr(self, "_h", None):
            N.lib().lbm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, case):
        """Queue one solve; returns its request id."""
        b = _CaseBuffers(case)
        rid = C.c_longlong()
        N.check(N.lib().lbm_server_submit(self._h, C.byref(b.cfg), C.byref(b.ini), C.byref(rid)),
                "lbm_server_submit")
        self._shapes[rid.value] = (b.nx, b.ny)
        return rid.value

    def wait(self, rid, timeout=-1.0):
        """True when the request finished, False when the timeout ran out."""
        code = N.lib().lbm_server_wait(self._h, int(rid), float(timeout))
        if code == N.LBM_ERR_TIMEOUT:
            return False
        N.check(code, "lbm_server_wait")
        return True

    def wait_any(self, timeout=-1.0):
        """Id of the next finished request, or None when the timeout ran out."""
        rid = C.c_longlong()
        code = N.lib().lbm_server_wait_any(self._h, float(timeout), C.byref(rid))
        if code == N.LBM_ERR_TIMEOUT:
            return None
        N.check(code, "lbm_server_wait_any")
        return rid.value

    def info(self, rid):
        i = N.LbmRequestInfo()
        N.check(N.lib().lbm_server_info(self._h, int(rid), C.byref(i)), "lbm_server_info")
        return {name: getattr(i, name) for name, _ in N.LbmRequestInfo._fields_}

    def result(self, rid):
        """(status, fields) of a finished request; fields as ``Solver.macro``."""
        nx, ny = self._shapes[rid]
        out = {k: np.empty(nx * ny) for k in ("rho", "ux", "uy", "T", "p")}
        code = N.lib().lbm_server_result(self._h, int(rid), *[_d(out[k]) for k in ("rho", "ux", "uy", "T", "p")])
        if code in (N.LBM_ERR_BUSY, N.LBM_ERR_NOT_FOUND, N.LBM_ERR_INVALID):
            N.check(code, "lbm_server_result")
        return code, {k: v.reshape(nx, ny) for k, v in out.items()}

    def cancel(self, rid):
        N.check(N.lib().lbm_server_cancel(self._h, int(rid)), "lbm_server_cancel")

    def release(self, rid):
        N.check(N.lib().lbm_server_release(self._h, int(rid)), "lbm_server_release")
        self._shapes.pop(rid, None)

    def stats(self):
        s = N.LbmServerStats()
        N.check(N.lib().lbm_server_get_stats(self._h, C.byref(s)), "lbm_server_get_stats")
        return {name: getattr(s, name) for name, _ in N.LbmServerStats._fields_}
