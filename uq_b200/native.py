"""ctypes binding of the C ABI in include/uq_lbm.h (uq_b200/lib/libuqlbm.so).

The shared library is the product: there is no Python or CPU fallback.
``lib()`` raises if the library is missing or a symbol is absent.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libuqlbm.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

LBM_OK = 0
LBM_ERR_EQUILIBRIUM = 1
LBM_ERR_INVALID = 2
LBM_ERR_CUDA = 3
LBM_ERR_NOMEM = 4
LBM_ERR_NONFINITE = 5
LBM_ERR_BUSY = 6
LBM_ERR_NOT_FOUND = 7
LBM_ERR_TIMEOUT = 8
LBM_ERR_CANCELLED = 9
STATUS_NAMES = {0: "ok", 1: "equilibrium", 2: "invalid", 3: "cuda", 4: "nomem", 5: "nonfinite",
                6: "busy", 7: "not_found", 8: "timeout", 9: "cancelled"}
LBM_REQ_QUEUED, LBM_REQ_RESIDENT, LBM_REQ_DONE = 0, 1, 2

PREC = {"f64": 0, "f32": 1}


class LbmConfig(C.Structure):
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


class LbmInit(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("numProps", C.c_int),
        ("bndArray", _ip), ("cellType", _ip),
        ("density", _dp), ("pressure", _dp), ("temp", _dp), ("velocityX", _dp), ("velocityY", _dp),
    ]


class LbmInfo(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("step", C.c_int), ("nsteps", C.c_int),
        ("dt", C.c_double), ("tstep", C.c_double), ("residual", C.c_double),
        ("precision", C.c_int), ("rkmethod", C.c_int), ("fmethod", C.c_int),
        ("device_bytes", C.c_size_t),
    ]


class LbmBatchOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("tile_x", C.c_int), ("tile_y", C.c_int), ("use_graph", C.c_int)]


class LbmServerOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("tile_x", C.c_int), ("tile_y", C.c_int), ("arena_bytes", C.c_size_t),
                ("hbm_fraction", C.c_double), ("max_resident", C.c_int), ("max_queued", C.c_int),
                ("use_graph", C.c_int), ("status_poll_steps", C.c_int), ("fast_lane_steps", C.c_int)]


class LbmRequestInfo(C.Structure):
    _fields_ = [("id", C.c_longlong), ("Nx", C.c_int), ("Ny", C.c_int), ("steps_total", C.c_int),
                ("steps_done", C.c_int), ("state", C.c_int), ("status", C.c_int), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double), ("step_admit", C.c_longlong),
                ("step_done", C.c_longlong)]


class LbmServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("admitted", C.c_longlong), ("completed", C.c_longlong),
                ("failed", C.c_longlong), ("cancelled", C.c_longlong), ("steps", C.c_longlong),
                ("lattice_updates", C.c_longlong), ("repacks", C.c_longlong), ("compactions", C.c_longlong),
                ("graph_captures", C.c_longlong), ("resident", C.c_int), ("queued", C.c_int),
                ("arena_nodes", C.c_longlong), ("arena_nodes_used", C.c_longlong), ("arena_bytes", C.c_size_t),
                ("busy_seconds", C.c_double), ("uptime_seconds", C.c_double),
                ("boundary_seconds", C.c_double), ("capture_seconds", C.c_double),
                ("steps_eager", C.c_longlong), ("steps_graph", C.c_longlong)]


# name -> (restype, argtypes); every function include/uq_lbm.h declares
SIGNATURES = {
    "lbm_create": (C.c_int, [C.POINTER(LbmConfig), C.POINTER(LbmInit), C.c_int, C.POINTER(C.c_void_p)]),
    "lbm_step": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
    "lbm_run": (C.c_int, [C.c_void_p, C.c_int, _ip, _dp, C.c_int]),
    "lbm_get_macro": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "lbm_get_dist": (C.c_int, [C.c_void_p, _dp, _dp]),
    "lbm_set_dist": (C.c_int, [C.c_void_p, _dp, _dp]),
    "lbm_get_info": (C.c_int, [C.c_void_p, C.POINTER(LbmInfo)]),
    "lbm_stream": (C.c_void_p, [C.c_void_p]),
    "lbm_destroy": (None, [C.c_void_p]),
    "lbm_last_error": (C.c_char_p, []),
    "lbm_batch_create": (C.c_int, [C.c_int, C.POINTER(LbmConfig), C.POINTER(LbmInit),
                                   C.POINTER(LbmBatchOptions), C.POINTER(C.c_void_p)]),
    "lbm_batch_step": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "lbm_batch_status": (C.c_int, [C.c_void_p, _ip]),
    "lbm_batch_residuals": (C.c_int, [C.c_void_p, _dp]),
    "lbm_batch_get_macro": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]),
    "lbm_batch_get_dist": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "lbm_batch_set_dist": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "lbm_batch_set_macro": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]),
    "lbm_batch_set_macro_all": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "lbm_batch_get_macro_all": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "lbm_batch_profile": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "lbm_batch_launches_per_step": (C.c_int, [C.c_void_p, C.c_int]),
    "lbm_batch_autotune": (C.c_int, [C.c_void_p, _ip, C.c_int, C.c_int, _ip, _dp]),
    "lbm_batch_nodes": (C.c_longlong, [C.c_void_p]),
    "lbm_batch_stream": (C.c_void_p, [C.c_void_p]),
    "lbm_batch_destroy": (None, [C.c_void_p]),
    "lbm_server_create": (C.c_int, [C.POINTER(LbmServerOptions), C.POINTER(C.c_void_p)]),
    "lbm_server_submit": (C.c_int, [C.c_void_p, C.POINTER(LbmConfig), C.POINTER(LbmInit), C.POINTER(C.c_longlong)]),
    "lbm_server_wait": (C.c_int, [C.c_void_p, C.c_longlong, C.c_double]),
    "lbm_server_wait_any": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_longlong)]),
    "lbm_server_info": (C.c_int, [C.c_void_p, C.c_longlong, C.POINTER(LbmRequestInfo)]),
    "lbm_server_result": (C.c_int, [C.c_void_p, C.c_longlong, _dp, _dp, _dp, _dp, _dp]),
    "lbm_server_cancel": (C.c_int, [C.c_void_p, C.c_longlong]),
    "lbm_server_release": (C.c_int, [C.c_void_p, C.c_longlong]),
    "lbm_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(LbmServerStats)]),
    "lbm_server_destroy": (None, [C.c_void_p]),
    "lbm_selftest_bounded_wait": (C.c_int, [C.c_int]),
    "lbm_mat_read_case": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "lbm_mat_case_get": (C.c_int, [C.c_void_p, C.POINTER(LbmConfig), C.POINTER(LbmInit)]),
    "lbm_mat_case_free": (None, [C.c_void_p]),
    "lbm_create_from_mat": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "lbm_mat_write_fields": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double,
                                       C.c_double, C.c_double, _dp, _dp, _dp, _dp]),
    "lbm_write_mat": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "lbm_mat_read_dist": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp, _dp, _dp]),
    "lbm_restore_mat": (C.c_int, [C.c_void_p, C.c_char_p]),
    "lbm_hdf5_write_fields": (C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_double, _dp, C.c_int, _dp, C.c_int, _dp, _dp]),
    "lbm_write_hdf5": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "lbm_step_noalloc": (C.c_int, [C.POINTER(LbmConfig), C.c_int, C.c_int, _ip, C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_void_p]),
}

_lib = None


class LbmError(RuntimeError):
    def __init__(self, code, where):
        msg = lib().lbm_last_error().decode(errors="replace") if _lib is not None else ""
        super().__init__("%s failed: %s (%s)" % (where, STATUS_NAMES.get(code, code), msg))
        self.code = code


def lib():
    """Load libuqlbm.so; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            raise RuntimeError("CUDA extension %s is missing: run `python -m uq_b200.build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code, where):
    if code != LBM_OK:
        raise LbmError(code, where)
