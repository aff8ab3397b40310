"""ctypes binding of the C ABI declared in include/lionbolt_b200.h.

The library is built in-tree (lionbolt_b200/liblionbolt_b200.so).  There is no CPU fallback:
if the shared library is missing or no CUDA device is present, every operator raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblionbolt_b200.so")

LB_OK = 0
LB_ERR_ARG = 1
LB_ERR_CUDA = 2
LB_ERR_OOM = 3
LB_ERR_CYCLE = 4
LB_ERR_TIMEOUT = 5
LB_ERR_NOCONV = 6
LB_ERR_NAN = 7
LB_ERR_STATE = 8
LB_ERR_BREAKDOWN = 9

SOLVER_SI = 0
SOLVER_GMRES = 1
SOLVER_FGMRES_ML = 2
SOLVER_FGMRES = 3

TIMER_NAMES = ("sweep", "m2d", "d2m", "krylov", "copy", "precond", "tally")

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_float_p = ctypes.POINTER(ctypes.c_float)
_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_ubyte_p = ctypes.POINTER(ctypes.c_ubyte)
_c_ll_p = ctypes.POINTER(ctypes.c_longlong)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); every symbol here is declared in include/lionbolt_b200.h
SIGNATURES = {
    "lb_version": (ctypes.c_int, []),
    "lb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "lb_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "lb_destroy": (ctypes.c_int, [_vp]),
    "lb_last_error": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int]),
    "lb_set_mesh": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_double_p, _c_int_p, _c_int_p, _c_int_p,
                                   ctypes.c_int]),
    "lb_set_quadrature": (ctypes.c_int, [_vp, ctypes.c_int, _c_double_p, _c_double_p]),
    "lb_sn_quadrature": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_double_p, _c_double_p]),
    "lb_set_xs": (ctypes.c_int, [_vp, ctypes.c_int, _c_double_p, _c_double_p]),
    "lb_get_schedule": (ctypes.c_int, [_vp, _c_int_p, _c_ubyte_p, _c_int_p, _c_int_p]),
    "lb_transport_inv": (ctypes.c_int, [_vp, _c_double_p]),
    "lb_scatter_apply": (ctypes.c_int, [_vp, _c_double_p]),
    "lb_boltzmann_matvec": (ctypes.c_int, [_vp, _c_double_p]),
    "lb_boltzmann_solve": (ctypes.c_int, [_vp, _c_double_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int, _c_int_p, _c_double_p]),
    "lb_mg_set_problem": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_double_p, _c_double_p, _c_double_p,
                                         _c_double_p, _c_double_p]),
    "lb_mg_solve": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   _c_int_p]),
    "lb_mg_get_results": (ctypes.c_int, [_vp, _c_double_p, _c_double_p]),
    "lb_get_timers": (ctypes.c_int, [_vp, _c_double_p, _c_ll_p]),
    "lb_reset_timers": (ctypes.c_int, [_vp]),
    "lb_sweep_stats": (ctypes.c_int, [_vp, _c_double_p, _c_double_p, _c_ll_p]),
    "lb_synchronize": (ctypes.c_int, [_vp]),
    "lb_probe_pipeline_timeout": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "lb_get_sweep_config": (ctypes.c_int, [_vp, _c_int_p]),
    "lb_mesh_types": (ctypes.c_int, [_vp, _c_int_p]),
    "lb_set_right_precond_diag": (ctypes.c_int, [_vp, ctypes.c_int, _c_double_p]),
    "lb_lp_set_groups": (ctypes.c_int, [_vp, ctypes.c_int, _c_int_p, _c_int_p]),
    "lb_beam_uncollided": (ctypes.c_int, [_vp, _c_double_p, _c_double_p, _c_double_p, _c_double_p, ctypes.c_double,
                                          ctypes.c_double, _c_double_p, _c_double_p]),
    "lb_lp_calibrate": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, _c_int_p, _c_int_p]),
    "lb_givens": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, _c_double_p, _c_double_p, _c_double_p]),
    "lb_cluster_info": (ctypes.c_int, [_vp, _c_int_p, _c_int_p]),
    "lb_cluster_layout": (ctypes.c_int, [_vp, _c_ll_p, _c_int_p, _c_int_p]),
    "lb_get_cluster_schedule": (ctypes.c_int, [_vp, _c_int_p, _c_int_p, _c_int_p]),
    "lb_mg_update_inputs": (ctypes.c_int, [_vp, _c_double_p, _c_double_p, _c_double_p, _c_double_p, _c_double_p]),
    "lb_mark": (ctypes.c_int, [_vp, ctypes.c_int]),
    "lb_transport_inv_noalloc": (ctypes.c_int, [_vp, ctypes.c_void_p]),
    "lb_elapsed_ms": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_double_p]),
    "lb_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "lb_batch_destroy": (ctypes.c_int, [_vp]),
    "lb_batch_last_error": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int]),
    "lb_batch_add_problem": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _c_double_p, _c_int_p, _c_int_p, _c_int_p,
                                            ctypes.c_int, ctypes.c_int, _c_double_p, _c_double_p, ctypes.c_int,
                                            ctypes.c_int, _c_double_p, _c_double_p, _c_double_p, _c_double_p,
                                            _c_double_p, _c_int_p]),
    "lb_batch_solve": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _c_int_p]),
    "lb_batch_get_results": (ctypes.c_int, [_vp, ctypes.c_int, _c_double_p, _c_double_p]),
    "lb_batch_info": (ctypes.c_int, [_vp, _c_int_p, _c_int_p, _c_double_p, _c_int_p, _c_ll_p, _c_ll_p]),
    "lb_m2d_device": (ctypes.c_int, [_vp, ctypes.c_void_p, ctypes.c_void_p]),
    "lb_d2m_device": (ctypes.c_int, [_vp, ctypes.c_void_p, ctypes.c_void_p]),
    "lb_lp_nparams": (ctypes.c_int, []),
    "lb_lp_init": (ctypes.c_int, [_vp, ctypes.c_ulonglong]),
    "lb_lp_set_weights": (ctypes.c_int, [_vp, _c_float_p]),
    "lb_lp_get_weights": (ctypes.c_int, [_vp, _c_float_p]),
    "lb_lp_enable": (ctypes.c_int, [_vp, ctypes.c_int]),
    "lb_lp_forward": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p, _c_float_p]),
    "lb_lp_apply": (ctypes.c_int, [_vp, _c_double_p, _c_double_p]),
    "lb_lp_loss_grad": (ctypes.c_int, [_vp, ctypes.c_int, _c_float_p, _c_float_p, _c_float_p, _c_double_p,
                                       _c_float_p]),
    "lb_lp_generate": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, _c_ll_p]),
    "lb_lp_num_samples": (ctypes.c_int, [_vp, _c_ll_p]),
    "lb_lp_get_samples": (ctypes.c_int, [_vp, _c_float_p, _c_float_p, _c_float_p]),
    "lb_lp_clear_samples": (ctypes.c_int, [_vp]),
    "lb_lp_train": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, _c_double_p]),
}

_lib = None


class LionboltError(RuntimeError):
    """Raised for every nonzero LB_* status (the reference stops through stophere)."""

    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


def load():
    """Load the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def dptr(a):
    return a.ctypes.data_as(_c_double_p)


def fptr(a):
    return a.ctypes.data_as(_c_float_p)


def as_f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def iptr(a):
    return a.ctypes.data_as(_c_int_p)


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def check(handle, status):
    if status != LB_OK:
        lib = load()
        buf = ctypes.create_string_buffer(512)
        if handle:
            lib.lb_last_error(handle, buf, 512)
        msg = buf.value.decode() or lib.lb_status_string(status).decode()
        raise LionboltError(status, msg)
    return status


def sn_quadrature(Ng, Nc):
    """GL x Chebyshev product quadrature of SNPrep.f90:39-76 (reference: Nc = 2 Ng)."""
    lib = load()
    k = np.zeros((Ng * Nc, 3))
    w = np.zeros(Ng * Nc)
    check(None, lib.lb_sn_quadrature(Ng, Nc, dptr(k), dptr(w)))
    return k, w


class Handle:
    """Owns one lb_handle (one device, one stream)."""

    def __init__(self, device=0):
        self.lib = load()
        h = _vp()
        st = self.lib.lb_create(int(device), ctypes.byref(h))
        if st != LB_OK:
            raise LionboltError(st, "lb_create failed: " + self.lib.lb_status_string(st).decode())
        self.h = h

    def call(self, name, *args):
        return check(self.h, getattr(self.lib, name)(self.h, *args))

    def timers(self):
        ms = np.zeros(len(TIMER_NAMES))
        n = np.zeros(len(TIMER_NAMES), dtype=np.int64)
        self.call("lb_get_timers", dptr(ms), n.ctypes.data_as(_c_ll_p))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(TIMER_NAMES)}

    def sweep_config(self):
        cfg = np.zeros(4, dtype=np.int32)
        st = self.lib.lb_get_sweep_config(self.h, iptr(cfg))
        if st != LB_OK:
            return None
        names = ("levels", "dataflow", "levels+prefetch", "element flags", "grouped directions", "cluster levels",
                 "cluster levels+type tables")
        kind = int(cfg[0])
        d = dict(schedule=names[kind] if 0 <= kind < len(names) else str(kind), threads=int(cfg[1]),
                 dirs_per_cta=int(cfg[2]), ilp=int(cfg[3]))
        if kind in (5, 6):
            d["min_ctas_per_sm"] = d.pop("dirs_per_cta")
            if d["ilp"] >= 2:
                d["schedule"] += "+element prefetch"
            if d["ilp"] == 3:
                d["schedule"] += "+previous in registers"
            if d["ilp"] >= 4:
                d["schedule"] += "+two previous in registers"
        return d

    def mesh_types(self):
        n = np.zeros(1, dtype=np.int32)
        self.call("lb_mesh_types", iptr(n))
        return int(n[0])

    def mark(self, slot):
        self.call("lb_mark", int(slot))

    def elapsed_ms(self, a, b):
        ms = np.zeros(1)
        self.call("lb_elapsed_ms", int(a), int(b), dptr(ms))
        return float(ms[0])

    def reset_timers(self):
        self.call("lb_reset_timers")

    def close(self):
        if self.h:
            self.lib.lb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
