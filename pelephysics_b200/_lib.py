"""ctypes binding of the engine's C ABI (include/pelephysics_b200.h).

The shared library is built in-tree by ``pelephysics_b200.build``; loading
fails loudly when it is missing -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
# PPB_LIB selects another build of the engine library
LIB_PATH = os.environ.get("PPB_LIB", os.path.join(HERE, "libppb200.so"))
HEADER = os.path.join(os.path.dirname(HERE), "include", "pelephysics_b200.h")

PPB_E_ARG, PPB_E_CUDA, PPB_E_MECH, PPB_E_STATE, PPB_E_INTEGRATE = -1, -2, -3, -4, 1
PPB_ENGINE_PLAIN, PPB_ENGINE_TUNED = 0, 1


class Options(C.Structure):
    """ppb_options (field order and meaning as in the header)."""

    _fields_ = [
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("max_order", C.c_int),
        ("max_steps", C.c_int),
        ("max_nls_iters", C.c_int),
        ("max_err_fails", C.c_int),
        ("jac_eval_freq", C.c_int),
        ("clean_init_massfrac", C.c_int),
        ("rk64_nsubsteps_guess", C.c_int),
        ("rk64_nsubsteps_min", C.c_int),
        ("rk64_nsubsteps_max", C.c_int),
        ("verbose", C.c_int),
        ("engine", C.c_int),
        ("lu_fp32", C.c_int),
        ("refine_sweeps", C.c_int),
        ("warps_per_block", C.c_int),
        ("use_graph", C.c_int),
        ("adjoint_checkpoint_interval", C.c_int),
        ("adjoint_memory_mb", C.c_int),
        ("team_lanes", C.c_int),
        ("register_budget", C.c_int),
        ("rk_method", C.c_int),
        ("rk_controller", C.c_int),
        ("use_erkstep", C.c_int),
        ("arkode_max_steps", C.c_int),
        ("eos", C.c_int),
        ("cost_order", C.c_int),
        ("rendezvous_cycles", C.c_int),
        ("arkode_barrier_us", C.c_int),
        ("adjoint_keep_segments", C.c_int),
    ]


class Array4(C.Structure):
    _fields_ = [
        ("p", C.c_void_p),
        ("jstride", C.c_long),
        ("kstride", C.c_long),
        ("nstride", C.c_long),
        ("lo", C.c_int * 3),
        ("hi", C.c_int * 3),
        ("ncomp", C.c_int),
    ]


class Array4i(Array4):
    pass


_lib = None


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pelephysics_b200 error {code}: {msg}")
        self.code = code


def lib():
    """Load libppb200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(
            f"{LIB_PATH} is missing: build it with `python -m pelephysics_b200.build` "
            "(the engine has no CPU fallback)"
        )
    L = C.CDLL(LIB_PATH)
    vp, ip, dp, lp = C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.POINTER(C.c_long)
    dpp = C.POINTER(C.c_double)
    L.ppb_default_options.argtypes = [C.POINTER(Options)]
    L.ppb_default_options.restype = None
    L.ppb_last_error.restype = C.c_char_p
    L.ppb_mechanism_info.argtypes = [C.c_char_p, ip, ip]
    L.ppb_species_name.argtypes = [C.c_char_p, C.c_int]
    L.ppb_species_name.restype = C.c_char_p
    L.ppb_create.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(vp)]
    L.ppb_init.argtypes = [vp, C.c_int, C.c_int, C.POINTER(Options)]
    L.ppb_set_typ_vals.argtypes = [vp, dpp, C.c_int]
    L.ppb_close.argtypes = [vp]
    L.ppb_destroy.argtypes = [vp]
    L.ppb_destroy.restype = None
    L.ppb_react_flat.argtypes = [vp, dp, dp, dp, dp, dpp, dpp, C.c_int, vp, lp]
    L.ppb_react_flat_device.argtypes = [vp, dp, dp, dp, dp, dpp, dpp, C.c_int, vp, lp]
    L.ppb_react_soa_device.argtypes = [vp, dp, dp, dp, dp, C.c_int, dpp, dpp, C.c_int, vp, lp]
    L.ppb_react_box.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), Array4, Array4, Array4, Array4,
                                Array4, Array4, Array4i, dpp, dpp, vp]
    L.ppb_get_cell_status.argtypes = [vp, ip, ip, C.c_int]
    L.ppb_production_rate.argtypes = [C.c_char_p, dp, dp, dp, C.c_int, C.c_int, vp]
    L.ppb_ajacobian.argtypes = [C.c_char_p, dp, dp, C.c_int, dp, C.c_int, C.c_int, vp]
    L.ppb_t_from_energy.argtypes = [C.c_char_p, C.c_int, dp, dp, dp, C.c_int, C.c_int, vp]
    L.ppb_reactor_rhs.argtypes = [C.c_char_p, C.c_int, C.c_double, dp, dp, dp, dp, dp, C.c_int, C.c_int, vp]
    L.ppb_get_cell_stats.argtypes = [vp, ip, C.c_int]
    L.ppb_last_ncells.argtypes = [vp]
    L.ppb_flatten.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)] + [Array4] * 5 + [dp, dp, dp, dp, vp]
    L.ppb_unflatten.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)] + [Array4] * 5 + [dp, dp, dp,
                                                                                              C.c_double, vp]
    L.ppb_probe_fp64_peak.argtypes = [dpp, vp]
    L.ppb_react_flat_device_noalloc.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(Options), dp, dp, dp, dp,
                                                C.c_double, C.c_int, vp, ip]
    L.ppb_molecular_weights.argtypes = [C.c_char_p, dpp]
    L.ppb_pyt2re.argtypes = [C.c_char_p, C.c_int, dp, dp, dp, dp, dp, C.c_int, vp]
    L.ppb_get_launch_config.argtypes = [vp, ip, ip, ip, dpp]
    L.ppb_get_rendezvous_cycles.argtypes = [vp, ip]
    L.ppb_get_arrhenius.argtypes = [vp, dpp, dpp, dpp]
    L.ppb_set_arrhenius.argtypes = [vp, dpp, dpp, dpp]
    L.ppb_adjoint_flat_device.argtypes = [vp, dp, dp, dp, dp, C.c_double, C.c_int, dp, dp, dp, dp, dp, vp]
    L.ppb_tangent_flat_device.argtypes = [vp, dp, dp, dp, dp, C.c_double, C.c_int, dp, dp, dp, dp, dp, vp]
    L.ppb_rhs_exact.argtypes = [C.c_char_p, C.c_int, C.c_double, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp,
                                C.c_int, vp]
    L.ppb_transport.argtypes = [C.c_char_p, C.c_int, dp, dp, dp, C.c_int, dp, dp, dp, dp, dp, C.c_int, vp]
    L.ppb_transport_box.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)] + [Array4] * 8 + [vp]
    _lib = L
    return L


def header_functions():
    """Names of the functions include/pelephysics_b200.h declares."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ppb_[a-z0-9_]+)\s*\(", txt)))


def check(code):
    if code < 0 or code == PPB_E_INTEGRATE:
        raise EngineError(code, lib().ppb_last_error().decode())
    return code


def default_options(**kw):
    o = Options()
    lib().ppb_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


def mechanism_info(name):
    n = C.c_int()
    r = C.c_int()
    check(lib().ppb_mechanism_info(name.encode(), C.byref(n), C.byref(r)))
    return n.value, r.value


def molecular_weights(name):
    import numpy as np

    nsp, _ = mechanism_info(name)
    mw = np.zeros(nsp)
    check(lib().ppb_molecular_weights(name.encode(), mw.ctypes.data_as(C.POINTER(C.c_double))))
    return mw


def species_names(name):
    nsp, _ = mechanism_info(name)
    return [lib().ppb_species_name(name.encode(), k).decode() for k in range(nsp)]
