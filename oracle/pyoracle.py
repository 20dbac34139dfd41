"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes access to the CPU checker.

Two libraries are wrapped:

* ``oracle/liboracle.so`` -- the table-driven C restatement of the
  reference's chemistry (mech_eval.c, reactor.c);
* ``oracle/_ref/libref_<mech>.so`` -- the reference's own generated
  ``mechanism.H`` kernels compiled on the host (ref_wrap.cpp).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module, always as the checker.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_LP = C.POINTER(C.c_long)
_lib = None
_ref = {}


def _p(a):
    return a.ctypes.data_as(_DP)


def build():
    subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True)
    subprocess.run(["bash", os.path.join(HERE, "build_ref.sh")], check=True)


class Options(C.Structure):
    _fields_ = [
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("max_order", C.c_int),
        ("max_steps", C.c_long),
        ("max_nls_iters", C.c_int),
        ("max_err_fails", C.c_int),
        ("jac_eval_freq", C.c_int),
        ("use_ref_kernels", C.c_int),
        ("rk64_nsubsteps_guess", C.c_int),
        ("rk64_nsubsteps_min", C.c_int),
        ("rk64_nsubsteps_max", C.c_int),
        ("typ_vals", _DP),
        ("eos", C.c_int),
        ("rhs_noise_seed", C.c_ulonglong),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("nsteps", C.c_long),
        ("nfe", C.c_long),
        ("nje", C.c_long),
        ("nsetups", C.c_long),
        ("nni", C.c_long),
        ("ncfn", C.c_long),
        ("netf", C.c_long),
        ("status", C.c_int),
        ("last_order", C.c_int),
        ("last_h", C.c_double),
    ]


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True)
        L = C.CDLL(path)
        L.ppo_mech.restype = C.c_void_p
        L.ppo_mech.argtypes = [C.c_char_p]
        L.ppo_nsp.argtypes = [C.c_char_p]
        L.ppo_nqss.argtypes = [C.c_char_p]
        L.ppo_qss_concentrations.argtypes = [C.c_void_p, _DP, C.c_double, _DP]
        L.ppo_qss_system.argtypes = [C.c_void_p, _DP, C.c_double, _DP]
        for fn in ("ppo_cv_R", "ppo_cp_R", "ppo_dcvpRdT", "ppo_species_internal_energy",
                   "ppo_species_enthalpy", "ppo_gibbs", "ppo_ckums", "ppo_ckhms"):
            getattr(L, fn).argtypes = [C.c_void_p, C.c_double, _DP]
        for fn in ("ppo_ckubms", "ppo_ckhbms", "ppo_ckcvbs", "ppo_ckcpbs"):
            getattr(L, fn).argtypes = [C.c_void_p, C.c_double, _DP]
            getattr(L, fn).restype = C.c_double
        L.ppo_ckrhoy.argtypes = [C.c_void_p, C.c_double, C.c_double, _DP]
        L.ppo_ckrhoy.restype = C.c_double
        L.ppo_get_t_given_ey.argtypes = [C.c_void_p, C.c_double, _DP, _DP]
        L.ppo_get_t_given_hy.argtypes = [C.c_void_p, C.c_double, _DP, _DP]
        L.ppo_production_rate.argtypes = [C.c_void_p, _DP, _DP, C.c_double]
        L.ppo_production_rate_abs.argtypes = [C.c_void_p, _DP, _DP, C.c_double]
        L.ppo_ckwc.argtypes = [C.c_void_p, C.c_double, _DP, _DP]
        L.ppo_ajacobian.argtypes = [C.c_void_p, _DP, _DP, C.c_double, C.c_int]
        L.ppo_dwdot.argtypes = [C.c_void_p, _DP, _DP, C.c_double, C.c_int]
        L.ppo_reactor_rhs.argtypes = [C.c_void_p, C.c_int, C.c_double, _DP, _DP, C.c_double,
                                      C.c_double, _DP]
        L.ppo_reactor_rhs.restype = C.c_double
        L.ppo_reactor_jac.argtypes = [C.c_void_p, C.c_int, _DP, _DP]
        L.ppo_default_options.argtypes = [C.POINTER(Options)]
        L.ppo_react_arkode.argtypes = [C.c_void_p, C.c_int, C.POINTER(ArkOptions), _DP, _DP, _DP, _DP, _IP,
                                       C.c_double, C.c_int, C.c_int, C.POINTER(ArkStats)]
        L.ppo_bdf_cell.argtypes = [C.c_void_p, C.c_int, C.POINTER(Options), _DP, _DP, C.c_double,
                                   C.c_double, C.c_double, C.POINTER(Stats)]
        L.ppo_rk64_cell.argtypes = [C.c_void_p, C.c_int, C.POINTER(Options), _DP, _DP, C.c_double,
                                    C.c_double, C.c_double]
        L.ppo_react_flat.argtypes = [C.c_char_p, C.c_int, C.POINTER(Options), C.c_int, _DP, _DP,
                                     _DP, _DP, C.c_double, C.c_int, C.c_int, _LP, _IP]
        L.ppo_react_flat_tables.argtypes = [C.c_void_p, C.c_int, C.POINTER(Options), C.c_int, _DP, _DP,
                                            _DP, _DP, C.c_double, C.c_int, C.c_int, _LP, _IP]
        L.ppo_react_flat_stats.argtypes = [C.c_char_p, C.c_int, C.POINTER(Options), C.c_int, _DP, _DP,
                                           _DP, _DP, C.c_double, C.c_int, C.c_int, _IP, _LP]
        L.ppo_mech_with_arrhenius.argtypes = [C.c_char_p, _DP, _DP, _DP]
        L.ppo_mech_with_arrhenius.restype = C.c_void_p
        L.ppo_mech_free.argtypes = [C.c_void_p]
        L.ppo_load_ref.argtypes = [C.c_char_p, C.c_char_p]
        L.ppo_species_name.argtypes = [C.c_char_p, C.c_int]
        L.ppo_species_name.restype = C.c_char_p
        L.ppo_mw.argtypes = [C.c_char_p, _DP]
        _lib = L
    return _lib


def reference_root():
    """The PelePhysics tree the reference kernels were built from: the
    PPB_REFERENCE_ROOT environment variable, else the root oracle/build_ref.sh
    recorded in _ref/reference_root; None when neither names an existing
    tree (e.g. on a machine that only has the prebuilt libraries)."""
    cands = [os.environ.get("PPB_REFERENCE_ROOT")]
    rec = os.path.join(HERE, "_ref", "reference_root")
    if os.path.exists(rec):
        cands.append(open(rec).read().strip())
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "Mechanisms")):
            return c
    return None


def ref_path(mech):
    return os.path.join(HERE, "_ref", f"libref_{mech}.so")


def have_ref(mech):
    return os.path.exists(ref_path(mech))


class Mech:
    """Table-driven oracle for one mechanism."""

    def __init__(self, name):
        self.name = name
        self.L = lib()
        self.M = self.L.ppo_mech(name.encode())
        if not self.M:
            raise KeyError(name)
        self.nsp = self.L.ppo_nsp(name.encode())
        self.nqss = self.L.ppo_nqss(name.encode())

    def qss_concentrations(self, sc, T):
        out = np.zeros(self.nqss)
        self.L.ppo_qss_concentrations(self.M, _p(np.ascontiguousarray(sc, float)), float(T), _p(out))
        return out

    def qss_system(self, sc, T):
        """The QSS balance system [I + C | -P/D], nqss x (nqss + 1)."""
        out = np.zeros(self.nqss * (self.nqss + 1))
        self.L.ppo_qss_system(self.M, _p(np.ascontiguousarray(sc, float)), float(T), _p(out))
        return out.reshape(self.nqss, self.nqss + 1)

    def species(self):
        return [self.L.ppo_species_name(self.name.encode(), k).decode() for k in range(self.nsp)]

    def mw(self):
        a = np.zeros(self.nsp)
        self.L.ppo_mw(self.name.encode(), _p(a))
        return a

    def _vecT(self, fn, T):
        out = np.zeros(self.nsp)
        getattr(self.L, fn)(self.M, float(T), _p(out))
        return out

    def gibbs(self, T):
        return self._vecT("ppo_gibbs", T)

    def cv_R(self, T):
        return self._vecT("ppo_cv_R", T)

    def cp_R(self, T):
        return self._vecT("ppo_cp_R", T)

    def species_internal_energy(self, T):
        return self._vecT("ppo_species_internal_energy", T)

    def species_enthalpy(self, T):
        return self._vecT("ppo_species_enthalpy", T)

    def ckums(self, T):
        return self._vecT("ppo_ckums", T)

    def ckhms(self, T):
        return self._vecT("ppo_ckhms", T)

    def ckubms(self, T, y):
        y = np.ascontiguousarray(y, float)
        return self.L.ppo_ckubms(self.M, float(T), _p(y))

    def ckhbms(self, T, y):
        y = np.ascontiguousarray(y, float)
        return self.L.ppo_ckhbms(self.M, float(T), _p(y))

    def ckcvbs(self, T, y):
        y = np.ascontiguousarray(y, float)
        return self.L.ppo_ckcvbs(self.M, float(T), _p(y))

    def ckcpbs(self, T, y):
        y = np.ascontiguousarray(y, float)
        return self.L.ppo_ckcpbs(self.M, float(T), _p(y))

    def ckrhoy(self, P, T, y):
        y = np.ascontiguousarray(y, float)
        return self.L.ppo_ckrhoy(self.M, float(P), float(T), _p(y))

    def t_given_ey(self, e, y, T0):
        y = np.ascontiguousarray(y, float)
        t = np.array([T0], float)
        ierr = self.L.ppo_get_t_given_ey(self.M, float(e), _p(y), _p(t))
        return t[0], ierr

    def t_given_hy(self, h, y, T0):
        y = np.ascontiguousarray(y, float)
        t = np.array([T0], float)
        ierr = self.L.ppo_get_t_given_hy(self.M, float(h), _p(y), _p(t))
        return t[0], ierr

    def production_rate(self, sc, T):
        sc = np.ascontiguousarray(sc, float)
        w = np.zeros(self.nsp)
        self.L.ppo_production_rate(self.M, _p(w), _p(sc), float(T))
        return w

    def production_rate_abs(self, sc, T):
        sc = np.ascontiguousarray(sc, float)
        w = np.zeros(self.nsp)
        self.L.ppo_production_rate_abs(self.M, _p(w), _p(sc), float(T))
        return w

    def ajacobian(self, sc, T, consP):
        sc = np.ascontiguousarray(sc, float)
        J = np.zeros((self.nsp + 1) ** 2)
        self.L.ppo_ajacobian(self.M, _p(J), _p(sc), float(T), int(consP))
        return J

    def reactor_rhs(self, reactor_type, t, y, rhoe, rhoesrc, src):
        y = np.ascontiguousarray(y, float)
        src = np.ascontiguousarray(src, float)
        f = np.zeros(self.nsp + 1)
        T = self.L.ppo_reactor_rhs(self.M, reactor_type, float(t), _p(y), _p(f), float(rhoe),
                                   float(rhoesrc), _p(src))
        return f, T

    def reactor_jac(self, reactor_type, y):
        y = np.ascontiguousarray(y, float)
        J = np.zeros((self.nsp + 1) ** 2)
        self.L.ppo_reactor_jac(self.M, reactor_type, _p(y), _p(J))
        return J.reshape(self.nsp + 1, self.nsp + 1)  # [col][row]


def options(**kw):
    o = Options()
    lib().ppo_default_options(C.byref(o))
    typ = kw.pop("typ_vals", None)
    for k, v in kw.items():
        setattr(o, k, v)
    if typ is not None:
        arr = np.ascontiguousarray(typ, float)
        o._typ = arr
        o.typ_vals = _p(arr)
    return o


def bdf_cell(mech, reactor_type, y, src, rhoe, rhoesrc, dt, **kw):
    M = Mech(mech)
    o = options(**kw)
    if o.use_ref_kernels:
        load_ref(mech)
    y = np.array(y, float)
    src = np.ascontiguousarray(src, float)
    st = Stats()
    flag = M.L.ppo_bdf_cell(M.M, reactor_type, C.byref(o), _p(y), _p(src), float(rhoe),
                            float(rhoesrc), float(dt), C.byref(st))
    return y, flag, st


def rk64_cell(mech, reactor_type, y, src, rhoe, rhoesrc, dt, **kw):
    M = Mech(mech)
    o = options(**kw)
    if o.use_ref_kernels:
        load_ref(mech)
    y = np.array(y, float)
    src = np.ascontiguousarray(src, float)
    n = M.L.ppo_rk64_cell(M.M, reactor_type, C.byref(o), _p(y), _p(src), float(rhoe),
                          float(rhoesrc), float(dt))
    return y, n


def react_flat(mech, reactor_type, rY, rYsrc, rX, rX_src, dt, method=0, nthreads=0, **kw):
    """Per-cell CPU integration of YCOrder arrays (modified in place)."""
    o = options(**kw)
    if o.use_ref_kernels:
        load_ref(mech)
    ncells = rX.shape[0]
    nfe = np.zeros(ncells, dtype=np.int64)
    st = np.zeros(ncells, dtype=np.int32)
    flag = lib().ppo_react_flat(mech.encode(), reactor_type, C.byref(o), method, _p(rY), _p(rYsrc),
                                _p(rX), _p(rX_src), float(dt), ncells, nthreads,
                                nfe.ctypes.data_as(_LP), st.ctypes.data_as(_IP))
    return flag, nfe, st


def react_flat_stats(mech, reactor_type, rY, rYsrc, rX, rX_src, dt, method=0, nthreads=0, **kw):
    """react_flat with the per-cell integrator counters: returns (flag,
    status[ncells], stats[ncells, 7]) with columns steps, RHS evaluations,
    Jacobian evaluations, factorisations, Newton iterations, error-test
    failures, convergence failures."""
    o = options(**kw)
    if o.use_ref_kernels:
        load_ref(mech)
    ncells = rX.shape[0]
    st = np.zeros(ncells, dtype=np.int32)
    stats = np.zeros((ncells, 7), dtype=np.int64)
    flag = lib().ppo_react_flat_stats(mech.encode(), reactor_type, C.byref(o), method, _p(rY), _p(rYsrc),
                                      _p(rX), _p(rX_src), float(dt), ncells, nthreads,
                                      st.ctypes.data_as(_IP), stats.ctypes.data_as(_LP))
    return flag, st, stats


class _MechHead(C.Structure):
    """Leading fields of PPBMechTables (mech_tables.h), up to rx_EaR."""

    _fields_ = [("name", C.c_char_p), ("nsp", C.c_int), ("nrxn", C.c_int), ("species", C.c_void_p)] + [
        (f, C.c_void_p) for f in ("mw", "imw", "tmid", "th_cv", "th_cp", "th_dcp", "th_u", "th_h", "th_g",
                                  "rx_orig", "rx_kind", "rx_rev")
    ] + [("rx_A", _DP), ("rx_beta", _DP), ("rx_EaR", _DP)]


def arrhenius(mech):
    """The mechanism tables' forward Arrhenius parameters (A SI, beta, Ea/R K)."""
    M = Mech(mech).M
    t = C.cast(C.c_void_p(M), C.POINTER(_MechHead)).contents
    R = t.nrxn
    A = np.ctypeslib.as_array(t.rx_A, shape=(R,)).copy()
    b = np.ctypeslib.as_array(t.rx_beta, shape=(R,)).copy()
    e = np.ctypeslib.as_array(t.rx_EaR, shape=(R,)).copy()
    return A, b, e


def react_flat_arrhenius(mech, A, beta, EaR, reactor_type, rY, rYsrc, rX, rX_src, dt, nthreads=0, **kw):
    """react_flat (BDF, table-driven kernels) with replaced Arrhenius parameters."""
    kw["use_ref_kernels"] = 0
    o = options(**kw)
    A = np.ascontiguousarray(A, float)
    beta = np.ascontiguousarray(beta, float)
    EaR = np.ascontiguousarray(EaR, float)
    L = lib()
    M = L.ppo_mech_with_arrhenius(mech.encode(), _p(A), _p(beta), _p(EaR))
    if not M:
        raise RuntimeError("ppo_mech_with_arrhenius failed")
    try:
        ncells = rX.shape[0]
        nfe = np.zeros(ncells, dtype=np.int64)
        st = np.zeros(ncells, dtype=np.int32)
        flag = L.ppo_react_flat_tables(M, reactor_type, C.byref(o), 0, _p(rY), _p(rYsrc), _p(rX), _p(rX_src),
                                       float(dt), ncells, nthreads, nfe.ctypes.data_as(_LP),
                                       st.ctypes.data_as(_IP))
    finally:
        L.ppo_mech_free(M)
    return flag, nfe, st


class ArkOptions(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("rk_method", C.c_int), ("rk_controller", C.c_int),
                ("max_steps", C.c_long), ("typ_vals_atol", _DP)]


class ArkStats(C.Structure):
    _fields_ = [("t", C.c_double), ("h", C.c_double), ("nst", C.c_long), ("nfe", C.c_long), ("netf", C.c_long),
                ("status", C.c_int)]


def react_arkode(mech, reactor_type, rY, rYsrc, rX, rX_src, dt, rtol=1e-6, atol=1e-10, rk_method=40,
                 rk_controller=0, max_steps=500, mask=None, atolv=None, nthreads=0):
    """ReactorArkode restatement: the batch as one explicit embedded RK
    integration (YCOrder arrays modified in place, rX advanced by the time
    reached).  Returns (status, dict of t, h, nst, nfe, netf)."""
    L = lib()
    o = ArkOptions(float(rtol), float(atol), int(rk_method), int(rk_controller), int(max_steps), None)
    if atolv is not None:
        atolv = np.ascontiguousarray(atolv, float)
        o.typ_vals_atol = _p(atolv)
    ncells = rX.shape[0]
    mk = None if mask is None else np.ascontiguousarray(mask, np.int32)
    st = ArkStats()
    flag = L.ppo_react_arkode(C.c_void_p(Mech(mech).M), reactor_type, C.byref(o), _p(rY), _p(rYsrc), _p(rX),
                              _p(rX_src), None if mk is None else mk.ctypes.data_as(_IP), float(dt), ncells,
                              nthreads, C.byref(st))
    return flag, {"t": st.t, "h": st.h, "nst": st.nst, "nfe": st.nfe, "netf": st.netf}


def load_ref(mech):
    rc = lib().ppo_load_ref(mech.encode(), ref_path(mech).encode())
    if rc != 0:
        raise RuntimeError(f"cannot load reference kernels for {mech}: {rc}")


class Ref:
    """The reference's own compiled mechanism kernels (oracle/_ref)."""

    def __init__(self, mech):
        if mech in _ref:
            self.L = _ref[mech]
        else:
            path = ref_path(mech)
            if not os.path.exists(path):
                raise FileNotFoundError(path)
            L = C.CDLL(path)
            for fn in ("ref_productionRate",):
                getattr(L, fn).argtypes = [_DP, _DP, C.c_double]
            L.ref_CKWC.argtypes = [C.c_double, _DP, _DP]
            L.ref_aJacobian.argtypes = [_DP, _DP, C.c_double, C.c_int]
            L.ref_DWDOT.argtypes = [_DP, _DP, C.c_double, C.c_int]
            for fn in ("ref_gibbs", "ref_speciesInternalEnergy", "ref_speciesEnthalpy", "ref_cv_R",
                       "ref_cp_R", "ref_dcvpRdT", "ref_CKUMS", "ref_CKHMS"):
                getattr(L, fn).argtypes = [_DP, C.c_double] if fn not in ("ref_CKUMS", "ref_CKHMS") \
                    else [C.c_double, _DP]
            for fn in ("ref_CKUBMS", "ref_CKHBMS", "ref_CKCVBS", "ref_CKCPBS"):
                getattr(L, fn).argtypes = [C.c_double, _DP]
                getattr(L, fn).restype = C.c_double
            L.ref_CKRHOY.argtypes = [C.c_double, C.c_double, _DP]
            L.ref_CKRHOY.restype = C.c_double
            L.ref_GET_T_GIVEN_EY.argtypes = [C.c_double, _DP, _DP]
            L.ref_GET_T_GIVEN_HY.argtypes = [C.c_double, _DP, _DP]
            L.ref_reactor_rhs.argtypes = [C.c_int, C.c_double, _DP, _DP, C.c_double, C.c_double, _DP]
            L.ref_reactor_rhs.restype = C.c_double
            L.ref_reactor_jac.argtypes = [C.c_int, _DP, _DP]
            L.ref_mw.argtypes = [_DP]
            L.ref_imw.argtypes = [_DP]
            _ref[mech] = L
            self.L = L
        self.nsp = self.L.ref_nsp()

    def mw(self):
        a = np.zeros(self.nsp)
        self.L.ref_mw(_p(a))
        return a

    def imw(self):
        a = np.zeros(self.nsp)
        self.L.ref_imw(_p(a))
        return a

    def production_rate(self, sc, T):
        sc = np.ascontiguousarray(sc, float)
        w = np.zeros(self.nsp)
        self.L.ref_productionRate(_p(w), _p(sc), float(T))
        return w

    def qss_concentrations(self, sc, T, nqss):
        """A QSS mechanism's steady-state concentrations (SI) at (sc, T)."""
        self.L.ref_sc_qss.argtypes = [_DP, _DP, C.c_double]
        out = np.zeros(64)
        self.L.ref_sc_qss(_p(out), _p(np.ascontiguousarray(sc, float)), float(T))
        return out[:nqss]

    def ajacobian(self, sc, T, consP):
        sc = np.ascontiguousarray(sc, float)
        J = np.zeros((self.nsp + 1) ** 2)
        self.L.ref_aJacobian(_p(J), _p(sc), float(T), int(consP))
        return J

    def vecT(self, fn, T):
        out = np.zeros(self.nsp)
        getattr(self.L, fn)(_p(out), float(T))
        return out

    def gibbs(self, T):
        return self.vecT("ref_gibbs", T)

    def species_internal_energy(self, T):
        return self.vecT("ref_speciesInternalEnergy", T)

    def species_enthalpy(self, T):
        return self.vecT("ref_speciesEnthalpy", T)

    def cv_R(self, T):
        return self.vecT("ref_cv_R", T)

    def cp_R(self, T):
        return self.vecT("ref_cp_R", T)

    def ckums(self, T):
        out = np.zeros(self.nsp)
        self.L.ref_CKUMS(float(T), _p(out))
        return out

    def ckhms(self, T):
        out = np.zeros(self.nsp)
        self.L.ref_CKHMS(float(T), _p(out))
        return out

    def ckubms(self, T, y):
        return self.L.ref_CKUBMS(float(T), _p(np.ascontiguousarray(y, float)))

    def ckhbms(self, T, y):
        return self.L.ref_CKHBMS(float(T), _p(np.ascontiguousarray(y, float)))

    def ckcvbs(self, T, y):
        return self.L.ref_CKCVBS(float(T), _p(np.ascontiguousarray(y, float)))

    def ckcpbs(self, T, y):
        return self.L.ref_CKCPBS(float(T), _p(np.ascontiguousarray(y, float)))

    def ckrhoy(self, P, T, y):
        return self.L.ref_CKRHOY(float(P), float(T), _p(np.ascontiguousarray(y, float)))

    def t_given_ey(self, e, y, T0):
        t = np.array([T0], float)
        ierr = self.L.ref_GET_T_GIVEN_EY(float(e), _p(np.ascontiguousarray(y, float)), _p(t))
        return t[0], ierr

    def t_given_hy(self, h, y, T0):
        t = np.array([T0], float)
        ierr = self.L.ref_GET_T_GIVEN_HY(float(h), _p(np.ascontiguousarray(y, float)), _p(t))
        return t[0], ierr

    def reactor_rhs(self, reactor_type, t, y, rhoe, rhoesrc, src):
        y = np.ascontiguousarray(y, float)
        f = np.zeros(self.nsp + 1)
        T = self.L.ref_reactor_rhs(reactor_type, float(t), _p(y), _p(f), float(rhoe),
                                   float(rhoesrc), _p(np.ascontiguousarray(src, float)))
        return f, T

    def reactor_jac(self, reactor_type, y):
        J = np.zeros((self.nsp + 1) ** 2)
        self.L.ref_reactor_jac(reactor_type, _p(np.ascontiguousarray(y, float)), _p(J))
        return J.reshape(self.nsp + 1, self.nsp + 1)


# ---------------------------------------------------------------- transport
TR_XI, TR_MU, TR_LAM, TR_DIAG, TR_CHI = 1, 2, 4, 8, 16
TR_ALL = TR_XI | TR_MU | TR_LAM | TR_DIAG | TR_CHI
_reftr = {}


def _tr_call(fn, flags, T, rho, Y):
    N = Y.shape[-1]
    D, chi = np.zeros(N), np.zeros(N)
    mu, xi, lam = C.c_double(), C.c_double(), C.c_double()
    y = np.ascontiguousarray(Y, float)
    fn(int(flags), float(T), float(rho), _p(y), _p(D), _p(chi), C.byref(mu), C.byref(xi), C.byref(lam))
    return D, chi, mu.value, xi.value, lam.value


def transport(mech, flags, T, rho, Y):
    """Mixture-averaged transport (Simple.H restatement) at one point:
    (Ddiag[N], chi[N], mu, xi, lam); see oracle.h for the flags."""
    L = lib()
    if not getattr(L, "_tr_set", False):
        L.ppo_transport.argtypes = [C.c_char_p, C.c_int, C.c_double, C.c_double, _DP, _DP, _DP, _DP, _DP, _DP]
        L._tr_set = True
    fn = lambda *a: L.ppo_transport(mech.encode(), *a)  # noqa: E731
    return _tr_call(fn, flags, T, rho, Y)


def reftr_path(mech):
    return os.path.join(HERE, "_ref", f"libreftr_{mech}.so")


def ref_transport(mech, flags, T, rho, Y):
    """The reference's own compiled SimpleTransport::transport (oracle/_ref)."""
    if mech not in _reftr:
        L = C.CDLL(reftr_path(mech))
        L.reftr_transport.argtypes = [C.c_int, C.c_double, C.c_double, _DP, _DP, _DP, _DP, _DP, _DP]
        _reftr[mech] = L
    return _tr_call(_reftr[mech].reftr_transport, flags, T, rho, Y)


def transport_batch(mech, flags, T, rho, Y, nthreads=0):
    """transport() over cells (Y [n, N] cell-major), OpenMP over cells."""
    L = lib()
    L.ppo_transport_batch.argtypes = [C.c_char_p, C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, C.c_int]
    n, N = Y.shape
    T, rho, Y = (np.ascontiguousarray(a, float) for a in (T, rho, Y))
    D, chi = np.zeros((n, N)), np.zeros((n, N))
    mu, xi, lam = np.zeros(n), np.zeros(n), np.zeros(n)
    L.ppo_transport_batch(mech.encode(), int(flags), n, _p(T), _p(rho), _p(Y), _p(D), _p(chi), _p(mu), _p(xi),
                          _p(lam), int(nthreads))
    return D, chi, mu, xi, lam


# ---------------------------------------------------------------- SRK EOS
_refsrk = {}


def _srk_lib():
    L = lib()
    if not getattr(L, "_srk_set", False):
        cp = C.c_char_p
        L.ppo_srk_rey2t.argtypes = [cp, C.c_double, C.c_double, _DP, _DP]
        for fn in ("ppo_srk_rty2e", "ppo_srk_rty2cv"):
            getattr(L, fn).argtypes = [cp, C.c_double, C.c_double, _DP]
            getattr(L, fn).restype = C.c_double
        for fn in ("ppo_srk_rty2ei", "ppo_srk_rty2c", "ppo_srk_rty2wdot"):
            getattr(L, fn).argtypes = [cp, C.c_double, C.c_double, _DP, _DP]
        L.ppo_reactor_rhs_srk.argtypes = [cp, C.c_double, _DP, _DP, C.c_double, C.c_double, _DP]
        L.ppo_reactor_rhs_srk.restype = C.c_double
        L._srk_set = True
    return L


class Srk:
    """The SRK equation of state for the e-reactor: the oracle's restatement
    (ref=False) or the reference's own compiled Source/Eos/SRK.H (ref=True)."""

    def __init__(self, mech, ref=False):
        self.mech, self.ref = mech, ref
        self.N = Mech(mech).nsp
        if ref:
            if mech not in _refsrk:
                L = C.CDLL(os.path.join(HERE, "_ref", f"librefsrk_{mech}.so"))
                L.refsrk_rey2t.argtypes = [C.c_double, C.c_double, _DP, _DP]
                for fn in ("refsrk_rty2e", "refsrk_rty2cv"):
                    getattr(L, fn).argtypes = [C.c_double, C.c_double, _DP]
                    getattr(L, fn).restype = C.c_double
                for fn in ("refsrk_rty2ei", "refsrk_rty2c", "refsrk_rty2wdot"):
                    getattr(L, fn).argtypes = [C.c_double, C.c_double, _DP, _DP]
                L.refsrk_reactor_rhs.argtypes = [C.c_double, _DP, _DP, C.c_double, C.c_double, _DP]
                L.refsrk_reactor_rhs.restype = C.c_double
                _refsrk[mech] = L
            self.L = _refsrk[mech]
        else:
            self.L = _srk_lib()

    def _call(self, name, *a):
        if self.ref:
            return getattr(self.L, "refsrk_" + name)(*a)
        return getattr(self.L, "ppo_srk_" + name)(self.mech.encode(), *a)

    def rey2t(self, R, E, Y, Tguess):
        T = np.array([float(Tguess)])
        y = np.ascontiguousarray(Y, float)
        self._call("rey2t", float(R), float(E), _p(y), _p(T))
        return T[0]

    def rty2e(self, R, T, Y):
        return self._call("rty2e", float(R), float(T), _p(np.ascontiguousarray(Y, float)))

    def rty2cv(self, R, T, Y):
        return self._call("rty2cv", float(R), float(T), _p(np.ascontiguousarray(Y, float)))

    def _vec(self, name, R, T, Y):
        out = np.zeros(self.N)
        self._call(name, float(R), float(T), _p(np.ascontiguousarray(Y, float)), _p(out))
        return out

    def rty2ei(self, R, T, Y):
        return self._vec("rty2ei", R, T, Y)

    def rty2c(self, R, T, Y):
        return self._vec("rty2c", R, T, Y)

    def rty2wdot(self, R, T, Y):
        return self._vec("rty2wdot", R, T, Y)

    def reactor_rhs(self, t_rel, y, rhoe, rhoesrc, src):
        y = np.ascontiguousarray(y, float)
        ydot = np.zeros(self.N + 1)
        s = np.ascontiguousarray(src, float)
        if self.ref:
            T = self.L.refsrk_reactor_rhs(float(t_rel), _p(y), _p(ydot), float(rhoe), float(rhoesrc), _p(s))
        else:
            T = self.L.ppo_reactor_rhs_srk(self.mech.encode(), float(t_rel), _p(y), _p(ydot), float(rhoe),
                                           float(rhoesrc), _p(s))
        return ydot, T


def mass_fraction_rows(rY, N):
    """Y_k = rhoY_k / sum_j rhoY_j per YCOrder row."""
    return rY[:, :N] / rY[:, :N].sum(1, keepdims=True)


def compare_to_reference(mech, reactor_type, rY0, rYsrc, rX, rX_src, dt, y_test, y_ref, Y_atol=1e-8, k=16,
                         k_more=256, nthreads=0, T_rtol=1e-6, **opts):
    """Integration parity of y_test against the oracle's y_ref (both YCOrder,
    integrated from rY0 over dt with the options opts).

    At rtol = atol = 1e-10 the CVODE algorithm is not continuous in the
    last bits of its arithmetic on some cells: a rounding-level change of a
    right-hand side can flip an accept/reject or a Jacobian-reuse decision,
    and the cell then ends on another step sequence whose result differs by
    up to the integration error (measured on the drm19 64^3 field: 6.5e-8 in
    Y between the oracle over the reference's compiled kernels and the same
    oracle over a table-driven restatement of them, whose rates differ only
    in the order of their floating-point operations; on slowly igniting
    LiDryer cells the step count ranges over 317..417 under such changes).
    Two implementations whose rates differ in the last bit land on either
    branch.  So a cell whose mass fractions differ from y_ref by more than
    Y_atol is integrated again by the oracle k times with every
    right-hand-side value moved by at most one ulp (rhs_noise_seed 1..k): the
    same algorithm run as k implementations that differ from it in the last
    bit.  The cell passes when y_test is within Y_atol of one of those
    results, or when its distance to y_ref is within their spread around
    y_ref (the reference's own rounding-level sensitivity at that cell).  A
    cell that passes neither way after k replicas gets k_more further ones.

    The temperature is judged the same way against T_rtol (relative).

    Returns max relative T error, max abs Y error against y_ref, the cells
    above Y_atol, the worst nearest-replica distances, and the cells that pass
    neither way in Y or in T ("cells_failing")."""
    N = rY0.shape[1] - 1
    Yt = mass_fraction_rows(y_test, N)
    Yr = mass_fraction_rows(y_ref, N)
    dY = np.abs(Yt - Yr).max(1)
    dT = np.abs(y_test[:, N] - y_ref[:, N]) / np.abs(y_ref[:, N])
    over = np.nonzero((dY > Y_atol) | (dT > T_rtol))[0]
    nearest = dY.copy()
    spread = np.zeros_like(dY)
    nearest_T = dT.copy()
    spread_T = np.zeros_like(dT)
    replicas = np.zeros(dY.size, dtype=int)

    def replicate(cells, seeds):
        for seed in seeds:
            yp = np.ascontiguousarray(rY0[cells])
            react_flat(mech, reactor_type, yp, np.ascontiguousarray(rYsrc[cells]), rX[cells].copy(),
                       np.ascontiguousarray(rX_src[cells]), dt, nthreads=nthreads, rhs_noise_seed=seed, **opts)
            Yp = mass_fraction_rows(yp, N)
            nearest[cells] = np.minimum(nearest[cells], np.abs(Yp - Yt[cells]).max(1))
            spread[cells] = np.maximum(spread[cells], np.abs(Yp - Yr[cells]).max(1))
            Tr = np.abs(y_ref[cells, N])
            nearest_T[cells] = np.minimum(nearest_T[cells], np.abs(yp[:, N] - y_test[cells, N]) / Tr)
            spread_T[cells] = np.maximum(spread_T[cells], np.abs(yp[:, N] - y_ref[cells, N]) / Tr)
            replicas[cells] += 1

    def failing_cells(cells):
        ok_Y = (nearest[cells] <= Y_atol) | (dY[cells] <= spread[cells])
        ok_T = (nearest_T[cells] <= T_rtol) | (dT[cells] <= spread_T[cells])
        return cells[~(ok_Y & ok_T)]

    if over.size:
        replicate(over, range(1, k + 1))
        fail = failing_cells(over)
        if fail.size and k_more > 0:
            replicate(fail, range(k + 1, k + k_more + 1))
            fail = failing_cells(fail)
    else:
        fail = over
    return {"cells": int(rY0.shape[0]), "max_rel_T": float(dT.max()), "max_abs_Y": float(dY.max()),
            "cells_over_Y_atol": int(over.size), "Y_atol": Y_atol,
            "max_abs_Y_nearest_replica": float(nearest.max()), "max_rel_T_nearest_replica": float(nearest_T.max()),
            "max_replicas_per_cell": int(replicas.max()),
            "cells_failing": int(fail.size), "failing_cells": [int(c) for c in fail[:16]]}
