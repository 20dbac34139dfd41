"""Python mirror of the reference's reactor interface over the C ABI.

``Reactor`` follows ``pele::physics::reactions::ReactorBase``
(Source/Reactions/ReactorBase.H:13-106): ``Reactor.create(name)`` as
``ReactorBase::create`` (Source/Factory.H:72-81), ``init(reactor_type,
ncells)``, ``react(...)`` on flat per-cell arrays or on a box, ``close()``.
The reference's ParmParse keys (``ode.rtol``, ``cvode.max_order``, ...) are
accepted as keyword options of ``init``.  Host arrays are numpy; device
arrays are torch CUDA tensors (torch is used for device memory only).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib

_KEYS = {
    # ParmParse key -> ppb_options field
    "ode.rtol": "rtol",
    "ode.atol": "atol",
    "cvode.max_order": "max_order",
    "ode.max_nls_iters": "max_nls_iters",
    "ode.clean_init_massfrac": "clean_init_massfrac",
    "ode.rk64_nsubsteps_guess": "rk64_nsubsteps_guess",
    "ode.rk64_nsubsteps_min": "rk64_nsubsteps_min",
    "ode.rk64_nsubsteps_max": "rk64_nsubsteps_max",
    "ode.verbose": "verbose",
}


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def _stream(stream):
    if stream is None:
        return None
    return getattr(stream, "cuda_stream", stream)


class Reactor:
    """A chemistry reactor on the GPU ("ReactorCvode", "ReactorRK64" or "ReactorArkode")."""

    def __init__(self, mechanism: str, integrator: str = "ReactorCvode"):
        self.mechanism = mechanism
        self.integrator = integrator
        self.nsp, self.nrxn = _lib.mechanism_info(mechanism)
        h = C.c_void_p()
        check(lib().ppb_create(mechanism.encode(), integrator.encode(), C.byref(h)))
        self._h = h
        self.reactor_type = None

    @classmethod
    def create(cls, identifier: str, mechanism: str):
        return cls(mechanism, identifier)

    def init(self, reactor_type: int, ncells: int = 0, **opts):
        o = _lib.default_options()
        fields = {f[0] for f in _lib.Options._fields_}
        for k, v in opts.items():
            key = _KEYS.get(k, k)
            if key not in fields:
                raise TypeError(f"unknown reactor option {k!r}")
            setattr(o, key, v)
        check(lib().ppb_init(self._h, int(reactor_type), int(ncells), C.byref(o)))
        self.reactor_type = reactor_type
        self.options = o
        return 0

    def set_typ_vals_ode(self, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        check(lib().ppb_set_typ_vals(self._h, v.ctypes.data_as(C.POINTER(C.c_double)), v.size))

    def react(self, rY, rYsrc, rX, rX_src, dt_react, time=0.0, ncells=None, stream=None, raise_on_fail=True):
        """Flat YCOrder react; numpy (host) or torch CUDA (device) arrays.

        Returns (cost, dt_react, time, code) with the reference's return
        conventions (cost = summed RHS evaluations for BDF, average RK steps
        for RK64).
        """
        if ncells is None:
            ncells = rX.shape[0]
        dt = C.c_double(dt_react)
        t = C.c_double(time)
        cost = C.c_long(0)
        fn = lib().ppb_react_flat if isinstance(rY, np.ndarray) else lib().ppb_react_flat_device
        for a in (rY, rYsrc, rX, rX_src):
            if isinstance(a, np.ndarray):
                assert a.dtype == np.float64 and a.flags.c_contiguous
        code = fn(self._h, _ptr(rY), _ptr(rYsrc), _ptr(rX), _ptr(rX_src), C.byref(dt), C.byref(t), int(ncells),
                  _stream(stream), C.byref(cost))
        if raise_on_fail or code < 0:
            check(code)
        return cost.value, dt.value, t.value, code

    def launch_config(self):
        """(warps_per_block, team_lanes, register_budget, tuned_ms) of the
        tuned engine (after the autotuner ran when warps_per_block was 0)."""
        w, t, rb = C.c_int(), C.c_int(), C.c_int()
        ms = C.c_double()
        check(lib().ppb_get_launch_config(self._h, C.byref(w), C.byref(t), C.byref(rb), C.byref(ms)))
        return w.value, t.value, rb.value, ms.value

    def rendezvous_cycles(self):
        """The block rendezvous bound (SM clocks) of the tuned BDF launches:
        the option when set, else the autotuner's pick or the block-size
        default; 0 without a rendezvous."""
        v = C.c_int()
        check(lib().ppb_get_rendezvous_cycles(self._h, C.byref(v)))
        return v.value

    # ---- differentiation (no counterpart in the reference)
    def get_arrhenius(self):
        """Forward Arrhenius parameters (A in SI units, beta, Ea/R in K)."""
        A, b, e = (np.zeros(self.nrxn) for _ in range(3))
        dpp = C.POINTER(C.c_double)
        check(lib().ppb_get_arrhenius(self._h, A.ctypes.data_as(dpp), b.ctypes.data_as(dpp), e.ctypes.data_as(dpp)))
        return A, b, e

    def set_arrhenius(self, A, beta, EaR):
        dpp = C.POINTER(C.c_double)
        A, beta, EaR = (np.ascontiguousarray(x, dtype=np.float64) for x in (A, beta, EaR))
        assert A.size == beta.size == EaR.size == self.nrxn
        check(lib().ppb_set_arrhenius(self._h, A.ctypes.data_as(dpp), beta.ctypes.data_as(dpp),
                                      EaR.ctypes.data_as(dpp)))

    def adjoint(self, rY0, rYsrc, rX, rX_src, dt_react, lam_y, stream=None):
        """Discrete adjoint of react() (torch CUDA tensors, YCOrder).

        Returns (y_out, lam_y0, lam_e, grad) with grad = [dL/dlnA | dL/dbeta |
        dL/d(Ea/R)] summed over the cells.
        """
        import torch

        n = rY0.shape[0]
        y_out = torch.empty_like(rY0)
        lam_y0 = torch.empty_like(rY0)
        lam_e = torch.empty_like(rX)
        grad = torch.empty(3 * self.nrxn, dtype=torch.float64, device=rY0.device)
        check(lib().ppb_adjoint_flat_device(self._h, _ptr(rY0), _ptr(rYsrc), _ptr(rX), _ptr(rX_src),
                                            float(dt_react), int(n), _ptr(lam_y), _ptr(y_out), _ptr(lam_y0),
                                            _ptr(lam_e), _ptr(grad), _stream(stream)))
        return y_out, lam_y0, lam_e, grad

    def tangent(self, rY0, rYsrc, rX, rX_src, dt_react, dy0=None, drX=None, dparams=None, stream=None):
        """Tangent-linear model of react(): returns (y_out, dy_out)."""
        import torch

        n = rY0.shape[0]
        y_out = torch.empty_like(rY0)
        dy_out = torch.empty_like(rY0)
        if dparams is None:
            dparams = torch.zeros(3 * self.nrxn, dtype=torch.float64, device=rY0.device)
        check(lib().ppb_tangent_flat_device(self._h, _ptr(rY0), _ptr(rYsrc), _ptr(rX), _ptr(rX_src),
                                            float(dt_react), int(n), _ptr(dy0), _ptr(drX), _ptr(dparams),
                                            _ptr(y_out), _ptr(dy_out), _stream(stream)))
        return y_out, dy_out

    def react_soa(self, y, src, rX, rX_src, dt_react, time=0.0, ld=None, ncells=None, stream=None,
                  raise_on_fail=True):
        """Species-major device arrays y[(N+1), ld], src[N, ld]."""
        if ncells is None:
            ncells = rX.shape[0]
        if ld is None:
            ld = y.shape[-1]
        dt = C.c_double(dt_react)
        t = C.c_double(time)
        cost = C.c_long(0)
        code = lib().ppb_react_soa_device(self._h, _ptr(y), _ptr(src), _ptr(rX), _ptr(rX_src), int(ld), C.byref(dt),
                                         C.byref(t), int(ncells), _stream(stream), C.byref(cost))
        if raise_on_fail or code < 0:
            check(code)
        return cost.value, dt.value, t.value, code

    @staticmethod
    def _array4(t, lo, hi, cls=_lib.Array4):
        """Array4 view of a contiguous torch tensor [ncomp, nz, ny, nx]
        covering exactly lo..hi."""
        v = cls()
        v.p = t.data_ptr()
        nc, nz, ny, nx = t.shape
        v.jstride, v.kstride, v.nstride = nx, nx * ny, nx * ny * nz
        v.lo[:] = list(lo)
        v.hi[:] = list(hi)
        v.ncomp = nc
        return v

    def flatten(self, lo, hi, rY, rYsrc, T, rEner, rEner_src, y_vect, src_vect, vect_energy, src_vect_energy,
                stream=None):
        """ReactorBase::flatten on torch CUDA tensors: box arrays shaped
        [ncomp, nz, ny, nx] into the component-major vectors y_vect[(N+1)
        ncells], src_vect[N ncells], vect_energy[ncells],
        src_vect_energy[ncells]."""
        a4 = lambda t: self._array4(t, lo, hi)
        check(lib().ppb_flatten(self._h, (C.c_int * 3)(*lo), (C.c_int * 3)(*hi), a4(rY), a4(rYsrc), a4(T), a4(rEner),
                                a4(rEner_src), _ptr(y_vect), _ptr(src_vect), _ptr(vect_energy),
                                _ptr(src_vect_energy), _stream(stream)))

    def unflatten(self, lo, hi, rY, T, rEner, rEner_src, FC, y_vect, vect_energy, FCunt, dt_react, stream=None):
        """ReactorBase::unflatten on torch CUDA tensors (FCunt: int64 per
        cell)."""
        a4 = lambda t: self._array4(t, lo, hi)
        check(lib().ppb_unflatten(self._h, (C.c_int * 3)(*lo), (C.c_int * 3)(*hi), a4(rY), a4(T), a4(rEner),
                                  a4(rEner_src), self._array4(FC, lo, hi, _lib.Array4i), _ptr(y_vect),
                                  _ptr(vect_energy), _ptr(FCunt), float(dt_react), _stream(stream)))

    def react_box(self, lo, hi, rY, rYsrc, T, rEner, rEner_src, FC, mask=None, dt_react=0.0, time=0.0,
                  stream=None, raise_on_fail=True):
        """Box react on torch CUDA tensors shaped [ncomp, nz, ny, nx] that
        cover exactly the box lo..hi (inclusive)."""
        lo3 = (C.c_int * 3)(*lo)
        hi3 = (C.c_int * 3)(*hi)
        a4 = lambda t, cls=_lib.Array4: self._array4(t, lo, hi, cls)
        m = _lib.Array4i()
        if mask is not None:
            m = a4(mask, _lib.Array4i)
        dt = C.c_double(dt_react)
        t = C.c_double(time)
        code = lib().ppb_react_box(self._h, lo3, hi3, a4(rY), a4(rYsrc), a4(T), a4(rEner), a4(rEner_src), a4(FC), m,
                                   C.byref(dt), C.byref(t), _stream(stream))
        if raise_on_fail or code < 0:
            check(code)
        return dt.value, t.value, code

    def cell_status(self, ncells):
        st = np.zeros(ncells, np.int32)
        cost = np.zeros(ncells, np.int32)
        check(lib().ppb_get_cell_status(self._h, st.ctypes.data_as(C.POINTER(C.c_int)),
                                        cost.ctypes.data_as(C.POINTER(C.c_int)), int(ncells)))
        return st, cost

    def cell_stats(self, ncells):
        """[ncells, 7]: steps, nfe, nje, nsetups, nni, netf, ncfn."""
        st = np.zeros((ncells, 7), np.int32)
        check(lib().ppb_get_cell_stats(self._h, st.ctypes.data_as(C.POINTER(C.c_int)), int(ncells)))
        return st

    def close(self):
        if self._h:
            lib().ppb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_fp64_peak():
    """Measured FP64 FMA throughput of the current GPU, GFLOP/s."""
    g = C.c_double()
    check(lib().ppb_probe_fp64_peak(C.byref(g), None))
    return g.value


def pyt2re(mechanism, P, T, Y, eh=0, stream=None):
    """Device EOS: (rho, e or h) from P, T, Y (torch CUDA float64 tensors)."""
    import torch

    n = T.shape[0]
    rho = torch.empty_like(T)
    e = torch.empty_like(T)
    check(lib().ppb_pyt2re(mechanism.encode(), int(eh), _ptr(P), _ptr(T), _ptr(Y), _ptr(rho), _ptr(e), int(n),
                           _stream(stream)))
    return rho, e
