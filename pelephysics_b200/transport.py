"""Mixture-averaged transport coefficients on the GPU (the reference's
SimpleTransport, Source/Transport/Simple.H, ideal-gas EOS).

``transport`` evaluates SimpleTransport::transport for every cell of a flat
batch (torch CUDA float64 tensors), ``transport_box`` mirrors
SimpleTransport::get_transport_coeffs on a box of Array4-shaped tensors
[ncomp, nz, ny, nx].  Both call the C ABI (``ppb_transport``,
``ppb_transport_box``).
"""

from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import check, lib

TR_XI, TR_MU, TR_LAM, TR_DIAG, TR_CHI = 1, 2, 4, 8, 16
TR_ALL = TR_XI | TR_MU | TR_LAM | TR_DIAG | TR_CHI


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(stream):
    return None if stream is None else C.c_void_p(getattr(stream, "cuda_stream", stream))


def transport(mechanism, T, rho, Y, flags=TR_ALL, stream=None):
    """T, rho [ncells]; Y [N, ld] species-major (ld >= ncells).  Returns a
    dict with the selected outputs: D [N, ld], chi [N, ld], mu, xi, lam
    [ncells]."""
    import torch

    N, ld = Y.shape
    n = T.shape[0]
    dev = Y.device
    out = {}
    if flags & TR_DIAG:
        out["D"] = torch.zeros((N, ld), dtype=torch.float64, device=dev)
    if flags & TR_CHI:
        out["chi"] = torch.zeros((N, ld), dtype=torch.float64, device=dev)
    for k, f in (("mu", TR_MU), ("xi", TR_XI), ("lam", TR_LAM)):
        if flags & f:
            out[k] = torch.zeros(n, dtype=torch.float64, device=dev)
    check(lib().ppb_transport(mechanism.encode(), int(flags), _p(T), _p(rho), _p(Y), int(ld), _p(out.get("D")),
                              _p(out.get("chi")), _p(out.get("mu")), _p(out.get("xi")), _p(out.get("lam")), int(n),
                              _stream(stream)))
    return out


def _a4(t, lo, hi):
    v = _lib.Array4()
    v.p = t.data_ptr()
    nc, nz, ny, nx = t.shape
    v.jstride, v.kstride, v.nstride = t.stride(2), t.stride(1), t.stride(0)
    v.lo[:] = list(lo)
    v.hi[:] = [lo[0] + nx - 1, lo[1] + ny - 1, lo[2] + nz - 1]
    v.ncomp = nc
    return v


def transport_box(mechanism, lo, hi, Y, T, rho, D, chi, mu, xi, lam, use_soret=False, alloc_lo=None,
                  stream=None):
    """get_transport_coeffs on the box lo..hi (inclusive) of tensors shaped
    [ncomp, nz, ny, nx] whose element [n, 0, 0, 0] sits at alloc_lo (default
    lo): the box may be an interior part of larger allocations."""
    alo = list(alloc_lo if alloc_lo is not None else lo)
    lo3 = (C.c_int * 3)(*lo)
    hi3 = (C.c_int * 3)(*hi)
    views = [_a4(t, alo, hi) for t in (Y, T, rho, D)]
    views.append(_a4(chi, alo, hi) if chi is not None else _lib.Array4())
    views += [_a4(t, alo, hi) for t in (mu, xi, lam)]
    check(lib().ppb_transport_box(mechanism.encode(), int(bool(use_soret)), lo3, hi3, *views, _stream(stream)))
