"""The allocation-free entry point (ppb_react_flat_device_noalloc).

It exists for callers that must not have a library allocate GPU memory --
applications whose device memory is owned by an arena allocator, such as
AMReX-based codes whose buffers all come from the AMReX Arena.  It runs the
tuned engine out of one static 32 MiB device array per GPU instead of
cudaMalloc'd scratch.  These checks call it through the C ABI and compare it
with the allocating device entry point (ppb_react_flat_device) on the same
cells and the same launch (block size, lanes per cell, register budget, cells
in index order), on two calls in a row.  Per-cell arithmetic does not depend
on how cells are scheduled, so the outputs must be bitwise equal.  The second
call must also leave the device's free memory unchanged (the first call may
load kernels).  This file is collected last so a failure here cannot hide the
other tests' results, and it passes both alone in a fresh process (where its
first call does the per-device set-up) and after the other tests.
"""

import ctypes as C

import numpy as np
import pytest

from pelephysics_b200 import _lib
from pelephysics_b200.reactor import Reactor
from tests.helpers import premix_oracle

pytestmark = pytest.mark.gpu

NOALLOC_BYTES = 32 << 20
NOALLOC_TABLES = 2 << 20


def _max_cells(N):
    """The documented per-call limit: (30 MiB - 1 KiB) / (8 (2N+1) + 12)."""
    return (NOALLOC_BYTES - NOALLOC_TABLES - 1024) // (8 * (2 * N + 1) + 12)


def _noalloc(torch, mech, integ, rtype, y, src, x, xs, dt, opts):
    nfail = C.c_int(-1)
    code = _lib.lib().ppb_react_flat_device_noalloc(mech.encode(), integ.encode(), rtype, C.byref(opts), y.data_ptr(),
                                                    src.data_ptr(), x.data_ptr(), xs.data_ptr(), dt, x.shape[0], None,
                                                    C.byref(nfail))
    torch.cuda.synchronize()
    return code, nfail.value


def _compare(torch, mech, integ, rtype, rY, src, rX, rXs, dt, kw, launch):
    """Allocating path once, then the allocation-free path twice: bitwise
    equal outputs, and no change of the device's free memory on the second
    call."""
    r = Reactor(mech, integ)
    r.init(rtype, rX.shape[0], use_graph=0, cost_order=0, **kw, **launch)
    y_ref = torch.as_tensor(rY, device="cuda").contiguous()
    x_ref = torch.as_tensor(rX, device="cuda")
    s_ref = torch.as_tensor(src, device="cuda").contiguous()
    xs_ref = torch.as_tensor(rXs, device="cuda")
    r.react(y_ref, s_ref, x_ref, xs_ref, dt)
    torch.cuda.synchronize()
    y_ref = y_ref.cpu().numpy()
    x_ref = x_ref.cpu().numpy()
    r.close()

    opts = _lib.default_options(**kw, **launch)
    free = []
    for call in range(2):  # the second call reuses the shared array's leftovers
        y = torch.as_tensor(rY, device="cuda").contiguous()
        x = torch.as_tensor(rX, device="cuda")
        s = torch.as_tensor(src, device="cuda").contiguous()
        xs = torch.as_tensor(rXs, device="cuda")
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info()[0]
        code, nfail = _noalloc(torch, mech, integ, rtype, y, s, x, xs, dt, opts)
        free.append((before, torch.cuda.mem_get_info()[0]))
        assert code == 0 and nfail == 0, (call, code, nfail, _lib.lib().ppb_last_error())
        assert np.array_equal(y.cpu().numpy(), y_ref), (call, np.abs(y.cpu().numpy() - y_ref).max())
        assert np.array_equal(x.cpu().numpy(), x_ref), call
    assert free[1][0] == free[1][1], f"free device memory changed across the second call: {free[1]}"


def test_noalloc_bdf_drm19_bitwise(cuda, oracle):
    mech, ncells = "drm19", 300
    rY, src, rX, rXs = premix_oracle(oracle, mech, ncells, 21, 1100.0, 1100.0, 0.6, 0.8)
    _compare(cuda, mech, "ReactorCvode", 1, rY, src, rX, rXs, 1e-5, dict(rtol=1e-10, atol=1e-10, max_order=5),
             dict(warps_per_block=8, team_lanes=32, register_budget=2))


def test_noalloc_rk64_type2_bitwise(cuda, oracle):
    mech, ncells = "LiDryer", 256
    rY, src, rX, rXs = premix_oracle(oracle, mech, ncells, 3, 1000.0, 400.0, 0.5, 1.5, reactor_type=2)
    _compare(cuda, mech, "ReactorRK64", 2, rY, src, rX, rXs, 1e-6, dict(atol=1e-10),
             dict(warps_per_block=4, team_lanes=32, register_budget=2))


def test_noalloc_heptane_at_the_documented_maximum(cuda, oracle):
    """heptane_lu_88sk at exactly the per-call maximum (22,028 cells), one
    128-lane team per cell; one cell more is rejected."""
    mech = "heptane_lu_88sk"
    N = 88
    ncells = _max_cells(N)
    assert ncells == 22028
    rY, src, rX, rXs = premix_oracle(oracle, mech, ncells, 5, 750.0, 650.0, 0.3, 1.7, P=20 * 1013250.0)
    _compare(cuda, mech, "ReactorCvode", 1, rY, src, rX, rXs, 1e-7, dict(rtol=1e-8, atol=1e-12, max_order=5),
             dict(warps_per_block=4, team_lanes=128, register_budget=1))
    torch = cuda
    y = torch.zeros(1, dtype=torch.float64, device="cuda")
    nfail = C.c_int()
    code = _lib.lib().ppb_react_flat_device_noalloc(mech.encode(), b"ReactorCvode", 1,
                                                    C.byref(_lib.default_options()), y.data_ptr(), y.data_ptr(),
                                                    y.data_ptr(), y.data_ptr(), 1e-7, ncells + 1, None, C.byref(nfail))
    assert code == _lib.PPB_E_ARG
    assert b"exceeds the allocation-free path's maximum" in _lib.lib().ppb_last_error()


def test_noalloc_srk_bitwise(cuda, oracle):
    """The SRK e-reactor option is honoured, not dropped."""
    mech, ncells = "drm19", 64
    rY, src, rX, rXs = premix_oracle(oracle, mech, ncells, 8, 1100.0, 900.0, 0.6, 0.8, P=50 * 1013250.0)
    s = oracle.Srk(mech)
    N = rY.shape[1] - 1
    rho = rY[:, :N].sum(1)
    # the reactor integrates rho e of the SRK EOS
    rX = np.array([rho[c] * s.rty2e(rho[c], rY[c, N], rY[c, :N] / rho[c]) for c in range(ncells)])
    _compare(cuda, mech, "ReactorCvode", 1, rY, src, rX, rXs, 1e-6, dict(rtol=1e-10, atol=1e-10, max_order=5, eos=1),
             dict(warps_per_block=4))


@pytest.mark.parametrize("field,value", [("eos", 7), ("team_lanes", 48), ("register_budget", 3),
                                         ("warps_per_block", 17), ("rendezvous_cycles", 10 ** 8)])
def test_noalloc_rejects_options_it_cannot_honour(cuda, field, value):
    torch = cuda
    opts = _lib.default_options(**{field: value})
    y = torch.zeros(4, dtype=torch.float64, device="cuda")
    nfail = C.c_int()
    code = _lib.lib().ppb_react_flat_device_noalloc(b"drm19", b"ReactorCvode", 1, C.byref(opts), y.data_ptr(),
                                                    y.data_ptr(), y.data_ptr(), y.data_ptr(), 1e-5, 1, None,
                                                    C.byref(nfail))
    assert code == _lib.PPB_E_ARG, (field, code)


def test_noalloc_rejects_srk_for_the_h_reactor(cuda):
    torch = cuda
    opts = _lib.default_options(eos=1)
    y = torch.zeros(4, dtype=torch.float64, device="cuda")
    nfail = C.c_int()
    code = _lib.lib().ppb_react_flat_device_noalloc(b"drm19", b"ReactorCvode", 2, C.byref(opts), y.data_ptr(),
                                                    y.data_ptr(), y.data_ptr(), y.data_ptr(), 1e-5, 1, None,
                                                    C.byref(nfail))
    assert code == _lib.PPB_E_ARG
    assert b"SRK" in _lib.lib().ppb_last_error()
