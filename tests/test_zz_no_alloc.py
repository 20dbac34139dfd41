"""The allocation-free entry point (ppb_react_flat_device_noalloc).

It exists for callers that must not have a library allocate GPU memory --
applications whose device memory is owned by an arena allocator, such as
AMReX-based codes whose buffers all come from the AMReX Arena.  It runs the
tuned engine out of one static 32 MiB device array per GPU instead of
cudaMalloc'd scratch.  These checks call it through the C ABI and compare it
with the allocating device entry point (ppb_react_flat_device) on the same
cells, on two calls in a row, within the integration tolerance the other
GPU tests use (T 1e-6 relative, mass fractions 1e-8 absolute).  This file is
collected last so a failure here cannot hide the other tests' results, and
it passes both alone in a fresh process (where its first call does the
per-device set-up) and after the other tests.
"""

import ctypes as C

import numpy as np
import pytest

from pelephysics_b200 import _lib
from pelephysics_b200.reactor import Reactor
from tests.helpers import premix_oracle

pytestmark = pytest.mark.gpu


def _noalloc(torch, mech, y, src, x, xs, dt, opts):
    nfail = C.c_int(-1)
    code = _lib.lib().ppb_react_flat_device_noalloc(mech.encode(), b"ReactorCvode", 1, C.byref(opts), y.data_ptr(),
                                                    src.data_ptr(), x.data_ptr(), xs.data_ptr(), dt, x.shape[0], None,
                                                    C.byref(nfail))
    torch.cuda.synchronize()
    return code, nfail.value


def test_noalloc_matches_allocating_entry_point(cuda, oracle):
    torch = cuda
    mech, dt, ncells = "drm19", 1e-5, 300
    rY, src, rX, rXs = premix_oracle(oracle, mech, ncells, 21, 1100.0, 1100.0, 0.6, 0.8)
    N = rY.shape[1] - 1
    kw = dict(rtol=1e-10, atol=1e-10, max_order=5)

    # the existing (allocating) device entry point
    r = Reactor(mech)
    r.init(1, ncells, use_graph=0, **kw)
    y_ref = torch.as_tensor(rY, device="cuda").contiguous()
    x_ref = torch.as_tensor(rX, device="cuda")
    s_ref = torch.as_tensor(src, device="cuda").contiguous()
    xs_ref = torch.as_tensor(rXs, device="cuda")
    r.react(y_ref, s_ref, x_ref, xs_ref, dt)
    torch.cuda.synchronize()
    y_ref = y_ref.cpu().numpy()
    x_ref = x_ref.cpu().numpy()
    r.close()

    opts = _lib.default_options(**kw)
    for call in range(2):  # the second call reuses the shared array's leftovers
        y = torch.as_tensor(rY, device="cuda").contiguous()
        x = torch.as_tensor(rX, device="cuda")
        s = torch.as_tensor(src, device="cuda").contiguous()
        xs = torch.as_tensor(rXs, device="cuda")
        code, nfail = _noalloc(torch, mech, y, s, x, xs, dt, opts)
        assert code == 0 and nfail == 0, (code, _lib.lib().ppb_last_error())
        y = y.cpu().numpy()
        dT = np.abs(y[:, N] - y_ref[:, N]) / y_ref[:, N]
        Yn = y[:, :N] / y[:, :N].sum(1, keepdims=True)
        Yr = y_ref[:, :N] / y_ref[:, :N].sum(1, keepdims=True)
        assert dT.max() <= 1e-6, (call, dT.max())
        assert np.abs(Yn - Yr).max() <= 1e-8, (call, np.abs(Yn - Yr).max())
        np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-15)


def test_noalloc_rejects_oversized_batch(cuda):
    torch = cuda
    opts = _lib.default_options()
    big = 10 ** 6
    y = torch.zeros(1, dtype=torch.float64, device="cuda")
    nfail = C.c_int()
    code = _lib.lib().ppb_react_flat_device_noalloc(b"drm19", b"ReactorCvode", 1, C.byref(opts), y.data_ptr(),
                                                    y.data_ptr(), y.data_ptr(), y.data_ptr(), 1e-5, big, None,
                                                    C.byref(nfail))
    assert code == _lib.PPB_E_ARG
    assert b"exceeds the allocation-free path's maximum" in _lib.lib().ppb_last_error()
