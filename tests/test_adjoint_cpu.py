"""CPU-side pieces of the derivative checks: the oracle's replaceable
Arrhenius parameters (used for finite differences) and the loss seed."""

import numpy as np

from pelephysics_b200 import adjoint as adj
from tests.helpers import premix_oracle


def test_oracle_arrhenius_copy_is_exact(oracle):
    mech, rtype, dt = "LiDryer", 1, 1e-5
    rY, src, rX, rXs = premix_oracle(oracle, mech, 4, 0, 1100.0, 300.0, 0.5, 1.5)
    A, b, e = oracle.arrhenius(mech)
    y1, y2 = rY.copy(), rY.copy()
    oracle.react_flat(mech, rtype, y1, src, rX.copy(), rXs, dt, rtol=1e-10, atol=1e-10, use_ref_kernels=0)
    oracle.react_flat_arrhenius(mech, A, b, e, rtype, y2, src, rX.copy(), rXs, dt, rtol=1e-10, atol=1e-10)
    np.testing.assert_array_equal(y1, y2)
    # faster rate constants move the integration (the parameters reach it)
    y3 = rY.copy()
    oracle.react_flat_arrhenius(mech, A * 1.5, b, e, rtype, y3, src, rX.copy(), rXs, dt, rtol=1e-10, atol=1e-10)
    assert np.all(np.isfinite(y3)) and np.any(np.abs(y3[:, -1] - y1[:, -1]) > 1e-6)


def test_loss_seed_matches_finite_differences():
    rng = np.random.default_rng(0)
    nc, n, ioh = 3, 6, 2
    y = rng.uniform(0.1, 1.0, size=(nc, n))
    y[:, -1] = 1500.0
    wT, wOH = rng.normal(size=nc), rng.normal(size=nc)
    L0, lam = adj.loss_T_OH(y, ioh, wT, wOH)
    for c in range(nc):
        for k in range(n):
            h = 1e-6 * abs(y[c, k])
            yp, ym = y.copy(), y.copy()
            yp[c, k] += h
            ym[c, k] -= h
            fd = (adj.loss_T_OH(yp, ioh, wT, wOH)[0] - adj.loss_T_OH(ym, ioh, wT, wOH)[0]) / (2 * h)
            assert abs(fd - lam[c, k]) <= 1e-5 * max(1.0, abs(fd))
