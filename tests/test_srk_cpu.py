"""The SRK equation of state on the CPU: the oracle's restatement against
the golden outputs of the reference's own compiled Source/Eos/SRK.H
(tests/golden/srk_<mech>.npz) and the ideal-gas limit."""

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
MECHS = ["LiDryer", "drm19", "dodecane_lu", "heptane_lu_88sk"]


def rel(a, b, floor=0.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), floor + 1e-300))


@pytest.mark.parametrize("mech", MECHS)
def test_oracle_srk_matches_reference(oracle, mech):
    g = np.load(os.path.join(HERE, "golden", f"srk_{mech}.npz"))
    s = oracle.Srk(mech)
    for c in range(g["T"].shape[0]):
        R, T, Y = g["rho"][c], g["T"][c], g["Y"][c]
        assert rel(s.rty2e(R, T, Y), g["e"][c]) <= 1e-13
        assert rel(s.rty2cv(R, T, Y), g["cv"][c]) <= 1e-13
        assert rel(s.rty2ei(R, T, Y), g["ei"][c], 1e-12 * np.max(np.abs(g["ei"][c]))) <= 1e-12
        assert rel(s.rty2c(R, T, Y), g["c"][c]) <= 1e-13
        w = g["wdot"][c]
        assert np.max(np.abs(s.rty2wdot(R, T, Y) - w)) <= 1e-12 * np.max(np.abs(w))
        assert rel(s.rey2t(R, g["e"][c], Y, T + 100.0), g["T_ey"][c]) <= 1e-12
        ydot, _ = s.reactor_rhs(2e-7, g["y"][c], R * g["e"][c], g["rhoesrc"][c], g["src"][c])
        ref = g["ydot"][c]
        assert np.max(np.abs(ydot - ref)) <= 1e-10 * np.max(np.abs(ref[:-1])) + 1e-10 * abs(ref[-1])


def test_srk_tends_to_the_ideal_gas(oracle):
    """At vanishing density the SRK energy, heat capacity and activities
    reduce to the ideal gas's (CKUBMS, CKCVBS, rho Y / W)."""
    mech = "drm19"
    s = oracle.Srk(mech)
    M = oracle.Mech(mech)
    rng = np.random.default_rng(0)
    Y = rng.uniform(size=s.N)
    Y /= Y.sum()
    T, R = 1200.0, 1e-9
    assert abs(s.rty2e(R, T, Y) - M.ckubms(T, Y)) <= 1e-6 * abs(M.ckubms(T, Y))
    assert abs(s.rty2cv(R, T, Y) - M.ckcvbs(T, Y)) <= 1e-6 * M.ckcvbs(T, Y)
    np.testing.assert_allclose(s.rty2c(R, T, Y), R * Y / M.mw(), rtol=1e-6)


def test_oracle_srk_reactor_tends_to_the_ideal_reactor(oracle):
    """The oracle's BDF with the SRK right-hand side and difference-quotient
    Jacobian against the ideal-gas BDF: close at 1 atm, apart at 50 atm."""
    from tests.helpers import premix_oracle

    mech, nc, dt = "drm19", 6, 1e-5
    out = {}
    for P in (1013250.0, 50 * 1013250.0):
        rY, src, rX, rXs = premix_oracle(oracle, mech, nc, 4, 1300.0, 300.0, 0.5, 1.0, P=P)
        s = oracle.Srk(mech)
        N = rY.shape[1] - 1
        rho = rY[:, :N].sum(1)
        rXs_ = np.array([rho[c] * s.rty2e(rho[c], rY[c, N], rY[c, :N] / rho[c]) for c in range(nc)])
        ys, yi = rY.copy(), rY.copy()
        f1, _, _ = oracle.react_flat(mech, 1, ys, np.ascontiguousarray(src), rXs_.copy(), rXs, dt, rtol=1e-10,
                                     atol=1e-10, max_order=5, eos=1)
        f2, _, _ = oracle.react_flat(mech, 1, yi, np.ascontiguousarray(src), rX.copy(), rXs, dt, rtol=1e-10,
                                     atol=1e-10, max_order=5)
        assert f1 == 0 and f2 == 0
        out[P] = np.max(np.abs(ys[:, N] - yi[:, N]) / yi[:, N])
    assert out[1013250.0] < 1e-4
    assert out[50 * 1013250.0] > 3 * out[1013250.0]
