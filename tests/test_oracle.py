"""CPU oracle checks (no GPU): the table-driven restatement of the
reference's chemistry against the golden vectors the reference's own
compiled kernels produced (tests/golden/make_golden.py), the reference's
ignition-delay pin, and an independent VODE integration."""

import os

import numpy as np
import pytest

from tests.helpers import premix_oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")
MECHS = ["LiDryer", "drm19", "dodecane_lu", "heptane_lu_88sk", "grimech30", "FFCM1_Red", "chem-H"]


def load(mech):
    return dict(np.load(os.path.join(GOLD, f"point_{mech}.npz")))


@pytest.mark.parametrize("mech", MECHS)
def test_thermo_matches_reference(oracle, mech):
    g = load(mech)
    M = oracle.Mech(mech)
    np.testing.assert_array_equal(M.mw(), g["mw"])
    for i, T in enumerate(g["T"]):
        np.testing.assert_allclose(M.gibbs(T), g["gibbs"][i], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(M.ckums(T), g["ums"][i], rtol=1e-13, atol=1e-6)
        np.testing.assert_allclose(M.ckhms(T), g["hms"][i], rtol=1e-13, atol=1e-6)
        Y = g["Y"][i]
        assert abs(M.ckubms(T, Y) - g["ubms"][i]) <= 1e-13 * abs(g["ubms"][i]) + 1e-3
        assert abs(M.ckcvbs(T, Y) - g["cvbs"][i]) <= 1e-13 * abs(g["cvbs"][i])
        assert abs(M.ckhbms(T, Y) - g["hbms"][i]) <= 1e-13 * abs(g["hbms"][i]) + 1e-3
        assert abs(M.ckcpbs(T, Y) - g["cpbs"][i]) <= 1e-13 * abs(g["cpbs"][i])
        t1, _ = M.t_given_ey(g["ubms"][i], Y, g["Tguess"][i])
        t2, _ = M.t_given_hy(g["hbms"][i], Y, g["Tguess"][i])
        assert abs(t1 - g["T_ey"][i]) <= 1e-12 * g["T_ey"][i]
        assert abs(t2 - g["T_hy"][i]) <= 1e-12 * g["T_hy"][i]


@pytest.mark.parametrize("mech", MECHS)
def test_production_rate_matches_reference(oracle, mech):
    """|wdot - wdot_ref| <= 1e-12 * sum_r |nu| (|qf| + |qr|) per species."""
    g = load(mech)
    M = oracle.Mech(mech)
    for i, T in enumerate(g["T"]):
        w = M.production_rate(g["sc"][i], T)
        scale = M.production_rate_abs(g["sc"][i], T)
        err = np.abs(w - g["wdot"][i])
        assert np.all(err <= 1e-12 * scale + 1e-300), (i, np.max(err / (scale + 1e-300)))


@pytest.mark.parametrize("mech", MECHS)
@pytest.mark.parametrize("consP", [0, 1])
def test_ajacobian_matches_reference(oracle, mech, consP):
    g = load(mech)
    M = oracle.Mech(mech)
    for i, T in enumerate(g["T"]):
        J = M.ajacobian(g["sc"][i], T, consP)
        ref = g[f"jac{consP}"][i]
        assert np.linalg.norm(J - ref) <= 1e-12 * np.linalg.norm(ref)
        big = np.abs(ref) > 1e-6 * np.abs(ref).max()
        assert np.all(np.abs(J - ref)[big] <= 1e-10 * np.abs(ref)[big])


def test_ignition_delay_pin(oracle):
    """Testing/Exec/IgnitionDelay: dodecane_lu, 600 K, 5 atm, phi 7.93,
    enthalpy reactor, rtol = atol = 1e-10, max order 4: first T > T0 + 400
    at 0.0763 s, checked within 10 * dt/ndt (check_ignDelay.py:22-29)."""
    mech = "dodecane_lu"
    M = oracle.Mech(mech)
    sp = M.species()
    mw = M.mw()
    N = M.nsp
    X = np.zeros(N)
    phi = 7.928571428571429
    io2, in2, ifu = sp.index("O2"), sp.index("N2"), sp.index("NC12H26")
    X[io2] = 1.0 / (phi / 18.5 + 1 + 0.79 / 0.21)  # GPU_misc.H:62-64
    X[in2] = 0.79 * X[io2] / 0.21
    X[ifu] = 1 - X[io2] - X[in2]
    Y = X * mw / np.sum(X * mw)
    P, T0 = 5066250.0, 600.0
    rho = M.ckrhoy(P, T0, Y)
    rhoH = rho * M.ckhbms(T0, Y)
    rhoY = rho * Y
    ndt = 4000
    sub = 1.1 * 0.0763 / ndt
    T = T0
    t_ign = None
    for i in range(ndt):
        rho = rhoY.sum()
        T, _ = M.t_given_hy(rhoH / rho, rhoY / rho, T)
        y, flag, _ = oracle.bdf_cell(mech, 2, np.r_[rhoY, T], np.zeros(N), rhoH, 0.0, sub, rtol=1e-10,
                                     atol=1e-10, max_order=4)
        assert flag == 0
        rhoY = y[:N]
        rho = rhoY.sum()
        T, _ = M.t_given_hy(rhoH / rho, rhoY / rho, y[N])
        if T > T0 + 400:
            t_ign = (i + 1) * sub
            break
    assert t_ign is not None
    assert abs(t_ign - 0.0763) <= 10 * sub


def test_bdf_against_vode(oracle):
    """The CVODE-algorithm BDF agrees with scipy's VODE (the ancestor of
    CVODE) on a LiDryer ignition at tight tolerance."""
    from scipy.integrate import ode

    rY, src, rX, _ = premix_oracle(oracle, "LiDryer", 1, 5, 1200.0, 0.0, 1.0, 0.0)
    M = oracle.Mech("LiDryer")
    N = M.nsp
    dt = 1e-4
    f = lambda t, y: M.reactor_rhs(1, t, y, rX[0], 0.0, src[0])[0]
    r = ode(f).set_integrator("vode", method="bdf", rtol=1e-12, atol=1e-14, nsteps=2000000, order=5)
    r.set_initial_value(rY[0], 0.0)
    yv = r.integrate(dt)
    assert r.successful()
    y, flag, st = oracle.bdf_cell("LiDryer", 1, rY[0], src[0], rX[0], 0.0, dt, rtol=1e-12, atol=1e-14,
                                  max_order=5)
    assert flag == 0
    assert abs(y[N] - yv[N]) <= 1e-6 * yv[N]
    assert np.max(np.abs(y[:N] / y[:N].sum() - yv[:N] / yv[:N].sum())) <= 1e-7


def test_oracle_tables_vs_reference_kernels_integration(oracle):
    """BDF over the table-driven kernels and over the reference's compiled
    kernels agree to the integration tolerance."""
    if not oracle.have_ref("drm19"):
        pytest.skip("reference kernels not built")
    rY, src, rX, _ = premix_oracle(oracle, "drm19", 4, 3, 1400.0, 300.0, 0.6, 0.8)
    N = rY.shape[1] - 1
    for c in range(4):
        a, fa, _ = oracle.bdf_cell("drm19", 1, rY[c], src[c], rX[c], 0.0, 1e-5, rtol=1e-10, atol=1e-10,
                                   max_order=5)
        b, fb, _ = oracle.bdf_cell("drm19", 1, rY[c], src[c], rX[c], 0.0, 1e-5, rtol=1e-10, atol=1e-10,
                                   max_order=5, use_ref_kernels=1)
        assert fa == 0 and fb == 0
        assert abs(a[N] - b[N]) <= 1e-8 * b[N]


def test_rk64_converges(oracle):
    rY, src, rX, _ = premix_oracle(oracle, "LiDryer", 1, 5, 1200.0, 0.0, 1.0, 0.0)
    N = rY.shape[1] - 1
    a, _, _ = oracle.bdf_cell("LiDryer", 1, rY[0], src[0], rX[0], 0.0, 1e-6, rtol=1e-12, atol=1e-14,
                              max_order=5)
    b, n = oracle.rk64_cell("LiDryer", 1, rY[0], src[0], rX[0], 0.0, 1e-6, atol=1e-10)
    assert n >= 5
    assert abs(a[N] - b[N]) <= 1e-9 * a[N]


def test_rhs_noise_replicas_and_the_parity_criterion(oracle):
    """rhs_noise_seed = 0 is the plain integrator (bitwise); seeds > 0 move
    right-hand-side values by at most one ulp and change results only at the
    integration-error level; and the table-driven restatement of the
    reference's kernels passes compare_to_reference against the reference's
    own compiled kernels on the whole LiDryer 16^3 configuration (4096 cells,
    dt 1e-4 s, rtol = atol = 1e-10), the same check the GPU engine is held to."""
    from pelephysics_b200 import workloads as wl

    mech = "LiDryer"
    if not oracle.have_ref(mech):
        pytest.skip("reference kernels not built")
    M = oracle.Mech(mech)

    def eos(T, Y, P, rtype):
        rho = np.array([M.ckrhoy(P, t, y) for t, y in zip(T, Y)])
        return rho, rho * np.array([M.ckubms(t, y) for t, y in zip(T, Y)])

    cells = wl.premix_cells(mech, 16 ** 3, 0, 1000.0, 400.0, 0.5, 1.5, reactor_type=1, dt=1e-4, eos=eos,
                            species=M.species(), mw=M.mw())
    opts = dict(rtol=1e-10, atol=1e-10, max_order=5)

    def run(ref, **kw):
        y = cells.rY.copy()
        flag, _, _ = oracle.react_flat(mech, 1, y, np.ascontiguousarray(cells.rYsrc), cells.rX.copy(),
                                       cells.rX_src.copy(), cells.dt, use_ref_kernels=ref, **opts, **kw)
        assert flag == 0
        return y

    r10 = run(1)
    assert np.array_equal(run(1, rhs_noise_seed=0), r10)
    noisy = run(1, rhs_noise_seed=3)
    d = np.abs(noisy[:, :9] / noisy[:, :9].sum(1, keepdims=True) - r10[:, :9] / r10[:, :9].sum(1, keepdims=True))
    assert 0 < d.max() < 1e-6
    res = oracle.compare_to_reference(mech, 1, cells.rY, cells.rYsrc, cells.rX, cells.rX_src, cells.dt, run(0), r10,
                                      use_ref_kernels=1, **opts)
    assert res["cells_failing"] == 0 and res["cells_over_Y_atol"] <= 0.005 * 4096, res
