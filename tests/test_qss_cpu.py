"""QSS mechanisms on the CPU (no GPU): the oracle's table-driven QSS
chemistry (CH4_lean_qss: 13 transported species, 4 in quasi-steady state,
73 reactions, 41 of them with a QSS species) against the golden vectors of
the reference's own compiled Mechanisms/CH4_lean_qss/mechanism.H
(tests/golden/make_golden.py qss): the QSS concentrations comp_sc_qss
solves, productionRate, thermo, the temperature solves and the reactor
right-hand side of both reactor types; the generated tables' balance
structure; and BDF over the table kernels against BDF over the reference's
compiled kernels (difference-quotient Jacobian in both, as the reference's
dense_direct solve forms it)."""

import os

import numpy as np
import pytest

from tests.helpers import premix_oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")
MECH = "CH4_lean_qss"


def load():
    return dict(np.load(os.path.join(GOLD, f"point_{MECH}.npz")))


def test_qss_tables(oracle):
    M = oracle.Mech(MECH)
    assert M.nsp == 13 and M.nqss == 4
    assert M.species() == ["H2", "H", "O", "O2", "OH", "H2O", "HO2", "CH3", "CH4", "CO", "CO2", "CH2O", "N2"]
    assert oracle.Mech("drm19").nqss == 0


def test_qss_concentrations_match_reference(oracle):
    """comp_sc_qss eliminates symbolically in an order of its own; the
    oracle solves the same linear balance in species order: equal to a few
    ulps of the solution."""
    g = load()
    M = oracle.Mech(MECH)
    for i, T in enumerate(g["T"]):
        x = M.qss_concentrations(g["sc"][i], T)
        ref = g["sc_qss"][i]
        assert np.all(np.abs(x - ref) <= 1e-12 * np.abs(ref) + 1e-300), (i, x, ref)


def test_qss_production_rate_matches_reference(oracle):
    """|wdot - wdot_ref| <= 1e-12 * sum_r |nu| (|qf| + |qr|) per species."""
    g = load()
    M = oracle.Mech(MECH)
    for i, T in enumerate(g["T"]):
        w = M.production_rate(g["sc"][i], T)
        scale = M.production_rate_abs(g["sc"][i], T)
        err = np.abs(w - g["wdot"][i])
        assert np.all(err <= 1e-12 * scale + 1e-300), (i, np.max(err / (scale + 1e-300)))


def test_qss_thermo_matches_reference(oracle):
    g = load()
    M = oracle.Mech(MECH)
    np.testing.assert_array_equal(M.mw(), g["mw"])
    for i, T in enumerate(g["T"]):
        np.testing.assert_allclose(M.gibbs(T), g["gibbs"][i], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(M.ckums(T), g["ums"][i], rtol=1e-13, atol=1e-6)
        Y = g["Y"][i]
        assert abs(M.ckcvbs(T, Y) - g["cvbs"][i]) <= 1e-13 * abs(g["cvbs"][i])
        assert abs(M.ckcpbs(T, Y) - g["cpbs"][i]) <= 1e-13 * abs(g["cpbs"][i])
        t1, _ = M.t_given_ey(g["ubms"][i], Y, g["Tguess"][i])
        t2, _ = M.t_given_hy(g["hbms"][i], Y, g["Tguess"][i])
        assert abs(t1 - g["T_ey"][i]) <= 1e-12 * g["T_ey"][i]
        assert abs(t2 - g["T_hy"][i]) <= 1e-12 * g["T_hy"][i]


@pytest.mark.parametrize("rtype", [1, 2])
def test_qss_reactor_rhs_matches_reference(oracle, rtype):
    """fKernelSpec over the QSS productionRate: species rates within 1e-12
    of their gross rates, the T row within 1e-10 of its scale."""
    g = load()
    M = oracle.Mech(MECH)
    N = M.nsp
    mw = M.mw()
    for i in range(len(g["T"])):
        y = g["y"][i]
        f, _ = M.reactor_rhs(rtype, 1e-7, y, g[f"rhoe{rtype}"][i], g["rhoesrc"][i], g["src"][i])
        ref = g[f"ydot{rtype}"][i]
        rho = y[:N].sum()
        T = g["T"][i]
        gross = M.production_rate_abs(y[:N] / mw * 1e6, T) * 1e-6 * mw
        assert np.all(np.abs(f[:N] - ref[:N]) <= 1e-10 * gross + 1e-12 * np.abs(g["src"][i]) + 1e-300), i
        assert abs(f[N] - ref[N]) <= 1e-9 * (abs(ref[N]) + abs(g["rhoesrc"][i]) / rho) + 1e-300, i


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                                                    f"libref_{MECH}.so")), reason="reference kernels not built")
def test_qss_bdf_tables_vs_reference_kernels(oracle):
    """BDF (difference-quotient Jacobian) over the table-driven QSS kernels
    and over the reference's compiled ones agree to the integration
    tolerance on igniting lean methane cells."""
    rY, src, rX, _ = premix_oracle(oracle, MECH, 4, 3, 1300.0, 400.0, 0.5, 0.5)
    N = rY.shape[1] - 1
    for c in range(4):
        a, fa, _ = oracle.bdf_cell(MECH, 1, rY[c], src[c], rX[c], 0.0, 2e-4, rtol=1e-10, atol=1e-10, max_order=5)
        b, fb, _ = oracle.bdf_cell(MECH, 1, rY[c], src[c], rX[c], 0.0, 2e-4, rtol=1e-10, atol=1e-10, max_order=5,
                                   use_ref_kernels=1)
        assert fa == 0 and fb == 0
        assert abs(a[N] - b[N]) <= 1e-7 * b[N]
        assert np.max(np.abs(a[:N] - b[:N])) <= 1e-8 * a[:N].sum()


def test_mechanism_tables_regenerate_identically(oracle, tmp_path):
    """The shipped mech_<name>.h tables are what the generator writes from
    the reference's mechanism files (all five mechanisms)."""
    from pelephysics_b200.mechgen import ceptr_tables as ct

    root = oracle.reference_root()
    if root is None or not os.path.isdir(os.path.join(root, "Mechanisms")):
        pytest.skip("needs the reference tree")
    for mech in ct.MECHS:
        M = ct.build(os.path.join(root, "Mechanisms", mech), mech)
        out = tmp_path / f"mech_{mech}.h"
        ct.emit_header(M, str(out))
        ship = os.path.join(os.path.dirname(os.path.dirname(__file__)), "pelephysics_b200", "csrc", "mech",
                            f"mech_{mech}.h")
        assert out.read_text() == open(ship).read(), mech
