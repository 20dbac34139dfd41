"""QSS mechanisms on the CPU (no GPU): the oracle's table-driven QSS
chemistry against the reference's own compiled Mechanisms/<mech>/mechanism.H
(golden vectors of tests/golden/make_golden.py qss): the QSS concentrations
comp_sc_qss solves, productionRate, thermo, the temperature solves and the
reactor right-hand side of both reactor types; the generated tables' balance
structure against the reference's generated comp_sc_qss, term for term; and
BDF over the table kernels against BDF over the reference's compiled kernels
(difference-quotient Jacobian in both, as the reference's dense_direct solve
forms it).

Mechanisms: CH4_lean_qss (13 transported species, 4 QSS) and C1-C2-NO_qss
(39, 5; two forward rates removed by the reduction) are pinned to the
reference at rounding level.  LuEthylene_qss (22, 10) is pinned in
structure, and its solve against exact rational elimination of the same
linear system: the reference's generated symbolic elimination for its
10-species coupled group loses accuracy on some states (measured on a
random state with a balance matrix of condition number 2: the reference's
CH2* off by 100 %, this solve within 2e-16 of the exact solution; on states
along ignition trajectories its error reaches 5.5e-6 relative, median
5.5e-16), so its rates are compared with the reference only where the
reference's own solve is accurate."""

import os
import re
from fractions import Fraction

import numpy as np
import pytest

from tests.helpers import premix_oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")
MECH = "CH4_lean_qss"
PINNED = ["CH4_lean_qss", "C1-C2-NO_qss"]
ALL = PINNED + ["LuEthylene_qss"]


def load(mech=MECH):
    return dict(np.load(os.path.join(GOLD, f"point_{mech}.npz")))


def exact_solve(system):
    """Gaussian elimination in rational arithmetic of [A | b]."""
    A = [[Fraction(float(v)) for v in row] for row in system]
    Q = len(A)
    for c in range(Q):
        p = max(range(c, Q), key=lambda i: abs(A[i][c]))
        A[c], A[p] = A[p], A[c]
        for i in range(c + 1, Q):
            f = A[i][c] / A[c][c]
            for j in range(c, Q + 1):
                A[i][j] -= f * A[c][j]
    x = [Fraction(0)] * Q
    for i in reversed(range(Q)):
        x[i] = (A[i][Q] - sum(A[i][j] * x[j] for j in range(i + 1, Q))) / A[i][i]
    return np.array([float(v) for v in x])


def test_qss_tables(oracle):
    M = oracle.Mech(MECH)
    assert M.nsp == 13 and M.nqss == 4
    assert M.species() == ["H2", "H", "O", "O2", "OH", "H2O", "HO2", "CH3", "CH4", "CO", "CO2", "CH2O", "N2"]
    assert oracle.Mech("drm19").nqss == 0


@pytest.mark.parametrize("mech", PINNED)
def test_qss_concentrations_match_reference(oracle, mech):
    """comp_sc_qss eliminates symbolically in an order of its own; the
    oracle solves the same linear balance in species order: equal to a few
    ulps of the solution."""
    g = load(mech)
    M = oracle.Mech(mech)
    for i, T in enumerate(g["T"]):
        x = M.qss_concentrations(g["sc"][i], T)
        ref = g["sc_qss"][i]
        assert np.all(np.abs(x - ref) <= 1e-12 * np.abs(ref) + 1e-300), (i, x, ref)


@pytest.mark.parametrize("mech", ALL)
def test_qss_solve_matches_exact_arithmetic(oracle, mech):
    """The species-order elimination against rational elimination of the
    same system, on the golden states."""
    g = load(mech)
    M = oracle.Mech(mech)
    for i, T in enumerate(g["T"]):
        x = M.qss_concentrations(g["sc"][i], T)
        ex = exact_solve(M.qss_system(g["sc"][i], T))
        assert np.all(np.abs(x - ex) <= 1e-13 * np.abs(ex) + 1e-300), (i, x, ex)


@pytest.mark.parametrize("mech", ALL)
def test_qss_production_rate_matches_reference(oracle, mech):
    """|wdot - wdot_ref| <= tol * sum_r |nu| (|qf| + |qr|) per species, tol =
    1e-12; for LuEthylene_qss tol = max(1e-12, 2 e_ref) with e_ref the
    largest relative error of the reference's own QSS concentrations against
    the exact solution of the balance system (its rates differ from these by
    what its solve lost, no more)."""
    g = load(mech)
    M = oracle.Mech(mech)
    for i, T in enumerate(g["T"]):
        tol = 1e-12
        if mech not in PINNED:
            ex = exact_solve(M.qss_system(g["sc"][i], T))
            tol = max(tol, 2.0 * np.max(np.abs(g["sc_qss"][i] - ex) / np.abs(ex)))
        w = M.production_rate(g["sc"][i], T)
        scale = M.production_rate_abs(g["sc"][i], T)
        err = np.abs(w - g["wdot"][i])
        assert np.all(err <= tol * scale + 1e-300), (i, tol, np.max(err / (scale + 1e-300)))


@pytest.mark.parametrize("mech", ALL)
def test_qss_thermo_matches_reference(oracle, mech):
    g = load(mech)
    M = oracle.Mech(mech)
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
@pytest.mark.parametrize("mech", PINNED)
def test_qss_reactor_rhs_matches_reference(oracle, rtype, mech):
    """fKernelSpec over the QSS productionRate: species rates within 1e-10
    of their gross rates, the T row within 1e-9 of its scale."""
    g = load(mech)
    M = oracle.Mech(mech)
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
    the reference's mechanism files (every mechanism the generator lists)."""
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


def _reference_balances(path):
    """Per QSS species of a generated comp_sc_qss: the (term, coefficient)
    lists of its production, loss and each coupling, term = 2 k (+1 for q_r)."""
    text = open(path).read()
    a = text.index("comp_sc_qss(amrex::Real* sc_qss")
    b = text.index("// Putting it all together", a)
    blocks = re.split(r"QSSA species (\d+): (\S+)", text[a:b])[1:]
    out = {}
    for i in range(0, len(blocks), 3):
        d = {"num": [], "den": [], "cpl": []}
        for st in blocks[i + 2].split(";"):
            if "amrex::Real" not in st:
                continue
            lhs, rhs = st.split("=", 1)
            lhs = lhs.replace("amrex::Real", "").strip()
            terms = [(2 * int(k) + (1 if w == "qr" else 0), float(c) if c else 1.0)
                     for c, w, k in re.findall(r"(?:(\d+\.\d+)\s*\*\s*)?(q[fr])_co\[(\d+)\]", rhs)]
            if lhs.endswith("_num"):
                d["num"] = terms
            elif lhs.endswith("_denom"):
                d["den"] = terms
            elif not lhs.endswith("_rhs"):
                d["cpl"].append(sorted(terms))
        out[int(blocks[i])] = d
    return out


@pytest.mark.parametrize("mech", ALL)
def test_qss_balance_structure_matches_reference(oracle, mech):
    """The generated tables' balance terms are those of the reference's
    generated comp_sc_qss, term for term and in order (a removed forward
    rate, 0 there, is left out here)."""
    from pelephysics_b200.mechgen import ceptr_tables as ct

    root = oracle.reference_root()
    if root is None or not os.path.isdir(os.path.join(root, "Mechanisms")):
        pytest.skip("needs the reference tree")
    M = ct.build(os.path.join(root, "Mechanisms", mech), mech)
    qi = M["qss_info"]
    removed = {k for k, pos in enumerate(qi["q_rx"]) if M["rxns"][pos]["rmf"]}
    ref = _reference_balances(os.path.join(root, "Mechanisms", mech, "mechanism.H"))
    assert sorted(ref) == list(range(len(M["qss"])))
    keep = lambda lst: [(t, c) for t, c in lst if not (t % 2 == 0 and t // 2 in removed)]
    for q in range(len(M["qss"])):
        mine = {"num": [], "den": [], "cpl": {}}
        for t in range(qi["q_off"][q], qi["q_off"][q + 1]):
            term, role, c = qi["q_term"][t], qi["q_role"][t], qi["q_coef"][t]
            if role == -1:
                mine["num"].append((term, c))
            elif role == -2:
                mine["den"].append((term, c))
            else:
                mine["cpl"].setdefault(role, []).append((term, c))
        assert keep(ref[q]["num"]) == mine["num"], q
        assert [t for t, _ in keep(ref[q]["den"])] == [t for t, _ in mine["den"]], q
        assert sorted(keep(c) for c in ref[q]["cpl"]) == sorted(sorted(v) for v in mine["cpl"].values()), q

