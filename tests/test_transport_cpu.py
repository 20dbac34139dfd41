"""Transport coefficients on the CPU: the oracle's restatement of the
reference's SimpleTransport against the golden outputs of the reference's
own compiled Simple.H (tests/golden/transport_<mech>.npz), flag subsets, and
the generated tables."""

import os

import numpy as np
import pytest

from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
MECHS = ["LiDryer", "drm19", "dodecane_lu", "heptane_lu_88sk"]


def golden(mech):
    return np.load(os.path.join(HERE, "golden", f"transport_{mech}.npz"))


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("mech", MECHS)
def test_oracle_matches_reference_transport(oracle, mech):
    g = golden(mech)
    for c in range(g["T"].shape[0]):
        D, chi, mu, xi, lam = oracle.transport(mech, oracle.TR_ALL, g["T"][c], g["rho"][c], g["Y"][c])
        assert rel(D, g["D"][c]) <= 1e-13
        assert rel(mu, g["mu"][c]) <= 1e-13 and rel(xi, g["xi"][c]) <= 1e-13 and rel(lam, g["lam"][c]) <= 1e-13
        light = g["chi"][c] != 0.0
        assert np.array_equal(chi != 0.0, light)
        assert rel(chi[light], g["chi"][c][light]) <= 1e-12


@pytest.mark.parametrize("mech", ["LiDryer", "heptane_lu_88sk"])
def test_flag_subsets(oracle, mech):
    g = golden(mech)
    T, rho, Y = g["T"][0], g["rho"][0], g["Y"][0]
    full = oracle.transport(mech, oracle.TR_ALL, T, rho, Y)
    D, chi, mu, xi, lam = oracle.transport(mech, oracle.TR_DIAG, T, rho, Y)
    np.testing.assert_array_equal(D, full[0])
    assert mu == 0.0 and xi == 0.0 and lam == 0.0 and not chi.any()
    # xi only with mu (Simple.H computes the bulk viscosity inside the mu branch)
    assert oracle.transport(mech, oracle.TR_XI, T, rho, Y)[3] == 0.0
    assert oracle.transport(mech, oracle.TR_XI | oracle.TR_MU, T, rho, Y)[3] == full[3]
    assert oracle.transport(mech, oracle.TR_LAM, T, rho, Y)[4] == full[4]


def test_binary_diffusion_fits_are_symmetric():
    """COFD_ij == COFD_ji bit for bit in every shipped mechanism."""
    import re

    for mech in MECHS:
        path = os.path.join(os.path.dirname(HERE), "pelephysics_b200", "csrc", "mech", f"trans_{mech}.h")
        txt = open(path).read()
        body = re.search(r"ppbt_" + mech + r"_fitdbin\[\] = \{(.*?)\};", txt, re.S).group(1)
        v = np.array([float(x) for x in body.replace("\n", " ").split(",") if x.strip()])
        N = int(round(np.sqrt(v.size / 4)))
        c = v.reshape(N, N, 4)  # [j][i][q]: index 4 (i + N j)
        np.testing.assert_array_equal(c, c.transpose(1, 0, 2))


@pytest.mark.skipif(po.reference_root() is None, reason="needs the reference tree")
def test_tables_regenerate_identically(tmp_path):
    from pelephysics_b200.mechgen import transport_tables as tt

    for mech in MECHS:
        T = tt.build(os.path.join(po.reference_root(), "Mechanisms", mech), mech)
        out = tmp_path / f"trans_{mech}.h"
        tt.emit_header(T, str(out))
        ship = os.path.join(os.path.dirname(HERE), "pelephysics_b200", "csrc", "mech", f"trans_{mech}.h")
        assert out.read_text() == open(ship).read()
