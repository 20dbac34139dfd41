"""GPU parity of the pointwise mechanism kernels, through the C ABI, against
the golden vectors of the reference's compiled kernels and the CPU oracle.

Tolerances (FP64 both sides; the sums are evaluated in a different order):
* rates: |wdot - ref| <= 1e-12 * sum_r |nu| (|q_f| + |q_r|) per species;
* Jacobian: Frobenius-relative <= 1e-12, and per-entry relative <= 1e-10
  for entries above 1e-6 of the largest;
* T from energy: relative <= 1e-12; reactor RHS: as the rates, scaled by
  the magnitude of the species terms."""

import os

import numpy as np
import pytest

from pelephysics_b200 import _lib
from tests.helpers import premix_oracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
MECHS = ["LiDryer", "drm19", "dodecane_lu", "heptane_lu_88sk", "grimech30", "FFCM1_Red", "chem-H"]


def load(mech):
    return dict(np.load(os.path.join(GOLD, f"point_{mech}.npz")))


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("mech", MECHS)
@pytest.mark.parametrize("team", [1, 32])
def test_production_rate(cuda, oracle, mech, team):
    torch = cuda
    g = load(mech)
    M = oracle.Mech(mech)
    n = g["T"].size
    N = M.nsp
    w = torch.zeros((n, N), dtype=torch.float64, device="cuda")
    sc, T = dev(torch, g["sc"]), dev(torch, g["T"])  # keep the inputs alive until the kernel ran
    _lib.check(_lib.lib().ppb_production_rate(mech.encode(), sc.data_ptr(), T.data_ptr(), w.data_ptr(), n, team,
                                              None))
    torch.cuda.synchronize()
    w = w.cpu().numpy()
    for i in range(n):
        scale = M.production_rate_abs(g["sc"][i], g["T"][i])
        err = np.abs(w[i] - g["wdot"][i])
        assert np.all(err <= 1e-12 * scale + 1e-300), (i, np.max(err / (scale + 1e-300)))


@pytest.mark.parametrize("mech", MECHS)
@pytest.mark.parametrize("team", [1, 32])
@pytest.mark.parametrize("consP", [0, 1])
def test_ajacobian(cuda, mech, team, consP):
    torch = cuda
    g = load(mech)
    n = g["T"].size
    nn = (g["sc"].shape[1] + 1) ** 2
    J = torch.zeros((n, nn), dtype=torch.float64, device="cuda")
    sc, T = dev(torch, g["sc"]), dev(torch, g["T"])
    _lib.check(_lib.lib().ppb_ajacobian(mech.encode(), sc.data_ptr(), T.data_ptr(), consP, J.data_ptr(), n, team,
                                        None))
    torch.cuda.synchronize()
    J = J.cpu().numpy()
    for i in range(n):
        ref = g[f"jac{consP}"][i]
        assert np.linalg.norm(J[i] - ref) <= 1e-12 * np.linalg.norm(ref)
        big = np.abs(ref) > 1e-6 * np.abs(ref).max()
        assert np.all(np.abs(J[i] - ref)[big] <= 1e-10 * np.abs(ref)[big])


@pytest.mark.parametrize("mech", MECHS)
@pytest.mark.parametrize("team", [1, 32])
def test_t_from_energy(cuda, mech, team):
    torch = cuda
    g = load(mech)
    n = g["T"].size
    for eh, key, ekey in ((0, "T_ey", "ubms"), (1, "T_hy", "hbms")):
        T = dev(torch, g["Tguess"])
        e, Y = dev(torch, g[ekey]), dev(torch, g["Y"])
        _lib.check(_lib.lib().ppb_t_from_energy(mech.encode(), eh, e.data_ptr(), Y.data_ptr(), T.data_ptr(), n, team,
                                                None))
        torch.cuda.synchronize()
        np.testing.assert_allclose(T.cpu().numpy(), g[key], rtol=1e-12)


@pytest.mark.parametrize("mech", ["LiDryer", "drm19", "dodecane_lu", "grimech30"])
@pytest.mark.parametrize("team", [1, 32])
@pytest.mark.parametrize("rtype", [1, 2])
def test_reactor_rhs(cuda, oracle, mech, team, rtype):
    torch = cuda
    ncells = 16
    rY, src, rX, rXs = premix_oracle(oracle, mech, ncells, 11, 900.0, 1500.0, 0.5, 1.0, reactor_type=rtype)
    rng = np.random.default_rng(3)
    src = rng.normal(0.0, 1e-3, src.shape) * rY[:, :-1] / 1e-5
    rXs = rng.normal(0.0, 1e3, ncells)
    rY[:, -1] += rng.uniform(-50, 50, ncells)  # Newton start away from the solution
    M = oracle.Mech(mech)
    N = M.nsp
    t = 3.0e-6
    out = torch.zeros((ncells, N + 1), dtype=torch.float64, device="cuda")
    d_y, d_x, d_xs, d_src = dev(torch, rY), dev(torch, rX), dev(torch, rXs), dev(torch, src)
    _lib.check(_lib.lib().ppb_reactor_rhs(mech.encode(), rtype, t, d_y.data_ptr(), d_x.data_ptr(), d_xs.data_ptr(),
                                          d_src.data_ptr(), out.data_ptr(), ncells, team, None))
    torch.cuda.synchronize()
    out = out.cpu().numpy()
    for c in range(ncells):
        ref, _ = M.reactor_rhs(rtype, t, rY[c], rX[c], rXs[c], src[c])
        scale = np.abs(ref[:N]).max()
        assert np.all(np.abs(out[c, :N] - ref[:N]) <= 1e-11 * scale)
        assert abs(out[c, N] - ref[N]) <= 1e-9 * abs(ref[N]) + 1e-11 * scale


@pytest.mark.parametrize("mech", MECHS)
def test_device_eos(cuda, oracle, mech):
    torch = cuda
    from pelephysics_b200.reactor import pyt2re

    g = load(mech)
    M = oracle.Mech(mech)
    n = g["T"].size
    P = np.full(n, 1013250.0 * 3)
    for eh in (0, 1):
        d_P, d_T, d_Y = dev(torch, P), dev(torch, g["T"]), dev(torch, g["Y"])
        rho, e = pyt2re(mech, d_P, d_T, d_Y, eh=eh)
        rho, e = rho.cpu().numpy(), e.cpu().numpy()
        for i in range(n):
            assert abs(rho[i] - M.ckrhoy(P[i], g["T"][i], g["Y"][i])) <= 1e-13 * rho[i]
            ref = M.ckhbms(g["T"][i], g["Y"][i]) if eh else M.ckubms(g["T"][i], g["Y"][i])
            assert abs(e[i] - ref) <= 1e-12 * abs(ref) + 1e-3
