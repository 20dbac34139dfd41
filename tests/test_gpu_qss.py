"""QSS mechanisms on the GPU, through the C ABI: CH4_lean_qss (13
transported species, 4 in quasi-steady state), C1-C2-NO_qss (39, 5; two
forward rates removed by the reduction), LuEthylene_qss (22, 10).

* pointwise: productionRate (one thread or one warp per cell) and the
  reactor right-hand side of both reactor types against the golden vectors
  of the reference's compiled mechanism.H for the two mechanisms pinned to
  it, and against the oracle for LuEthylene_qss (the reference's own
  elimination for its 10-species group loses accuracy on some states; the
  oracle is pinned to exact arithmetic, tests/test_qss_cpu.py), at the bars
  of the other mechanisms' pointwise tests (rates within 1e-12 of their
  gross rates);
* integration: react() (tuned BDF, difference-quotient Jacobian, as the
  reference's dense_direct solve) against the oracle's BDF over the
  reference's compiled kernels (over the table kernels for LuEthylene_qss),
  with the replica criterion (T 1e-6 relative, Y 1e-8 absolute,
  compare_to_reference) for cells whose step sequence parts in the last bit;
* block size: CH4_lean_qss runs 16 warps per block by default (sixteen
  cell workspaces fit one SM) and gives the same bits at 8;
* the option checks: a QSS mechanism runs on the tuned FP64 BDF only, and
  has no analytical Jacobian here."""

import os

import numpy as np
import pytest

from pelephysics_b200 import _lib
from pelephysics_b200.reactor import Reactor
from tests.helpers import premix_oracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
MECH = "CH4_lean_qss"


PINNED = ["CH4_lean_qss", "C1-C2-NO_qss"]
ALL = PINNED + ["LuEthylene_qss"]


def load(mech=MECH):
    return dict(np.load(os.path.join(GOLD, f"point_{mech}.npz")))


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("team", [1, 32])
@pytest.mark.parametrize("mech", ALL)
def test_qss_production_rate(cuda, oracle, team, mech):
    torch = cuda
    g = load(mech)
    M = oracle.Mech(mech)
    n, N = g["T"].size, M.nsp
    w = torch.zeros((n, N), dtype=torch.float64, device="cuda")
    sc, T = dev(torch, g["sc"]), dev(torch, g["T"])
    code = _lib.lib().ppb_production_rate(mech.encode(), sc.data_ptr(), T.data_ptr(), w.data_ptr(), n, team, None)
    if team == 1 and code != 0:
        pytest.skip("the one-thread pointwise buffer is too small for this mechanism")  # reported, not silent
    _lib.check(code)
    torch.cuda.synchronize()
    w = w.cpu().numpy()
    for i in range(n):
        scale = M.production_rate_abs(g["sc"][i], g["T"][i])
        ref = g["wdot"][i] if mech in PINNED else M.production_rate(g["sc"][i], g["T"][i])
        err = np.abs(w[i] - ref)
        assert np.all(err <= 1e-12 * scale + 1e-300), (i, np.max(err / (scale + 1e-300)))


@pytest.mark.parametrize("team", [1, 32])
@pytest.mark.parametrize("rtype", [1, 2])
@pytest.mark.parametrize("mech", PINNED)
def test_qss_reactor_rhs(cuda, oracle, team, rtype, mech):
    torch = cuda
    g = load(mech)
    M = oracle.Mech(mech)
    N = M.nsp
    n = g["T"].size
    mw = M.mw()
    out = torch.zeros((n, N + 1), dtype=torch.float64, device="cuda")
    d_y, d_x, d_xs, d_src = dev(torch, g["y"]), dev(torch, g[f"rhoe{rtype}"]), dev(torch, g["rhoesrc"]), \
        dev(torch, g["src"])
    code = _lib.lib().ppb_reactor_rhs(mech.encode(), rtype, 1e-7, d_y.data_ptr(), d_x.data_ptr(), d_xs.data_ptr(),
                                      d_src.data_ptr(), out.data_ptr(), n, team, None)
    if team == 1 and code != 0:
        pytest.skip("the one-thread pointwise buffer is too small for this mechanism")
    _lib.check(code)
    torch.cuda.synchronize()
    out = out.cpu().numpy()
    for i in range(n):
        y, ref = g["y"][i], g[f"ydot{rtype}"][i]
        rho = y[:N].sum()
        gross = M.production_rate_abs(y[:N] / mw * 1e6, g["T"][i]) * 1e-6 * mw
        assert np.all(np.abs(out[i, :N] - ref[:N]) <= 1e-10 * gross + 1e-12 * np.abs(g["src"][i]) + 1e-300), i
        assert abs(out[i, N] - ref[N]) <= 1e-9 * (abs(ref[N]) + abs(g["rhoesrc"][i]) / rho) + 1e-300, i


@pytest.mark.parametrize("mech,rtype,nc,dt", [("CH4_lean_qss", 1, 128, 1e-3), ("CH4_lean_qss", 2, 64, 2e-3),
                                               ("C1-C2-NO_qss", 1, 64, 1e-3), ("LuEthylene_qss", 1, 64, 5e-4)])
def test_qss_react_vs_reference_kernels(cuda, oracle, mech, rtype, nc, dt):
    """Lean premixed cells (T 1700..2100 K, phi 0.5..1.0) through ignition.
    The difference-quotient Jacobian carries rounding of the right-hand side
    amplified by 1 / increment (~1e8) into the Newton iteration, so more cells
    than with an analytical Jacobian part on another step sequence: the
    oracle over the table kernels and the oracle over the reference's kernels
    differ by up to 1.5e-8 in Y and 1.2e-7 in T on the CH4_lean_qss cells,
    and on 18 of the 64 C1-C2-NO_qss cells (slow NO chemistry) by up to
    3e-8 in Y.  Cells above either bar are judged against replicas of the
    reference (compare_to_reference, T and Y)."""
    use_ref = 1 if mech in PINNED else 0
    if use_ref and not oracle.have_ref(mech):
        pytest.skip("reference kernels not built")
    opts = dict(rtol=1e-10, atol=1e-10, max_order=5)
    rY, src, rX, rXs = premix_oracle(oracle, mech, nc, 6, 1700.0, 400.0, 0.5, 0.5, reactor_type=rtype)
    ref = rY.copy()
    flag, _, _ = oracle.react_flat(mech, rtype, ref, src, rX.copy(), rXs, dt, use_ref_kernels=use_ref, **opts)
    assert flag == 0
    r = Reactor(mech)
    r.init(rtype, nc, **opts)
    y = rY.copy()
    cost, _, _, code = r.react(y, src.copy(), rX.copy(), rXs.copy(), dt)
    assert code == 0 and cost > 0
    N = rY.shape[1] - 1
    assert np.max(np.abs(y[:, N] - rY[:, N])) > 10.0  # the cells ignite within dt
    res = oracle.compare_to_reference(mech, rtype, rY, src, rX, rXs, dt, y, ref, use_ref_kernels=use_ref, **opts)
    assert res["cells_failing"] == 0, res
    assert res["max_rel_T"] <= 1e-5 and res["max_abs_Y"] <= 1e-7, res


def test_qss_block_size_changes_no_bits(cuda, oracle):
    """The default launch of CH4_lean_qss is one 16-warp block per SM (one
    rendezvous for all its warps); 8-warp blocks give the same bits and the
    same per-cell counters, as block size only changes when a cell's warp
    runs."""
    nc, dt = 600, 1e-3
    rY, src, rX, rXs = premix_oracle(oracle, MECH, nc, 7, 1700.0, 400.0, 0.5, 0.5, reactor_type=1)
    outs, stats, picks = [], [], []
    for wpb in (0, 8):
        r = Reactor(MECH)
        r.init(1, nc, rtol=1e-10, atol=1e-10, max_order=5, warps_per_block=wpb)
        y = rY.copy()
        _, _, _, code = r.react(y, src.copy(), rX.copy(), rXs.copy(), dt)
        assert code == 0
        outs.append(y)
        stats.append(r.cell_stats(nc))
        picks.append(r.launch_config()[0])
    assert picks == [16, 8]
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(stats[0], stats[1])


def test_qss_option_checks(cuda):
    for integ, extra in (("ReactorRK64", {}), ("ReactorCvode", {"lu_fp32": 1}), ("ReactorCvode", {"engine": 0}),
                         ("ReactorArkode", {}), ("ReactorCvode", {"eos": 1}),
                         ("ReactorCvode", {"warps_per_block": 12})):
        r = Reactor(MECH, integ)
        with pytest.raises(_lib.EngineError):
            r.init(1, 4, **extra)
    # no analytical Jacobian for a QSS mechanism
    import torch

    sc = torch.ones((2, 13), dtype=torch.float64, device="cuda")
    T = torch.full((2,), 1200.0, dtype=torch.float64, device="cuda")
    J = torch.zeros((2, 14 * 14), dtype=torch.float64, device="cuda")
    code = _lib.lib().ppb_ajacobian(MECH.encode(), sc.data_ptr(), T.data_ptr(), 0, J.data_ptr(), 2, 32, None)
    assert code != 0
