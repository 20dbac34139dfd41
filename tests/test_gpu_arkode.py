"""ReactorArkode on the GPU against the oracle's restatement of the same
batch-coupled ERK integration (oracle/arkode.c) on the same seeded batches.

Both integrate the batch as one problem with one adaptive step, so besides
the state they must agree on the step count and the number of right-hand-side
evaluations; the state agrees far inside the integration bar (only the
summation order of the batch norm and of the per-cell reductions differ)."""

import numpy as np
import pytest

from pelephysics_b200 import _lib
from pelephysics_b200.reactor import Reactor
from tests.helpers import premix_oracle

pytestmark = pytest.mark.gpu

REFERENCE_IDS = [20, 30, 31, 40, 41, 42, 43, 50, 51, 52, 53, 54, 60, 80]


def batch(oracle, mech, nc, seed=3, T0=1000.0, dT=400.0, P=1013250.0):
    rY, src, rX, rXs = premix_oracle(oracle, mech, nc, seed, T0, dT, 0.5, 1.5, P=P)
    rng = np.random.default_rng(seed + 100)
    src = np.ascontiguousarray(rng.standard_normal(src.shape) * 1e-3 * rY[:, :-1] / 1e-5)
    rXs = rng.standard_normal(nc) * 1e-3 * np.abs(rX) / 1e-5
    return rY, src, rX, rXs


def compare(y, ref, T_rtol=1e-9, Y_atol=1e-11):
    N = ref.shape[1] - 1
    assert np.all(np.isfinite(y))
    dT = np.max(np.abs(y[:, N] - ref[:, N]) / ref[:, N])
    Yg = y[:, :N] / y[:, :N].sum(1, keepdims=True)
    Yr = ref[:, :N] / ref[:, :N].sum(1, keepdims=True)
    assert dT <= T_rtol, f"max rel T difference {dT:.3e}"
    assert np.abs(Yg - Yr).max() <= Y_atol, f"max abs Y difference {np.abs(Yg - Yr).max():.3e}"


@pytest.mark.parametrize("mech,dt,nc", [("LiDryer", 2e-6, 64), ("drm19", 1e-6, 40)])
def test_flat_path_matches_oracle(cuda, oracle, mech, dt, nc):
    """Host flat path: the default table (ZONNEVELD_5_3_4) and PID whatever
    rk_method / rk_controller say, as the reference's flat react does."""
    rY, src, rX, rXs = batch(oracle, mech, nc)
    opts = dict(rtol=1e-8, atol=1e-10)
    ref, xr = rY.copy(), rX.copy()
    flag, st = oracle.react_arkode(mech, 1, ref, src, xr, rXs, dt, **opts)
    assert flag == 0
    r = Reactor(mech, "ReactorArkode")
    r.init(1, nc, **opts, rk_method=80, rk_controller=2)
    y, x = rY.copy(), rX.copy()
    cost, dtr, t, code = r.react(y, src.copy(), x, rXs.copy(), dt, 0.5)
    assert code == 0 and dtr == dt and t == 0.5 + dt
    assert cost == st["nfe"]
    stats = r.cell_stats(nc)
    assert np.all(stats[:, 0] == st["nst"]) and np.all(stats[:, 5] == st["netf"])
    compare(y, ref)
    np.testing.assert_allclose(x, xr, rtol=1e-15, atol=0)


@pytest.mark.parametrize("tid", REFERENCE_IDS)
def test_box_path_every_table(cuda, oracle, tid):
    """Box path: rk_method selects the table and rk_controller the controller
    (each table with one of the four controllers), with masked cells."""
    torch = cuda
    mech, rtype, dt = "LiDryer", 1, 2e-6
    nx, ny, nz = 4, 3, 2
    n = nx * ny * nz
    ctl = REFERENCE_IDS.index(tid) % 4
    rY, src, rX, rXs = batch(oracle, mech, n, seed=tid)
    N = rY.shape[1] - 1
    M = oracle.Mech(mech)
    mask = np.ones(n, np.int32)
    mask[[2, 7]] = -1
    # the flatten step starts T from the stored value and recomputes it from
    # the energy; the oracle starts from the same recomputed T
    T0 = np.array([M.t_given_ey(rX[c] / rY[c, :N].sum(), rY[c, :N] / rY[c, :N].sum(), rY[c, N])[0]
                   for c in range(n)])
    y0 = rY.copy()
    y0[:, N] = T0
    opts = dict(rtol=1e-8, atol=1e-10)
    ref, xr = y0.copy(), rX.copy()
    flag, st = oracle.react_arkode(mech, rtype, ref, src, xr, rXs, dt, rk_method=tid, rk_controller=ctl, mask=mask,
                                   **opts)
    assert flag == 0
    r = Reactor(mech, "ReactorArkode")
    r.init(rtype, n, **opts, rk_method=tid, rk_controller=ctl)

    def box(a, nc):
        return torch.as_tensor(np.ascontiguousarray(a.T.reshape(nc, nz, ny, nx)), device="cuda")

    bY, bS = box(rY[:, :N], N), box(src, N)
    bT, bE, bEs = box(rY[:, N:], 1), box(rX[:, None], 1), box(rXs[:, None], 1)
    bFC = torch.zeros((1, nz, ny, nx), dtype=torch.float64, device="cuda")
    bM = torch.as_tensor(mask.reshape(1, nz, ny, nx), device="cuda")
    dtr, t, code = r.react_box((0, 0, 0), (nx - 1, ny - 1, nz - 1), bY, bS, bT, bE, bEs, bFC, bM, dt_react=dt)
    assert code == 0 and dtr == dt
    outY = bY.cpu().numpy().reshape(N, n).T
    outT = bT.cpu().numpy().reshape(n)
    outE = bE.cpu().numpy().reshape(n)
    outFC = bFC.cpu().numpy().reshape(n)
    on = mask == 1
    np.testing.assert_array_equal(outY[~on], rY[~on, :N])
    assert np.all(outFC[~on] == 0.0) and np.all(outFC[on] == st["nfe"])
    compare(np.c_[outY[on], ref[on, N]], ref[on])
    np.testing.assert_allclose(outE[on], xr[on], rtol=1e-15, atol=0)
    # unflatten: T from the new energy, starting from the integrated T
    for c in np.nonzero(on)[0]:
        Tn, _ = M.t_given_ey(outE[c] / outY[c].sum(), outY[c] / outY[c].sum(), ref[c, N])
        assert abs(outT[c] - Tn) <= 1e-9 * Tn


def test_device_path_and_typical_values(cuda, oracle):
    """Device flat path (energies advanced in place by the kernel) with
    typical values scaling atol: the host path's bits and the oracle's
    answer with the same absolute tolerances."""
    torch = cuda
    mech, dt, nc = "drm19", 1e-6, 96
    rY, src, rX, rXs = batch(oracle, mech, nc, seed=11)
    N = rY.shape[1] - 1
    typ = np.r_[np.full(N, 1e-3), 1e3]
    opts = dict(rtol=1e-7, atol=1e-9)
    ref, xr = rY.copy(), rX.copy()
    flag, st = oracle.react_arkode(mech, 1, ref, src, xr, rXs, dt, atolv=typ * opts["atol"], **opts)
    assert flag == 0
    rh = Reactor(mech, "ReactorArkode")
    rh.init(1, nc, **opts)
    rh.set_typ_vals_ode(typ)
    yh, xh = rY.copy(), rX.copy()
    rh.react(yh, src.copy(), xh, rXs.copy(), dt)
    rd = Reactor(mech, "ReactorArkode")
    rd.init(1, nc, **opts)
    rd.set_typ_vals_ode(typ)
    yd = torch.as_tensor(rY, device="cuda").contiguous()
    xd = torch.as_tensor(rX, device="cuda")
    cost, dtr, t, code = rd.react(yd, torch.as_tensor(src, device="cuda"), xd, torch.as_tensor(rXs, device="cuda"), dt)
    assert code == 0 and cost == st["nfe"]
    np.testing.assert_array_equal(yd.cpu().numpy(), yh)
    np.testing.assert_allclose(xd.cpu().numpy(), xh, rtol=1e-15, atol=0)
    compare(yh, ref)


def test_step_cap_reports_the_interval_reached(cuda, oracle):
    """arkode_max_steps reached: PPB_E_INTEGRATE, every cell flagged
    too-much-work, dt_react = the time reached (the reference's MOD_REACTOR
    bookkeeping) and rX advanced by it; the state is the oracle's at the same
    step."""
    mech, dt, nc = "drm19", 1e-5, 16
    rY, src, rX, rXs = batch(oracle, mech, nc, seed=5, T0=1400.0)
    opts = dict(rtol=1e-8, atol=1e-10)
    ref, xr = rY.copy(), rX.copy()
    flag, st = oracle.react_arkode(mech, 1, ref, src, xr, rXs, dt, max_steps=4, **opts)
    assert flag == -1 and st["t"] < dt
    r = Reactor(mech, "ReactorArkode")
    r.init(1, nc, **opts, arkode_max_steps=4)
    y, x = rY.copy(), rX.copy()
    cost, dtr, t, code = r.react(y, src.copy(), x, rXs.copy(), dt, raise_on_fail=False)
    assert code == _lib.PPB_E_INTEGRATE
    # the initial-step estimate differences f(y0 + hg f0) - f0 at a tiny hg,
    # which magnifies the last-bit differences of the two right-hand sides:
    # the few steps taken agree to ~1e-8, not to the last bit
    assert abs(dtr - st["t"]) <= 1e-6 * st["t"] and t == dtr
    stt, _ = r.cell_status(nc)
    assert np.all(stt == -1)
    compare(y, ref, T_rtol=1e-6, Y_atol=1e-8)
    np.testing.assert_allclose(x, rX + dtr * rXs, rtol=1e-15, atol=0)


@pytest.mark.parametrize("mech,tid,dt,nc,P", [("dodecane_lu", 80, 2e-7, 12, 40 * 1013250.0),
                                               ("heptane_lu_88sk", 40, 1e-8, 8, 20 * 1013250.0)])
def test_large_mechanisms(cuda, oracle, mech, tid, dt, nc, P):
    """The largest stage count (13, Fehlberg 8(7)) on dodecane_lu and the
    default table on heptane_lu_88sk (shared workspace 89 KB and 120 KB per
    block; heptane at 20 atm is stable only below ~5e-12 s steps for the
    explicit scheme, hence the 1e-8 s interval)."""
    torch = cuda
    rY, src, rX, rXs = batch(oracle, mech, nc, seed=7, T0=900.0, P=P)
    N = rY.shape[1] - 1
    M = oracle.Mech(mech)
    T0 = np.array([M.t_given_ey(rX[c] / rY[c, :N].sum(), rY[c, :N] / rY[c, :N].sum(), rY[c, N])[0]
                   for c in range(nc)])
    y0 = rY.copy()
    y0[:, N] = T0
    opts = dict(rtol=1e-8, atol=1e-12)
    ref, xr = y0.copy(), rX.copy()
    flag, st = oracle.react_arkode(mech, 1, ref, src, xr, rXs, dt, rk_method=tid, max_steps=5000, **opts)
    assert flag == 0
    r = Reactor(mech, "ReactorArkode")
    r.init(1, nc, **opts, rk_method=tid, arkode_max_steps=5000)
    nx = nc
    bY = torch.as_tensor(np.ascontiguousarray(rY[:, :N].T.reshape(N, 1, 1, nx)), device="cuda")
    bS = torch.as_tensor(np.ascontiguousarray(src.T.reshape(N, 1, 1, nx)), device="cuda")
    bT = torch.as_tensor(rY[:, N].reshape(1, 1, 1, nx).copy(), device="cuda")
    bE = torch.as_tensor(rX.reshape(1, 1, 1, nx).copy(), device="cuda")
    bEs = torch.as_tensor(rXs.reshape(1, 1, 1, nx).copy(), device="cuda")
    bFC = torch.zeros((1, 1, 1, nx), dtype=torch.float64, device="cuda")
    dtr, t, code = r.react_box((0, 0, 0), (nx - 1, 0, 0), bY, bS, bT, bE, bEs, bFC, dt_react=dt)
    assert code == 0
    outY = bY.cpu().numpy().reshape(N, nc).T
    assert np.all(bFC.cpu().numpy() == st["nfe"])
    compare(np.c_[outY, ref[:, N]], ref, Y_atol=1e-10)


def test_empty_batch_and_all_masked(cuda, oracle):
    torch = cuda
    r = Reactor("LiDryer", "ReactorArkode")
    r.init(1, 0)
    e = np.zeros((0, 10))
    cost, dt, t, code = r.react(e, np.zeros((0, 9)), np.zeros(0), np.zeros(0), 1e-5, 1.0, ncells=0)
    assert code == 0 and cost == 0 and abs(t - (1.0 + 1e-5)) < 1e-15
    # a box whose every cell is masked: nothing integrates, the time advances
    rY, src, rX, rXs = batch(oracle, "LiDryer", 4)
    N = rY.shape[1] - 1
    r.init(1, 4)
    bY = torch.as_tensor(np.ascontiguousarray(rY[:, :N].T.reshape(N, 1, 1, 4)), device="cuda")
    keep = bY.clone()
    one = lambda a: torch.as_tensor(np.ascontiguousarray(a).reshape(1, 1, 1, 4), device="cuda")
    bFC = torch.ones((1, 1, 1, 4), dtype=torch.float64, device="cuda")
    bM = torch.full((1, 1, 1, 4), -1, dtype=torch.int32, device="cuda")
    bS = torch.as_tensor(np.ascontiguousarray(src.T.reshape(N, 1, 1, 4)), device="cuda")
    dtr, t, code = r.react_box((0, 0, 0), (3, 0, 0), bY, bS, one(rY[:, N]), one(rX), one(rXs), bFC, bM,
                               dt_react=1e-6)
    assert code == 0 and dtr == 1e-6
    assert torch.equal(bY, keep) and torch.all(bFC == 0)


def test_grid_barrier_bound_runs_out_and_the_next_call_is_clean(cuda, oracle):
    """The cooperative launch's grid barrier gives up after arkode_barrier_us.
    With a bound of 0 a block that has to wait gives up at once: the call ends
    (no hang) with PPB_E_CUDA and the timeout message.  The same reactor, given
    the default bound again, then reproduces a fresh reactor's result bit for
    bit (the barrier words are cleared before every launch)."""
    mech, dt, nc = "drm19", 1e-6, 4096
    rY, src, rX, rXs = batch(oracle, mech, nc, seed=11)
    opts = dict(rtol=1e-8, atol=1e-10)
    r = Reactor(mech, "ReactorArkode")
    r.init(1, nc, **opts, arkode_barrier_us=0)
    with pytest.raises(_lib.EngineError, match="grid barrier timed out"):
        r.react(rY.copy(), src.copy(), rX.copy(), rXs.copy(), dt)
    r.init(1, nc, **opts)
    y, x = rY.copy(), rX.copy()
    _, _, _, code = r.react(y, src.copy(), x, rXs.copy(), dt)
    assert code == 0
    fresh = Reactor(mech, "ReactorArkode")
    fresh.init(1, nc, **opts)
    yf, xf = rY.copy(), rX.copy()
    fresh.react(yf, src.copy(), xf, rXs.copy(), dt)
    assert np.array_equal(y, yf) and np.array_equal(x, xf)
    with pytest.raises(_lib.EngineError):
        Reactor(mech, "ReactorArkode").init(1, nc, arkode_barrier_us=-1)
