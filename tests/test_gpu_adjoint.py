"""GPU checks of the engine's derivatives of react() (no reference
counterpart; the derivatives are checked against the CPU oracle).

* Pointwise: the exact Jacobian of the reactor right-hand side (T from the
  energy constraint), its energy column and its parameter derivatives
  against central finite differences of a CPU restatement of the RHS
  (oracle production rates and thermo, T solved to 1e-14; relative step
  1e-4): 1e-5 relative per column and row block.
* Integration: the discrete adjoint against the tangent-linear model on the
  same cells (dot-product identity to 1e-9 relative; both integrate
  through one compiled call site, so their trajectories agree bit for bit);
  the adjoint gradient independent of the checkpoint interval and of
  whether the reverse sweep reads the forward run's copy of a segment or
  recomputes it (bit for bit); the loss gradient against central
  finite differences (step 1e-6 relative) of the CPU oracle integrator at
  rtol = atol = 1e-13, 1e-2 relative on the dominant components.
"""

import numpy as np
import pytest

from pelephysics_b200 import adjoint as adj
from pelephysics_b200.reactor import Reactor
from tests.helpers import premix_oracle

pytestmark = pytest.mark.gpu

OPTS = dict(rtol=1e-10, atol=1e-10, max_order=5)


def rhs_tight(M, rtype, t, y, rhoe, rhoesrc, src):
    """fKernelSpec (ReactorUtils.H:358-415) on the CPU with T solved tightly."""
    N = M.nsp
    mw = M.mw()
    rho = y[:N].sum()
    Y = y[:N] / rho
    e = (rhoe + rhoesrc * t) / rho
    T = y[N]
    for _ in range(200):
        E = M.ckubms(T, Y) if rtype == 1 else M.ckhbms(T, Y)
        cv = M.ckcvbs(T, Y) if rtype == 1 else M.ckcpbs(T, Y)
        dT = (e - E) / cv
        T += dT
        if abs(dT) < 1e-14 * T:
            break
    cv = M.ckcvbs(T, Y) if rtype == 1 else M.ckcpbs(T, Y)
    sc = rho * Y / mw * 1e6
    wdot = M.production_rate(sc, T)
    ek = M.ckums(T) if rtype == 1 else M.ckhms(T)
    f = np.empty(N + 1)
    f[:N] = wdot * 1e-6 * mw + src
    f[N] = (rhoesrc - f[:N] @ ek) / (rho * cv)
    return f


def burnt_cells(oracle, mech, n, rtype, T0, dT, t_pre):
    """Premixed cells advanced t_pre with the oracle (radicals present)."""
    rY, src, rX, rXs = premix_oracle(oracle, mech, n, 3, T0, dT, 0.6, 1.0, reactor_type=rtype)
    if t_pre > 0:
        flag, _, _ = oracle.react_flat(mech, rtype, rY, src, rX.copy(), rXs, t_pre, **OPTS)
        assert flag == 0
    return rY, src, rX, rXs


@pytest.mark.parametrize("mech,rtype", [("LiDryer", 1), ("drm19", 1), ("drm19", 2)])
def test_rhs_exact_jacobian_fd(cuda, oracle, mech, rtype):
    torch = cuda
    nc = 3
    rY, src, rX, rXs = burnt_cells(oracle, mech, nc, rtype, 1300.0, 500.0, 2e-4)
    M = oracle.Mech(mech)
    N = M.nsp
    n = N + 1
    dev = "cuda"
    t = 0.0
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    f, J, fE, _, _, _ = adj.rhs_exact(mech, rtype, t, g(rY), g(rX), g(rXs), g(src))
    f, J, fE = f.cpu().numpy(), J.cpu().numpy(), fE.cpu().numpy()
    mw = M.mw()
    for c in range(nc):
        y = rY[c]
        f0 = rhs_tight(M, rtype, t, y, rX[c], rXs[c], src[c])
        # f against the rounding scale of the net rates (sum |nu| (|q_f| + |q_r|))
        rho = y[:N].sum()
        gross = M.production_rate_abs(y[:N] / mw * 1e6, y[N]) * 1e-6 * mw
        ek = M.ckums(y[N]) if rtype == 1 else M.ckhms(y[N])
        cv = M.ckcvbs(y[N], y[:N] / rho) if rtype == 1 else M.ckcpbs(y[N], y[:N] / rho)
        tol = 1e-7 * np.append(gross, gross @ np.abs(ek) / (rho * cv)) + 1e-300
        assert np.all(np.abs(f[c] - f0) <= tol), np.max(np.abs(f[c] - f0) / tol)
        # f does not depend on the T slot (T comes from the energy)
        assert np.all(J[c, N] == 0.0)
        for j in range(N):
            # step max(1e-4 |y_j|, 1e-6 rho): smaller steps on trace species
            # are swamped by the rounding of the net rates and of the T solve
            h = max(1e-4 * abs(y[j]), 1e-6 * rho)
            yp, ym = y.copy(), y.copy()
            yp[j] += h
            ym[j] -= h
            fd = (rhs_tight(M, rtype, t, yp, rX[c], rXs[c], src[c]) -
                  rhs_tight(M, rtype, t, ym, rX[c], rXs[c], src[c])) / (2 * h)
            col = J[c, j]
            floor = 1e-9 / max(abs(y[j]), 1e-6 * rho)
            # species rows and the T row have their own scales
            for rows in (slice(0, N), slice(N, n)):
                scale = np.abs(fd[rows]).max() + floor * np.abs(f0[rows]).max()
                err = np.abs(col[rows] - fd[rows]).max()
                assert err <= 1e-5 * scale, (c, j, rows, err, scale)
        h = 1e-6 * abs(rX[c])
        fd = (rhs_tight(M, rtype, t, y, rX[c] + h, rXs[c], src[c]) -
              rhs_tight(M, rtype, t, y, rX[c] - h, rXs[c], src[c])) / (2 * h)
        for rows in (slice(0, N), slice(N, n)):
            assert np.abs(fE[c][rows] - fd[rows]).max() <= 1e-5 * np.abs(fd[rows]).max() + 1e-30


@pytest.mark.parametrize("mech,rtype", [("drm19", 2)])
def test_rhs_param_vjp_fd(cuda, oracle, mech, rtype):
    torch = cuda
    nc = 2
    rY, src, rX, rXs = burnt_cells(oracle, mech, nc, rtype, 1400.0, 300.0, 2e-4)
    M = oracle.Mech(mech)
    N = M.nsp
    rng = np.random.default_rng(5)
    v = rng.normal(size=(nc, N + 1))
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    _, _, _, vy, vE, vp = adj.rhs_exact(mech, rtype, 0.0, g(rY), g(rX), g(rXs), g(src), v=g(v))
    vp = vp.cpu().numpy()
    A, b, e = oracle.arrhenius(mech)
    R = A.size
    L = oracle.lib()
    Mp = oracle.Mech(mech)

    def vf(c, A_, b_, e_):
        ptr = L.ppo_mech_with_arrhenius(mech.encode(), *(oracle._p(np.ascontiguousarray(x)) for x in (A_, b_, e_)))
        Mp.M = ptr
        try:
            return v[c] @ rhs_tight(Mp, rtype, 0.0, rY[c], rX[c], rXs[c], src[c])
        finally:
            L.ppo_mech_free(ptr)

    for c in range(nc):
        top = np.argsort(-np.abs(vp[c, :R]))[:6]
        for r in top:
            eps = 1e-6
            Ap, Am = A.copy(), A.copy()
            Ap[r] *= np.exp(eps)
            Am[r] *= np.exp(-eps)
            fd = (vf(c, Ap, b, e) - vf(c, Am, b, e)) / (2 * eps)
            assert abs(vp[c, r] - fd) <= 1e-5 * abs(fd) + 1e-12, ("lnA", c, r, vp[c, r], fd)
            bp, bm = b.copy(), b.copy()
            bp[r] += eps
            bm[r] -= eps
            fd = (vf(c, A, bp, e) - vf(c, A, bm, e)) / (2 * eps)
            assert abs(vp[c, R + r] - fd) <= 1e-5 * abs(fd) + 1e-12, ("beta", c, r)
            h = eps * max(abs(e[r]), 100.0)
            ep, em = e.copy(), e.copy()
            ep[r] += h
            em[r] -= h
            fd = (vf(c, A, b, ep) - vf(c, A, b, em)) / (2 * h)
            assert abs(vp[c, 2 * R + r] - fd) <= 1e-5 * abs(fd) + 1e-15, ("EaR", c, r)


def adjoint_setup(oracle, mech, rtype, nc, dt, interval=16, **kw):
    rY, src, rX, rXs = premix_oracle(oracle, mech, nc, 4, 1100.0, 500.0, 0.5, 1.5, reactor_type=rtype)
    r = Reactor(mech)
    r.init(rtype, nc, **OPTS, adjoint_checkpoint_interval=interval, **kw)
    return r, rY, src, rX, rXs


@pytest.mark.parametrize("mech,rtype,dt", [("LiDryer", 1, 1e-4), ("drm19", 2, 2e-4), ("drm19", 1, 1e-4)])
def test_adjoint_tangent_dot_product(cuda, oracle, mech, rtype, dt):
    torch = cuda
    nc = 24
    r, rY, src, rX, rXs = adjoint_setup(oracle, mech, rtype, nc, dt, interval=5)
    n = rY.shape[1]
    R = r.nrxn
    rng = np.random.default_rng(11)
    lam = rng.normal(size=(nc, n))
    dy0 = rng.normal(size=(nc, n)) * 1e-3 * np.abs(rY)
    dE = rng.normal(size=nc) * 1e-3 * np.abs(rX)
    dp = np.concatenate([rng.normal(size=R) * 1e-2, rng.normal(size=R) * 1e-3, rng.normal(size=R)])
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    ya, lam_y0, lam_e, grad = r.adjoint(g(rY), g(src), g(rX), g(rXs), dt, g(lam))
    yt, dy = r.tangent(g(rY), g(src), g(rX), g(rXs), dt, dy0=g(dy0), drX=g(dE), dparams=g(dp))
    ya, yt = ya.cpu().numpy(), yt.cpu().numpy()
    st, _ = r.cell_status(nc)
    assert np.all(st == 0)
    # the same discrete trajectory in both
    np.testing.assert_array_equal(ya, yt)
    # and the same integration as react() to its parity bar
    y = rY.copy()
    x = rX.copy()
    r.react(y, src.copy(), x, rXs.copy(), dt)
    np.testing.assert_allclose(ya[:, -1], y[:, -1], rtol=1e-6)
    lhs = np.sum(lam * dy.cpu().numpy())
    rhs = np.sum(lam_y0.cpu().numpy() * dy0) + np.sum(lam_e.cpu().numpy() * dE) + grad.cpu().numpy() @ dp
    terms = np.abs(lam * dy.cpu().numpy()).sum()
    assert abs(lhs - rhs) <= 1e-9 * terms, (lhs, rhs, terms)


def test_adjoint_checkpoint_interval_invariance(cuda, oracle):
    torch = cuda
    mech, rtype, dt, nc = "drm19", 2, 2e-4, 16
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    out = []
    for interval in (1, 3, 16, 1000):
        r, rY, src, rX, rXs = adjoint_setup(oracle, mech, rtype, nc, dt, interval=interval)
        lam = np.random.default_rng(2).normal(size=rY.shape)
        ya, ly0, le, gr = r.adjoint(g(rY), g(src), g(rX), g(rXs), dt, g(lam))
        out.append([t.cpu().numpy() for t in (ya, ly0, le, gr)])
        r.close()
    for o in out[1:]:
        for a, b in zip(out[0], o):
            np.testing.assert_array_equal(a, b)


def test_adjoint_segment_copies_change_no_bits(cuda, oracle):
    """The reverse sweep reads each segment from the forward run's copy, or,
    when the copies do not fit (a small adjoint_memory_mb) or are off
    (adjoint_keep_segments = 0), recomputes it from its checkpoint: the same
    records either way, so the same bits.  The small budgets leave room for
    some of the copies only (a budget too small for the checkpoints ends the
    call with an error, which is allowed here)."""
    from pelephysics_b200._lib import EngineError

    torch = cuda
    mech, rtype, dt, nc = "drm19", 2, 2e-4, 24
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    out = []
    for keep, mb in ((1, 16384), (0, 16384), (1, 12), (1, 8), (1, 6)):
        r, rY, src, rX, rXs = adjoint_setup(oracle, mech, rtype, nc, dt, interval=64, adjoint_keep_segments=keep,
                                            adjoint_memory_mb=mb)
        lam = np.random.default_rng(3).normal(size=rY.shape)
        try:
            ya, ly0, le, gr = r.adjoint(g(rY), g(src), g(rX), g(rXs), dt, g(lam))
        except EngineError:
            assert mb < 100
            r.close()
            continue
        st, _ = r.cell_status(nc)
        assert np.all(st == 0)
        out.append([t.cpu().numpy() for t in (ya, ly0, le, gr)])
        r.close()
    assert len(out) >= 3
    for o in out[1:]:
        for a, b in zip(out[0], o):
            np.testing.assert_array_equal(a, b)


@pytest.mark.slow
def test_adjoint_loss_gradient_vs_oracle_fd(cuda, oracle):
    """The adjoint workload's loss on a few cells against finite differences
    of the CPU oracle integrator, both at rtol = atol = 1e-13, for the
    largest gradients with respect to ln A, beta and Ea/R and two initial
    mass densities.

    * Central differences with the configuration's step, 1e-6 relative,
      within 1 %: at that step the differences of the adaptive integrator
      carry step-controller noise (a parameter change moves the step
      sequence; measured scatter 1e-4 .. 5e-3).
    * Richardson-extrapolated central differences, (4 D(h/2) - D(h)) / 3
      with h = 1e-3 relative, within 1e-4: the larger step puts the noise
      far below the truncation error, which the extrapolation removes to
      O(h^4) (measured worst 4.5e-5; 1.3e-5 with h = 3e-3)."""
    torch = cuda
    mech, rtype, t_end, nc = "drm19", 2, 5e-4, 6
    OPTS = dict(rtol=1e-13, atol=1e-13, max_order=5, max_steps=100000)
    rY, src, rX, rXs = premix_oracle(oracle, mech, nc, 4, 1100.0, 500.0, 0.5, 1.5, reactor_type=rtype)
    M = oracle.Mech(mech)
    ioh = [s.upper() for s in M.species()].index("OH")
    w = np.random.default_rng(4).normal(size=(2, nc))
    r = Reactor(mech)
    r.init(rtype, nc, **OPTS)
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    y = rY.copy()
    x = rX.copy()
    r.react(y, src.copy(), x, rXs.copy(), t_end)
    _, lam = adj.loss_T_OH(y, ioh, w[0], w[1])
    _, lam_y0, _, grad = r.adjoint(g(rY), g(src), g(rX), g(rXs), t_end, g(lam))
    grad, lam_y0 = grad.cpu().numpy(), lam_y0.cpu().numpy()
    A, b, e = oracle.arrhenius(mech)
    R = A.size

    def L_of(A_, b_, e_, y0=rY):
        yy = y0.copy()
        flag, _, _ = oracle.react_flat_arrhenius(mech, A_, b_, e_, rtype, yy, src, rX.copy(), rXs, t_end, **OPTS)
        assert flag == 0
        return adj.loss_T_OH(yy, ioh, w[0], w[1])[0]

    c = int(np.argmax(np.abs(lam_y0).sum(1)))
    sp = [s.upper() for s in M.species()]
    # (name, adjoint value, L as a function of a relative parameter change d)
    cases = []
    for r_ in np.argsort(-np.abs(grad[:R]))[:4]:
        cases.append((("lnA", r_), grad[r_], lambda d, r_=r_: L_of(np.where(np.arange(R) == r_, A * np.exp(d), A), b, e),
                      1.0))
    for r_ in np.argsort(-np.abs(grad[R:2 * R]))[:3]:
        sc = max(abs(b[r_]), 1.0)
        cases.append((("beta", r_), grad[R + r_], lambda d, r_=r_, sc=sc: L_of(A, b + sc * d * (np.arange(R) == r_), e),
                      sc))
    for r_ in np.argsort(-np.abs(grad[2 * R:]))[:3]:
        sc = max(abs(e[r_]), 100.0)
        cases.append((("EaR", r_), grad[2 * R + r_],
                      lambda d, r_=r_, sc=sc: L_of(A, b, e + sc * d * (np.arange(R) == r_)), sc))
    for k in (sp.index("CH4"), sp.index("O2")):
        sc = rY[c, k]

        def Ly(d, k=k, sc=sc):
            yp = rY.copy()
            yp[c, k] += sc * d
            return L_of(A, b, e, yp)

        cases.append((("y0", k), lam_y0[c, k], Ly, sc))
    for name, adj_val, f, sc in cases:
        fd6 = (f(1e-6) - f(-1e-6)) / (2e-6) / sc
        assert abs(adj_val - fd6) <= 1e-2 * abs(fd6), (name, adj_val, fd6)
        h = 1e-3
        d1 = (f(h) - f(-h)) / (2 * h)
        d2 = (f(h / 2) - f(-h / 2)) / h
        fdr = (4 * d2 - d1) / 3 / sc
        assert abs(adj_val - fdr) <= 1e-4 * abs(fdr), (name, adj_val, fdr)


def test_autograd_wrapper_matches_adjoint(cuda, oracle):
    torch = cuda
    mech, rtype, dt, nc = "LiDryer", 1, 1e-4, 8
    r, rY, src, rX, rXs = adjoint_setup(oracle, mech, rtype, nc, dt)
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    y0 = g(rY).requires_grad_(True)
    x0 = g(rX).requires_grad_(True)
    p = torch.as_tensor(adj.params_of(r), device="cuda").requires_grad_(True)
    y = adj.ReactFunction.apply(y0, x0, p, r, g(src), g(rXs), dt)
    w = torch.as_tensor(np.random.default_rng(1).normal(size=rY.shape), device="cuda")
    (y * w).sum().backward()
    _, ly0, le, gr = r.adjoint(g(rY), g(src), g(rX), g(rXs), dt, w)
    assert torch.equal(y0.grad, ly0) and torch.equal(x0.grad, le) and torch.equal(p.grad, gr)
