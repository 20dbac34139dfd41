"""Transport coefficients on the GPU (ppb_transport, ppb_transport_box)
against the reference's compiled SimpleTransport (golden fixtures) and the
oracle's restatement.  Bar: 1e-13 relative (the kernel and the reference
differ only in the order of the mixture sums and in the last bit of exp)."""

import os

import numpy as np
import pytest

from pelephysics_b200 import transport as tr

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
MECHS = ["LiDryer", "drm19", "dodecane_lu", "heptane_lu_88sk"]


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


def soa(torch, Y, pad=5):
    """[ncells, N] -> species-major [N, ncells + pad] on the device."""
    n, N = Y.shape
    out = torch.full((N, n + pad), np.nan, dtype=torch.float64, device="cuda")
    out[:, :n] = torch.as_tensor(Y.T)
    return out


@pytest.mark.parametrize("mech", MECHS)
def test_flat_matches_reference_golden(cuda, mech):
    torch = cuda
    g = np.load(os.path.join(HERE, "golden", f"transport_{mech}.npz"))
    n = g["T"].shape[0]
    out = tr.transport(mech, torch.as_tensor(g["T"], device="cuda"), torch.as_tensor(g["rho"], device="cuda"),
                       soa(torch, g["Y"]), tr.TR_ALL)
    torch.cuda.synchronize()
    D = out["D"].cpu().numpy()[:, :n].T
    chi = out["chi"].cpu().numpy()[:, :n].T
    assert rel(D, g["D"]) <= 1e-13
    for k in ("mu", "xi", "lam"):
        assert rel(out[k].cpu().numpy(), g[k]) <= 1e-13, k
    light = g["chi"] != 0.0
    assert np.array_equal(chi != 0.0, light)
    assert rel(chi[light], g["chi"][light]) <= 1e-12


@pytest.mark.parametrize("mech,n", [("drm19", 1000), ("heptane_lu_88sk", 100)])
def test_flat_matches_oracle_on_a_batch(cuda, oracle, mech, n):
    torch = cuda
    N = oracle.Mech(mech).nsp
    rng = np.random.default_rng(5)
    T = rng.uniform(300.0, 3000.0, n)
    rho = 10.0 ** rng.uniform(-5, -1, n)
    Y = rng.uniform(size=(n, N)) ** 3
    Y[rng.uniform(size=(n, N)) < 0.2] = 0.0
    Y /= Y.sum(1, keepdims=True)
    out = tr.transport(mech, torch.as_tensor(T, device="cuda"), torch.as_tensor(rho, device="cuda"), soa(torch, Y, 0))
    D = out["D"].cpu().numpy().T
    for c in range(0, n, max(1, n // 50)):
        Dr, chir, mur, xir, lamr = oracle.transport(mech, oracle.TR_ALL, T[c], rho[c], Y[c])
        assert rel(D[c], Dr) <= 1e-13
        assert rel(out["mu"][c].item(), mur) <= 1e-13 and rel(out["lam"][c].item(), lamr) <= 1e-13
        assert rel(out["xi"][c].item(), xir) <= 1e-13


def test_flag_subsets_and_empty(cuda):
    torch = cuda
    mech = "drm19"
    g = np.load(os.path.join(HERE, "golden", f"transport_{mech}.npz"))
    T = torch.as_tensor(g["T"], device="cuda")
    rho = torch.as_tensor(g["rho"], device="cuda")
    Y = soa(torch, g["Y"])
    full = tr.transport(mech, T, rho, Y)
    only_d = tr.transport(mech, T, rho, Y, tr.TR_DIAG)
    assert set(only_d) == {"D"} and torch.equal(only_d["D"][:, :T.shape[0]], full["D"][:, :T.shape[0]])
    xi_alone = tr.transport(mech, T, rho, Y, tr.TR_XI)
    assert torch.all(xi_alone["xi"] == 0)  # the bulk viscosity comes with mu only
    lam = tr.transport(mech, T, rho, Y, tr.TR_LAM)
    assert torch.equal(lam["lam"], full["lam"])
    e = torch.zeros((21, 0), dtype=torch.float64, device="cuda")
    z = torch.zeros(0, dtype=torch.float64, device="cuda")
    assert tr.transport(mech, z, z, e)["D"].numel() == 0


@pytest.mark.parametrize("use_soret", [False, True])
def test_box_path_with_ghost_cells(cuda, use_soret):
    """get_transport_coeffs on the interior of allocations with 2 ghost
    cells: the interior equals the flat path on the same cells, the ghosts
    are untouched, and chi is written only with use_soret."""
    torch = cuda
    mech = "LiDryer"
    N, g = 9, 2
    nx, ny, nz = 7, 5, 3
    rng = np.random.default_rng(9)
    shape = (nz + 2 * g, ny + 2 * g, nx + 2 * g)
    T = torch.as_tensor(rng.uniform(400.0, 2500.0, (1,) + shape), device="cuda")
    rho = torch.as_tensor(rng.uniform(1e-4, 1e-3, (1,) + shape), device="cuda")
    Yh = rng.uniform(size=(N,) + shape)
    Yh /= Yh.sum(0, keepdims=True)
    Y = torch.as_tensor(Yh, device="cuda")
    sentinel = -7.0
    D = torch.full((N,) + shape, sentinel, dtype=torch.float64, device="cuda")
    chi = torch.full((N,) + shape, sentinel, dtype=torch.float64, device="cuda")
    mu, xi, lam = (torch.full((1,) + shape, sentinel, dtype=torch.float64, device="cuda") for _ in range(3))
    alo = (-g, -g, -g)
    lo, hi = (0, 0, 0), (nx - 1, ny - 1, nz - 1)
    tr.transport_box(mech, lo, hi, Y, T, rho, D, chi, mu, xi, lam, use_soret=use_soret, alloc_lo=alo)
    torch.cuda.synchronize()
    inner = (slice(None), slice(g, g + nz), slice(g, g + ny), slice(g, g + nx))
    Tf = T[inner].reshape(-1).contiguous()
    rf = rho[inner].reshape(-1).contiguous()
    Yf = Y[inner].reshape(N, -1).contiguous()
    flat = tr.transport(mech, Tf, rf, Yf, tr.TR_ALL if use_soret else tr.TR_ALL & ~tr.TR_CHI)
    assert torch.equal(D[inner].reshape(N, -1), flat["D"])
    for name, t in (("mu", mu), ("xi", xi), ("lam", lam)):
        assert torch.equal(t[inner].reshape(-1), flat[name]), name
    if use_soret:
        assert torch.equal(chi[inner].reshape(N, -1), flat["chi"])
    else:
        assert torch.all(chi == sentinel)
    mask = torch.ones(shape, dtype=torch.bool, device="cuda")
    mask[inner[1:]] = False
    for t in (D, mu, xi, lam):
        assert torch.all(t[:, mask] == sentinel)
