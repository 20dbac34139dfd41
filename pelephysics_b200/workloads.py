"""Seeded synthetic reacting fields with the shapes of the benchmark configs.

The reference has no public input fields for this path (its drivers build
cells from an initial condition or a plotfile, Testing/Exec/ReactEval/
main.cpp:204-387), so the benchmark cases are generated here from a fixed
recipe:

* ``premix_cells``: per-cell T = T0 + dT U(0,1) then phi = phi0 + dphi U(0,1)
  (numpy default_rng(seed), drawn in that order), fuel/O2/N2 mole fractions
  with 3.76 N2 per O2 at pressure P (1 atm by default), density and energy
  from the ideal gas (CKRHOY, CKUBMS/CKHBMS) -- the LiDryer 16^3 case uses it
  directly;
* ``fourier_field``: a [0,1]-normalised sum of random 3-D Fourier modes
  (integer wave vectors in [1,4]^3, phases U(0, 2 pi), unit amplitudes);
* ``drm19_field``: drm19 at 64^3: T = 1100 + 1100 s(x) with s the 8-mode
  field of seed 1, phi = 0.6 + 0.8 U, P = 1 atm; cells with s > 0.7 are
  burnt: they take the composition of a premixed cell of the nearest phi
  that was integrated for 1 ms at constant volume from 1700 K (the 256-entry
  pool data/drm19_burnt_pool.npz, made by data/make_burnt_pool.py), at the
  cell's own T;
* ``dodecane_field``: dodecane_lu on 128 x 128 x 64 (1,048,576 cells),
  P = 40 atm, T = 700 + 600 s(x) with s seed-2 white noise smoothed by a
  Gaussian of sigma = 4 cells (periodic, by FFT) and [0,1]-normalised,
  phi = 0.5 + 1.5 U, and advective species sources rYsrc_k ~ N(0,
  (1e-3 rho Y_k / dt)^2) made mass-conserving by subtracting
  Y_k sum_j rYsrc_j; dt = 2e-6 s;
* ``heptane_cells``: heptane_lu_88sk, 262,144 cells, P = 20 atm,
  T = 750 + 650 U, phi = 0.3 + 1.7 U (seed 5), dt = 1e-5 s (rtol 1e-8,
  atol 1e-12 in the benchmark).

Mass fractions are YCOrder per cell; energies are rho*e (reactor type 1) or
rho*h (type 2).  Density and energy come from an EOS callable
``eos(T, Y, P, reactor_type) -> (rho, rho*e)``; the default is the engine's
device EOS (Fuego PYT2RE on the GPU).
"""

from __future__ import annotations

import os

import numpy as np

from . import _lib

P_ATM = 1013250.0  # dyn/cm^2

# fuel species and O2 per unit fuel for the shipped mechanisms
FUELS = {
    "LiDryer": ("H2", 0.5),
    "drm19": ("CH4", 2.0),
    "dodecane_lu": ("NC12H26", 18.5),
    "heptane_lu_88sk": ("nc7h16", 11.0),
    "CH4_lean_qss": ("CH4", 2.0),
    "C1-C2-NO_qss": ("CH4", 2.0),
    "LuEthylene_qss": ("C2H4", 3.0),
    "grimech30": ("CH4", 2.0),
    "FFCM1_Red": ("CH4", 2.0),
    "chem-H": ("H2", 0.5),
}


def mole_fractions(mech, phi, species):
    """Fuel/O2/N2 premix: X_fuel = phi X_O2 / nu_O2, X_N2 = 3.76 X_O2."""
    fuel, nu = FUELS[mech]
    low = [s.lower() for s in species]
    i_f, i_o, i_n = low.index(fuel.lower()), low.index("o2"), low.index("n2")
    phi = np.asarray(phi, float)
    xo = 1.0 / (1.0 + 3.76 + phi / nu)
    X = np.zeros(phi.shape + (len(species),))
    X[..., i_o] = xo
    X[..., i_n] = 3.76 * xo
    X[..., i_f] = phi / nu * xo
    return X


def mass_fractions(X, mw):
    Y = X * mw
    return Y / Y.sum(axis=-1, keepdims=True)


def fourier_field(shape, nmodes, seed):
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 5, size=(nmodes, 3))
    ph = rng.uniform(0.0, 2 * np.pi, size=nmodes)
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")
    s = np.zeros(shape)
    for m in range(nmodes):
        s += np.cos(2 * np.pi * (k[m, 0] * x + k[m, 1] * y + k[m, 2] * z) + ph[m])
    s -= s.min()
    return s / s.max()


def _device_state(mech, T, Y, P, reactor_type, device):
    """rho, rho*e (or rho*h) on the device from T, Y at pressure P."""
    import torch

    from .reactor import pyt2re

    n = T.shape[0]
    Td = torch.as_tensor(T, dtype=torch.float64, device=device)
    Yd = torch.as_tensor(np.ascontiguousarray(Y), dtype=torch.float64, device=device)
    Pd = torch.full((n,), float(P), dtype=torch.float64, device=device)
    rho, e = pyt2re(mech, Pd, Td, Yd, eh=1 if reactor_type == 2 else 0)
    torch.cuda.synchronize()
    return rho.cpu().numpy(), (rho * e).cpu().numpy()


class Cells:
    """Flat YCOrder batch: rY [n, N+1] (rhoY then T), rYsrc [n, N], rX, rX_src."""

    def __init__(self, mech, rY, rYsrc, rX, rX_src, reactor_type, dt, meta=None):
        self.mech = mech
        self.rY = np.ascontiguousarray(rY)
        self.rYsrc = np.ascontiguousarray(rYsrc)
        self.rX = np.ascontiguousarray(rX)
        self.rX_src = np.ascontiguousarray(rX_src)
        self.reactor_type = reactor_type
        self.dt = dt
        self.meta = meta or {}

    @property
    def ncells(self):
        return self.rX.shape[0]

    def copy(self):
        return Cells(self.mech, self.rY.copy(), self.rYsrc.copy(), self.rX.copy(), self.rX_src.copy(),
                     self.reactor_type, self.dt, dict(self.meta))


def device_eos(mech, device="cuda"):
    return lambda T, Y, P, rtype: _device_state(mech, T, Y, P, rtype, device)


def premix_cells(mech, ncells, seed, T0, dT, phi0, dphi, P=P_ATM, reactor_type=1, dt=1e-4, device="cuda",
                 eos=None, species=None, mw=None):
    species = species or _lib.species_names(mech)
    mw = _lib.molecular_weights(mech) if mw is None else mw
    eos = eos or device_eos(mech, device)
    rng = np.random.default_rng(seed)
    T = T0 + dT * rng.uniform(size=ncells)
    phi = phi0 + dphi * rng.uniform(size=ncells)
    Y = mass_fractions(mole_fractions(mech, phi, species), mw)
    rho, rhoE = eos(T, Y, P, reactor_type)
    N = len(species)
    rY = np.zeros((ncells, N + 1))
    rY[:, :N] = rho[:, None] * Y
    rY[:, N] = T
    return Cells(mech, rY, np.zeros((ncells, N)), rhoE, np.zeros(ncells), reactor_type, dt,
                 {"T": T, "phi": phi, "P": P})


def ch4_lean_qss(ncells=65536, device="cuda"):
    """The QSS workload: CH4_lean_qss (13 transported species, 4 in steady
    state) homogeneous e-reactors, T 1100-2100 K, phi 0.5-1.0 (seed 6),
    1 atm, dt 1e-5 s."""
    return premix_cells("CH4_lean_qss", ncells, 6, 1100.0, 1000.0, 0.5, 0.5, reactor_type=1, dt=1e-5, device=device)


def lidryer_16(device="cuda"):
    """LiDryer, 16^3 cells, T 1000-1400 K, phi 0.5-2, 1 atm, dt 1e-4 s (seed 0)."""
    return premix_cells("LiDryer", 16 ** 3, 0, 1000.0, 400.0, 0.5, 1.5, reactor_type=1, dt=1e-4, device=device)


def burnt_pool():
    """(phi, Y) of the committed burnt-composition pool for drm19."""
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "drm19_burnt_pool.npz"))
    return d["phi"], d["Y"]


def drm19_field(n=64, device="cuda", seed=1, burnt_threshold=0.7, eos=None, species=None, mw=None):
    """drm19 on an n^3 box: the 64^3 case of the benchmark (see module doc)."""
    mech = "drm19"
    species = species or _lib.species_names(mech)
    mw = _lib.molecular_weights(mech) if mw is None else mw
    eos = eos or device_eos(mech, device)
    N = len(species)
    s = fourier_field((n, n, n), 8, seed).reshape(-1)
    ncells = s.size
    rng = np.random.default_rng(seed)
    T = 1100.0 + 1100.0 * s
    phi = 0.6 + 0.8 * rng.uniform(size=ncells)
    Y = mass_fractions(mole_fractions(mech, phi, species), mw)
    burnt = s > burnt_threshold
    if burnt.any():
        pphi, pY = burnt_pool()
        idx = np.clip(np.rint((phi[burnt] - pphi[0]) / (pphi[-1] - pphi[0]) * (len(pphi) - 1)).astype(int), 0,
                      len(pphi) - 1)
        Y[burnt] = pY[idx]
    rho, rhoE = eos(T, Y, P_ATM, 1)
    rY = np.zeros((ncells, N + 1))
    rY[:, :N] = rho[:, None] * Y
    rY[:, N] = T
    return Cells(mech, rY, np.zeros((ncells, N)), rhoE, np.zeros(ncells), 1, 1e-5,
                 {"T": T, "phi": phi, "burnt": burnt, "s": s})


def drm19_adjoint(ncells=65536, device="cuda", eos=None, species=None, mw=None):
    """The adjoint workload: drm19 homogeneous reactors of the h/c_p type
    (constant rho), T = 1100 + 500 U, phi = 0.5 + 1.5 U (seed 3), 1 atm,
    integrated over 5e-4 s; loss weights (w_T, w_OH) ~ N(0, 1) from seed 4
    in meta["w"] (2 x ncells)."""
    cells = premix_cells("drm19", ncells, 3, 1100.0, 500.0, 0.5, 1.5, reactor_type=2, dt=5e-4, device=device,
                         eos=eos, species=species, mw=mw)
    cells.meta["w"] = np.random.default_rng(4).normal(size=(2, ncells))
    return cells


def smoothed_field(shape, seed, sigma):
    """White noise (default_rng(seed)) smoothed by a periodic Gaussian of
    standard deviation sigma cells, normalised to [0, 1]."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    k = [np.fft.fftfreq(m) for m in shape]
    kz, ky, kx = np.meshgrid(*k, indexing="ij")
    g = np.exp(-2.0 * (np.pi * sigma) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    s = np.real(np.fft.ifftn(np.fft.fftn(w) * g))
    s -= s.min()
    return s / s.max()


def dodecane_field(shape=(64, 128, 128), device="cuda", seed=2, sigma=4.0, eos=None, species=None, mw=None):
    """dodecane_lu on a 128 x 128 x 64 box (see module doc)."""
    mech = "dodecane_lu"
    species = species or _lib.species_names(mech)
    mw = _lib.molecular_weights(mech) if mw is None else mw
    eos = eos or device_eos(mech, device)
    N = len(species)
    dt = 2e-6
    s = smoothed_field(shape, seed, sigma).reshape(-1)
    ncells = s.size
    rng = np.random.default_rng(seed + 100)
    T = 700.0 + 600.0 * s
    phi = 0.5 + 1.5 * rng.uniform(size=ncells)
    Y = mass_fractions(mole_fractions(mech, phi, species), mw)
    P = 40.0 * P_ATM
    rho, rhoE = eos(T, Y, P, 1)
    rY = np.zeros((ncells, N + 1))
    rY[:, :N] = rho[:, None] * Y
    rY[:, N] = T
    src = rng.standard_normal((ncells, N)) * (1e-3 * rY[:, :N] / dt)
    src -= Y * src.sum(axis=1, keepdims=True)
    return Cells(mech, rY, src, rhoE, np.zeros(ncells), 1, dt, {"T": T, "phi": phi, "s": s, "P": P})


def heptane_cells(ncells=262144, device="cuda", seed=5, eos=None, species=None, mw=None):
    """heptane_lu_88sk, 64^3 cells (see module doc)."""
    return premix_cells("heptane_lu_88sk", ncells, seed, 750.0, 650.0, 0.3, 1.7, P=20.0 * P_ATM, reactor_type=1,
                        dt=1e-5, device=device, eos=eos, species=species, mw=mw)

