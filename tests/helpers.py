"""Shared test helpers: premixed initial states built with the CPU oracle."""

import numpy as np

FUELS = {"LiDryer": ("H2", 0.5), "drm19": ("CH4", 2.0), "dodecane_lu": ("NC12H26", 18.5),
         "heptane_lu_88sk": ("nc7h16", 11.0), "CH4_lean_qss": ("CH4", 2.0), "C1-C2-NO_qss": ("CH4", 2.0),
         "LuEthylene_qss": ("C2H4", 3.0), "grimech30": ("CH4", 2.0),
         "FFCM1_Red": ("CH4", 2.0), "chem-H": ("H2", 0.5)}
P_ATM = 1013250.0


def premix_oracle(po, mech, ncells, seed, T0, dT, phi0, dphi, P=P_ATM, reactor_type=1):
    """YCOrder cells (rY with T in the last slot, rhoE) from the oracle's EOS."""
    M = po.Mech(mech)
    sp = [s.lower() for s in M.species()]
    mw = M.mw()
    fuel, nu = FUELS[mech]
    rng = np.random.default_rng(seed)
    T = T0 + dT * rng.uniform(size=ncells)
    phi = phi0 + dphi * rng.uniform(size=ncells)
    N = M.nsp
    rY = np.zeros((ncells, N + 1))
    rX = np.zeros(ncells)
    for c in range(ncells):
        X = np.zeros(N)
        xo = 1.0 / (1.0 + 3.76 + phi[c] / nu)
        X[sp.index("o2")] = xo
        X[sp.index("n2")] = 3.76 * xo
        X[sp.index(fuel.lower())] = phi[c] / nu * xo
        Y = X * mw / np.sum(X * mw)
        rho = M.ckrhoy(P, T[c], Y)
        e = M.ckubms(T[c], Y) if reactor_type == 1 else M.ckhbms(T[c], Y)
        rY[c, :N] = rho * Y
        rY[c, N] = T[c]
        rX[c] = rho * e
    return rY, np.zeros((ncells, N)), rX, np.zeros(ncells)
