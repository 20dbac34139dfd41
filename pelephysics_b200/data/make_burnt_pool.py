"""Generate drm19_burnt_pool.npz: burnt drm19 compositions for the 64^3 field.

Each of 256 premixed CH4/air cells (phi evenly spaced in [0.6, 1.4], 1 atm,
1700 K) is integrated for 1 ms at constant volume with the FP64 CPU oracle
(rtol 1e-8, atol 1e-10, BDF order <= 5); the resulting mass fractions are the
"equilibrium-like" compositions the field's burnt cells take.  Run from the
repository root: python -m pelephysics_b200.data.make_burnt_pool
"""

import os

import numpy as np

from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    M = po.Mech("drm19")
    sp = [s.lower() for s in M.species()]
    mw = M.mw()
    N = M.nsp
    phis = np.linspace(0.6, 1.4, 256)
    rY = np.zeros((256, N + 1))
    rX = np.zeros(256)
    for c, phi in enumerate(phis):
        X = np.zeros(N)
        xo = 1.0 / (1.0 + 3.76 + phi / 2.0)
        X[sp.index("o2")], X[sp.index("n2")], X[sp.index("ch4")] = xo, 3.76 * xo, phi / 2.0 * xo
        Y = X * mw / np.sum(X * mw)
        rho = M.ckrhoy(1013250.0, 1700.0, Y)
        rY[c, :N] = rho * Y
        rY[c, N] = 1700.0
        rX[c] = rho * M.ckubms(1700.0, Y)
    flag, _, st = po.react_flat("drm19", 1, rY, np.zeros((256, N)), rX, np.zeros(256), 1e-3, rtol=1e-8,
                                atol=1e-10, max_order=5)
    assert flag == 0, flag
    Yb = np.clip(rY[:, :N], 0.0, None)
    Yb /= Yb.sum(axis=1, keepdims=True)
    np.savez_compressed(os.path.join(HERE, "drm19_burnt_pool.npz"), phi=phis, Y=Yb, T_end=rY[:, N])
    print("T after 1 ms:", rY[:, N].min(), rY[:, N].max())


if __name__ == "__main__":
    main()
