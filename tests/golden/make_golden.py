"""Generate the pointwise golden vectors from the reference's own kernels.

Runs in a container that has the reference tree: it compiles
Mechanisms/<mech>/mechanism.H through oracle/build_ref.sh and evaluates the
reference's generated functions (productionRate, aJacobian in both consP
modes, CKUBMS/CKHBMS/CKCVBS/CKCPBS, CKUMS/CKHMS, gibbs, GET_T_GIVEN_EY/HY)
on seeded random states.  The .npz files it writes are the committed
fixtures the tests compare the CPU oracle and the CUDA kernels against.

Usage: python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402

POINTS = {"LiDryer": 16, "drm19": 16, "dodecane_lu": 6, "heptane_lu_88sk": 4}


def states(nsp, npts, seed):
    rng = np.random.default_rng(seed)
    T = rng.uniform(300.0, 3500.0, npts)
    # keep clear of the NASA-7 mid-point where the polynomial switches
    T[np.abs(T - 1000.0) < 1.0] += 5.0
    # SI concentrations spanning seven decades, some exactly zero
    sc = rng.uniform(0.0, 1.0, (npts, nsp)) * 10.0 ** rng.uniform(-6, 1, (npts, nsp))
    sc[rng.uniform(size=(npts, nsp)) < 0.1] = 0.0
    Y = rng.uniform(0.0, 1.0, (npts, nsp)) ** 3
    Y /= Y.sum(axis=1, keepdims=True)
    return T, sc, Y


def main():
    po.build()
    for seed, (mech, npts) in enumerate(POINTS.items()):
        R = po.Ref(mech)
        N = R.nsp
        T, sc, Y = states(N, npts, 1000 + seed)
        out = {"T": T, "sc": sc, "Y": Y, "mw": R.mw(), "imw": R.imw()}
        out["wdot"] = np.array([R.production_rate(sc[i], T[i]) for i in range(npts)])
        out["jac0"] = np.array([R.ajacobian(sc[i], T[i], 0) for i in range(npts)])
        out["jac1"] = np.array([R.ajacobian(sc[i], T[i], 1) for i in range(npts)])
        out["gibbs"] = np.array([R.gibbs(t) for t in T])
        out["ums"] = np.array([R.ckums(t) for t in T])
        out["hms"] = np.array([R.ckhms(t) for t in T])
        out["ubms"] = np.array([R.ckubms(T[i], Y[i]) for i in range(npts)])
        out["hbms"] = np.array([R.ckhbms(T[i], Y[i]) for i in range(npts)])
        out["cvbs"] = np.array([R.ckcvbs(T[i], Y[i]) for i in range(npts)])
        out["cpbs"] = np.array([R.ckcpbs(T[i], Y[i]) for i in range(npts)])
        # temperature from energy: target energies at T, Newton started 150 K away
        Tguess = T + np.where(T > 1900.0, -150.0, 150.0)
        out["Tguess"] = Tguess
        out["T_ey"] = np.array([R.t_given_ey(out["ubms"][i], Y[i], Tguess[i])[0] for i in range(npts)])
        out["T_hy"] = np.array([R.t_given_hy(out["hbms"][i], Y[i], Tguess[i])[0] for i in range(npts)])
        path = os.path.join(HERE, f"point_{mech}.npz")
        np.savez_compressed(path, **out)
        print(mech, npts, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
