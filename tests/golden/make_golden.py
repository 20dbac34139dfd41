"""Generate the pointwise golden vectors from the reference's own kernels.

Runs in a container that has the reference tree: it compiles
Mechanisms/<mech>/mechanism.H through oracle/build_ref.sh and evaluates the
reference's generated functions (productionRate, aJacobian in both consP
modes, CKUBMS/CKHBMS/CKCVBS/CKCPBS, CKUMS/CKHMS, gibbs, GET_T_GIVEN_EY/HY)
on seeded random states, and the reference's SimpleTransport::transport
(Source/Transport/Simple.H, compiled by oracle/build_ref.sh with the
mechanism's transport fits) on seeded (T, rho, Y), and the reference's
SRK equation of state (Source/Eos/SRK.H) on seeded (rho, T, Y), and a QSS
mechanism's productionRate with the QSS concentrations it solves.  The .npz files it writes
are the committed fixtures the tests compare the CPU oracle and the CUDA
kernels against.

Usage: python tests/golden/make_golden.py [point|transport|srk|qss|<mech>]   (default all)
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402

POINTS = {"LiDryer": 16, "drm19": 16, "dodecane_lu": 6, "heptane_lu_88sk": 4, "grimech30": 8,
          "FFCM1_Red": 12, "chem-H": 12}


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


TRANSPORT_POINTS = {"LiDryer": 24, "drm19": 24, "dodecane_lu": 12, "heptane_lu_88sk": 8}


def transport_main():
    for seed, (mech, npts) in enumerate(TRANSPORT_POINTS.items()):
        N = po.Mech(mech).nsp
        rng = np.random.default_rng(2000 + seed)
        T = rng.uniform(300.0, 3000.0, npts)
        rho = 10.0 ** rng.uniform(-5, -1, npts)
        Y = rng.uniform(0.0, 1.0, (npts, N)) ** 4
        Y[rng.uniform(size=(npts, N)) < 0.15] = 0.0
        Y /= Y.sum(axis=1, keepdims=True)
        res = [po.ref_transport(mech, po.TR_ALL, T[i], rho[i], Y[i]) for i in range(npts)]
        out = {"T": T, "rho": rho, "Y": Y, "D": np.array([r[0] for r in res]), "chi": np.array([r[1] for r in res]),
               "mu": np.array([r[2] for r in res]), "xi": np.array([r[3] for r in res]),
               "lam": np.array([r[4] for r in res])}
        path = os.path.join(HERE, f"transport_{mech}.npz")
        np.savez_compressed(path, **out)
        print(mech, npts, os.path.getsize(path), "bytes")


SRK_POINTS = {"LiDryer": 16, "drm19": 16, "dodecane_lu": 8, "heptane_lu_88sk": 6}


def srk_main():
    """The reference's compiled Source/Eos/SRK.H on seeded (rho, T, Y):
    RTY2E, RTY2Cv, RTY2Ei, RTY2C, RTY2WDOT, REY2T (from T + 100 K) and the
    e-reactor right-hand side over them."""
    for seed, (mech, npts) in enumerate(SRK_POINTS.items()):
        R = po.Srk(mech, ref=True)
        N = R.N
        rng = np.random.default_rng(3000 + seed)
        T = rng.uniform(300.0, 2500.0, npts)
        rho = 10.0 ** rng.uniform(-4, -0.7, npts)
        Y = rng.uniform(0.0, 1.0, (npts, N)) ** 3
        Y /= Y.sum(axis=1, keepdims=True)
        src = rng.normal(size=(npts, N)) * 1e-2
        rhoesrc = rng.normal(size=npts) * 1e5
        out = {"T": T, "rho": rho, "Y": Y, "src": src, "rhoesrc": rhoesrc}
        out["e"] = np.array([R.rty2e(rho[i], T[i], Y[i]) for i in range(npts)])
        out["cv"] = np.array([R.rty2cv(rho[i], T[i], Y[i]) for i in range(npts)])
        out["ei"] = np.array([R.rty2ei(rho[i], T[i], Y[i]) for i in range(npts)])
        out["c"] = np.array([R.rty2c(rho[i], T[i], Y[i]) for i in range(npts)])
        out["wdot"] = np.array([R.rty2wdot(rho[i], T[i], Y[i]) for i in range(npts)])
        out["T_ey"] = np.array([R.rey2t(rho[i], out["e"][i], Y[i], T[i] + 100.0) for i in range(npts)])
        y = np.c_[rho[:, None] * Y, T + 30.0]
        out["y"] = y
        rhs = [R.reactor_rhs(2e-7, y[i], rho[i] * out["e"][i], rhoesrc[i], src[i]) for i in range(npts)]
        out["ydot"] = np.array([r[0] for r in rhs])
        path = os.path.join(HERE, f"srk_{mech}.npz")
        np.savez_compressed(path, **out)
        print(mech, npts, os.path.getsize(path), "bytes")


QSS_POINTS = {"CH4_lean_qss": 32, "C1-C2-NO_qss": 24, "LuEthylene_qss": 24}


def qss_main():
    """A QSS mechanism's compiled mechanism.H on seeded states: its
    productionRate (with the QSS concentrations it solves, comp_sc_qss),
    thermo, GET_T_GIVEN_EY/HY and the reactor right-hand side of both
    reactor types over them (its aJacobian needs CEPTR's symbolic build and
    is not used: the engine differences the right-hand side, as the
    reference's dense_direct solve does)."""
    for seed, (mech, npts) in enumerate(QSS_POINTS.items()):
        R = po.Ref(mech)
        N = R.nsp
        nq = po.Mech(mech).nqss
        T, sc, Y = states(N, npts, 4000 + seed)
        out = {"T": T, "sc": sc, "Y": Y, "mw": R.mw(), "imw": R.imw()}
        out["wdot"] = np.array([R.production_rate(sc[i], T[i]) for i in range(npts)])
        out["sc_qss"] = np.array([R.qss_concentrations(sc[i], T[i], nq) for i in range(npts)])
        out["gibbs"] = np.array([R.gibbs(t) for t in T])
        out["ums"] = np.array([R.ckums(t) for t in T])
        out["hms"] = np.array([R.ckhms(t) for t in T])
        out["ubms"] = np.array([R.ckubms(T[i], Y[i]) for i in range(npts)])
        out["hbms"] = np.array([R.ckhbms(T[i], Y[i]) for i in range(npts)])
        out["cvbs"] = np.array([R.ckcvbs(T[i], Y[i]) for i in range(npts)])
        out["cpbs"] = np.array([R.ckcpbs(T[i], Y[i]) for i in range(npts)])
        Tguess = T + np.where(T > 1900.0, -150.0, 150.0)
        out["Tguess"] = Tguess
        out["T_ey"] = np.array([R.t_given_ey(out["ubms"][i], Y[i], Tguess[i])[0] for i in range(npts)])
        out["T_hy"] = np.array([R.t_given_hy(out["hbms"][i], Y[i], Tguess[i])[0] for i in range(npts)])
        # reactor right-hand side (SI-free CGS state rho Y, T) with sources
        rng = np.random.default_rng(5000 + seed)
        rho = 10.0 ** rng.uniform(-4, -2, npts)
        y = np.c_[rho[:, None] * Y, T + 20.0]
        src = rng.normal(size=(npts, N)) * 1e-3
        rhoesrc = rng.normal(size=npts) * 1e4
        out.update({"rho": rho, "y": y, "src": src, "rhoesrc": rhoesrc})
        for rt, key in ((1, "ubms"), (2, "hbms")):
            rhoe = rho * out[key]
            out[f"rhoe{rt}"] = rhoe
            res = [R.reactor_rhs(rt, 1e-7, y[i], rhoe[i], rhoesrc[i], src[i]) for i in range(npts)]
            out[f"ydot{rt}"] = np.array([r[0] for r in res])
        path = os.path.join(HERE, f"point_{mech}.npz")
        np.savez_compressed(path, **out)
        print(mech, npts, os.path.getsize(path), "bytes")


def main():
    po.build()
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("all", "transport"):
        transport_main()
    if what in ("all", "srk"):
        srk_main()
    if what in ("all", "qss"):
        qss_main()
    if what in ("transport", "srk", "qss"):
        return
    # `python make_golden.py <mech>` writes that mechanism's point file only
    for seed, (mech, npts) in enumerate(POINTS.items()):
        if what not in ("all", "point") and what != mech:
            continue
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
