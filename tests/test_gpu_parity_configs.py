"""Integration parity on the benchmark configurations themselves, against the
oracle over the reference's own compiled mechanism kernels (oracle/_ref):

* the drm19 64^3 field (unburnt, igniting and burnt cells; dt 1e-5 s,
  rtol = atol = 1e-10, BDF orders <= 5), the same seeded 8,192-cell sample
  the benchmark reports, for the tuned engine (FP64 LU and FP32 factor with
  FP64 refinement) and the plain per-cell engine;
* the LiDryer 16^3 = 4,096-cell configuration (dt 1e-4 s, rtol = atol =
  1e-10), every cell, orders <= 5 and the reference default <= 2.

The bar is T within 1e-6 relative and Y_k within 1e-8 absolute.  A cell whose
mass fractions differ by more than 1e-8 from the oracle's is held to 16
replicas of the oracle whose right-hand-side values are moved by at most one
ulp (compare_to_reference in oracle/pyoracle.py): at rtol = 1e-10 the CVODE
algorithm takes a different step sequence on some cells when its arithmetic
changes in the last bit, and those sequences end up to 6.5e-8 apart in Y
(the oracle over a table-driven restatement of the reference's kernels is
that far from the oracle over the kernels themselves, on the same cells).
Such a cell passes when it lies within 1e-8 of a replica or within the
replicas' spread around the reference (a cell that does neither gets 256
more replicas: slowly igniting LiDryer cells take 317 to 417 steps under
such changes); at most 0.5 % of the cells may need that, and none may be
further than 1e-7 from the reference.  With the reference's default
max_order = 2 the LiDryer cells agree to ~1e-12 with no such cell.
"""

import numpy as np
import pytest
import torch

from pelephysics_b200 import workloads as wl
from pelephysics_b200.reactor import Reactor

pytestmark = pytest.mark.gpu

OPTS = dict(rtol=1e-10, atol=1e-10)


def _sample(ncells, n):
    """The benchmark's oracle sample of the 64^3 field."""
    return np.sort(np.random.default_rng(7).permutation(ncells)[:n])


def _gpu_react(cells, opts, idx=None, integ="ReactorCvode"):
    rY = cells.rY if idx is None else cells.rY[idx]
    src = cells.rYsrc if idx is None else cells.rYsrc[idx]
    rX = cells.rX if idx is None else cells.rX[idx]
    rXs = cells.rX_src if idx is None else cells.rX_src[idx]
    r = Reactor(cells.mech, integ)
    r.init(cells.reactor_type, rX.shape[0], **opts)
    y = torch.as_tensor(np.ascontiguousarray(rY), device="cuda")
    s = torch.as_tensor(np.ascontiguousarray(src), device="cuda")
    x = torch.as_tensor(np.ascontiguousarray(rX), device="cuda")
    xs = torch.as_tensor(np.ascontiguousarray(rXs), device="cuda")
    cost, dt, t, code = r.react(y, s, x, xs, cells.dt)
    torch.cuda.synchronize()
    status, _ = r.cell_status(rX.shape[0])
    r.close()
    assert code == 0 and (status == 0).all()
    return y.cpu().numpy()


def _oracle(oracle, cells, idx, opts):
    y = np.ascontiguousarray(cells.rY[idx])
    flag, _, st = oracle.react_flat(cells.mech, cells.reactor_type, y, np.ascontiguousarray(cells.rYsrc[idx]),
                                    cells.rX[idx].copy(), cells.rX_src[idx].copy(), cells.dt, use_ref_kernels=1,
                                    **opts)
    assert flag == 0
    return y


def _check(oracle, cells, idx, y_gpu, y_ref, opts, max_over_frac=0.005):
    r = oracle.compare_to_reference(cells.mech, cells.reactor_type, cells.rY[idx], cells.rYsrc[idx], cells.rX[idx],
                                    cells.rX_src[idx], cells.dt, y_gpu, y_ref, use_ref_kernels=1, **opts)
    assert r["max_rel_T"] <= 1e-6, r
    assert r["cells_failing"] == 0, r
    assert r["cells_over_Y_atol"] <= max_over_frac * r["cells"], r
    assert r["max_abs_Y"] <= 1e-7, r
    return r


@pytest.fixture(scope="module")
def drm19_field():
    return wl.drm19_field(64, device="cuda")


@pytest.fixture(scope="module")
def drm19_oracle(oracle, drm19_field):
    idx = _sample(drm19_field.ncells, 8192)
    return idx, _oracle(oracle, drm19_field, idx, dict(max_order=5, **OPTS))


@pytest.mark.parametrize("extra", [dict(), dict(lu_fp32=1, refine_sweeps=1)], ids=["fp64_lu", "fp32_factor"])
def test_drm19_field_tuned_vs_reference_kernels(cuda, oracle, drm19_field, drm19_oracle, extra):
    idx, y_ref = drm19_oracle
    assert drm19_field.meta["burnt"][idx].any() and (~drm19_field.meta["burnt"][idx]).any()
    opts = dict(max_order=5, **OPTS)
    y = _gpu_react(drm19_field, dict(engine=1, **opts, **extra))
    _check(oracle, drm19_field, idx, y[idx], y_ref, opts)


def test_drm19_field_plain_vs_reference_kernels(cuda, oracle, drm19_field, drm19_oracle):
    idx, y_ref = drm19_oracle
    opts = dict(max_order=5, **OPTS)
    y = _gpu_react(drm19_field, dict(engine=0, **opts), idx=idx)
    _check(oracle, drm19_field, idx, y, y_ref, opts)


@pytest.mark.parametrize("engine", [1, 0], ids=["tuned", "plain"])
@pytest.mark.parametrize("max_order", [5, 2])
def test_lidryer_16cubed_vs_reference_kernels(cuda, oracle, engine, max_order):
    cells = wl.lidryer_16(device="cuda")
    assert cells.ncells == 4096 and cells.dt == 1e-4
    idx = np.arange(cells.ncells)
    opts = dict(max_order=max_order, **OPTS)
    y_ref = _oracle(oracle, cells, idx, opts)
    y = _gpu_react(cells, dict(engine=engine, **opts))
    _check(oracle, cells, idx, y, y_ref, opts)



# Mechanisms of the reference that run on kernels compiled for another
# mechanism of the same species count: (mechanism, cells, T0, dT, phi0, dphi)
# of premixed e-reactors at 1 atm, dt 1e-5 s.
MORE_MECHS = {
    "grimech30": (256, 1100.0, 1000.0, 0.5, 1.0),  # GRI-Mech 3.0, 53 species, 325 reactions
    "FFCM1_Red": (256, 1100.0, 1000.0, 0.5, 1.0),  # 21 species, 124 reactions
    "chem-H": (256, 1000.0, 400.0, 0.5, 1.5),  # 9 species, 27 reactions
}


@pytest.mark.parametrize("engine", ["tuned", "tuned_fp32", "plain"])
@pytest.mark.parametrize("mech", list(MORE_MECHS))
def test_more_mechanisms_premixed_vs_reference_kernels(cuda, oracle, mech, engine):
    """A mechanism with its own tables on the kernels of its species count
    (Lindemann and Troe fall-off and explicit third bodies among its
    reactions): premixed e-reactors at rtol = atol = 1e-10 against the
    oracle integrator over the reference's compiled kernels of that
    mechanism (Mechanisms/<mech>/mechanism.H)."""
    n, T0, dT, phi0, dphi = MORE_MECHS[mech]
    cells = wl.premix_cells(mech, n, 8, T0, dT, phi0, dphi, reactor_type=1, dt=1e-5)
    idx = np.arange(n)
    opts = dict(OPTS, engine=0 if engine == "plain" else 1)
    if engine == "tuned_fp32":
        opts["lu_fp32"] = 1
    y_gpu = _gpu_react(cells, opts)
    y_ref = _oracle(oracle, cells, idx, OPTS)
    _check(oracle, cells, idx, y_gpu, y_ref, OPTS)
