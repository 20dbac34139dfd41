"""ReactorArkode on the CPU: the explicit tables against the Butcher order
conditions, the generated C header against the tables, and the oracle's
restatement of the batch-coupled ERK integration (convergence against a
tight high-order solution, masks, the step cap)."""

import os

import numpy as np
import pytest

from pelephysics_b200 import erk_tables as et
from tests.helpers import premix_oracle

# ode.rk_method numbers the reference accepts (ReactorArkode.cpp:25-86)
REFERENCE_IDS = [20, 30, 31, 40, 41, 42, 43, 50, 51, 52, 53, 54, 60, 80]


def test_every_reference_method_has_a_table():
    assert sorted(et.TABLES) == REFERENCE_IDS
    assert et.DEFAULT == 40 and et.TABLES[40]["name"] == "ZONNEVELD_5_3_4"


@pytest.mark.parametrize("tid", REFERENCE_IDS)
def test_table_meets_order_conditions(tid):
    t = et.TABLES[tid]
    assert et.check_order(t), t["name"]
    # and not one order more (the stated orders are the true ones)
    higher = et.order_residuals(t, t["b"], t["q"] + 1)[-1]
    assert higher > 1e-6, t["name"]


def test_order_conditions_catch_a_wrong_coefficient():
    t = et.TABLES[52]
    bad = dict(t, A=[row[:] for row in t["A"]])
    bad["A"][3][1] += et.F(1, 10**6)
    bad["c"] = [sum(r) for r in bad["A"]]
    assert not et.check_order(bad)


def test_tree_counts():
    # rooted trees with 1..8 vertices (OEIS A000081)
    assert [len(et.trees(k)) for k in range(1, 9)] == [1, 1, 2, 4, 9, 20, 48, 115]


def test_header_is_generated_from_the_tables():
    with open(et.HEADER_PATH) as fh:
        assert fh.read() == et.header()


def _batch(oracle, mech, nc, seed=3):
    rY, src, rX, rXs = premix_oracle(oracle, mech, nc, seed, 1000.0, 400.0, 0.5, 1.5)
    return rY, np.ascontiguousarray(src), rX, rXs


def test_oracle_converges_with_rtol(oracle):
    """LiDryer igniting within the step: the default table's error against
    Fehlberg 8(7) at rtol 1e-13 falls with rtol."""
    mech, dt, nc = "LiDryer", 2e-5, 8
    rY, src, rX, rXs = premix_oracle(oracle, mech, nc, 3, 1400.0, 200.0, 0.5, 1.5)
    src = np.ascontiguousarray(src)
    ref = rY.copy()
    flag, _ = oracle.react_arkode(mech, 1, ref, src, rX.copy(), rXs, dt, rtol=1e-13, atol=1e-16, rk_method=80,
                                  max_steps=10**6)
    assert flag == 0
    assert np.min(ref[:, -1] - rY[:, -1]) > 500.0  # every cell ignites
    errs = []
    for rtol in (1e-5, 1e-7, 1e-9):
        y = rY.copy()
        flag, st = oracle.react_arkode(mech, 1, y, src, rX.copy(), rXs, dt, rtol=rtol, atol=1e-16, max_steps=10**6)
        assert flag == 0 and st["t"] == dt
        errs.append(np.max(np.abs(y[:, -1] - ref[:, -1]) / ref[:, -1]))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 2e-8


def test_oracle_mask_and_empty(oracle):
    mech, dt, nc = "LiDryer", 1e-6, 8
    rY, src, rX, rXs = _batch(oracle, mech, nc)
    mask = np.ones(nc, np.int32)
    mask[[1, 6]] = -1
    y = rY.copy()
    x = rX.copy()
    flag, st = oracle.react_arkode(mech, 1, y, src, x, rXs, dt, rtol=1e-8, atol=1e-10, mask=mask)
    assert flag == 0
    np.testing.assert_array_equal(y[[1, 6]], rY[[1, 6]])
    assert np.all(y[mask == 1, -1] != rY[mask == 1, -1])
    # the unmasked cells integrate as a batch of their own
    sub = rY[mask == 1].copy()
    flag2, st2 = oracle.react_arkode(mech, 1, sub, np.ascontiguousarray(src[mask == 1]), rX[mask == 1].copy(),
                                     rXs[mask == 1], dt, rtol=1e-8, atol=1e-10)
    np.testing.assert_array_equal(sub, y[mask == 1])
    assert st2["nst"] == st["nst"]
    # nothing to integrate: the time still advances
    y = rY.copy()
    flag, st = oracle.react_arkode(mech, 1, y, src, rX.copy(), rXs, dt, mask=-np.ones(nc, np.int32))
    assert flag == 0 and st["t"] == dt and st["nst"] == 0
    np.testing.assert_array_equal(y, rY)


def test_oracle_step_cap_stops_at_the_last_step(oracle):
    mech, dt, nc = "drm19", 1e-5, 6
    rY, src, rX, rXs = _batch(oracle, mech, nc)
    rXs[:] = 1e3
    y = rY.copy()
    x = rX.copy()
    flag, st = oracle.react_arkode(mech, 1, y, src, x, rXs, dt, rtol=1e-8, atol=1e-10, max_steps=3)
    assert flag == -1 and st["nst"] == 3 and 0.0 < st["t"] < dt
    np.testing.assert_allclose(x, rX + st["t"] * rXs, rtol=1e-15)
    assert np.all(np.isfinite(y))


def test_generated_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "%s"\nint main(void){return ppb_erk_tables[0].stages == 2 ? 0 : 1;}\n'
                   % et.HEADER_PATH)
    exe = tmp_path / "t"
    assert os.system(f"gcc -std=c11 -Wall -Werror -o {exe} {src}") == 0
    assert os.system(str(exe)) == 0
