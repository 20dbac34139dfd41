"""Cells over ranks (pelephysics_b200/partition.py): contiguous cell ranges
balanced by the previous call's per-cell cost, and the int64 sum all-reduce
of the counters, on CPU: the range planner alone, then two gloo ranks whose
reactor is the CPU oracle (the engine's ranks differ only in the reactor and
the NCCL backend)."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pelephysics_b200.partition import ShardedReactor, balanced_ranges


def _check_cover(ranges, n):
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert a <= b == c <= d


def test_equal_split_without_history():
    assert balanced_ranges(np.zeros(10), 3) == [(0, 3), (3, 6), (6, 10)]
    assert balanced_ranges(np.zeros(2), 4) == [(0, 0), (0, 1), (1, 1), (1, 2)]
    assert balanced_ranges(np.zeros(0), 2) == [(0, 0), (0, 0)]


@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_cost_balanced_split(nranks):
    rng = np.random.default_rng(nranks)
    cost = rng.integers(10, 500, size=1000).astype(float)
    cost[100:120] = 5000  # an igniting patch
    r = balanced_ranges(cost, nranks)
    _check_cover(r, cost.size)
    sums = np.array([cost[a:b].sum() for a, b in r])
    # each cut is within one cell of its target: no rank is off by more than
    # the largest single cell cost
    assert np.max(np.abs(sums - cost.sum() / nranks)) <= cost.max()


def test_one_heavy_cell_and_bad_input():
    cost = np.ones(9)
    cost[4] = 100.0
    r = balanced_ranges(cost, 2)
    _check_cover(r, 9)
    assert r[0][1] in (4, 5)  # the heavy cell alone decides the cut
    with pytest.raises(ValueError):
        balanced_ranges(np.array([1.0, -1.0]), 2)
    with pytest.raises(ValueError):
        balanced_ranges(np.ones(3), 0)


class OracleReactor:
    """A CPU stand-in with the engine reactor's react / cell_stats /
    cell_status methods (the oracle's BDF on the range)."""

    def __init__(self, po, mech, opts):
        self.po, self.mech, self.opts = po, mech, opts

    def react(self, rY, rYsrc, rX, rX_src, dt, raise_on_fail=True):
        flag, st, stats = self.po.react_flat_stats(self.mech, 1, rY, np.ascontiguousarray(rYsrc), rX,
                                                   np.ascontiguousarray(rX_src), dt, **self.opts)
        self.status, self.stats = st, stats

    def cell_stats(self, m):
        return self.stats[:m]

    def cell_status(self, m):
        return self.status[:m], self.stats[:m, 1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import pyoracle as po
        from tests.helpers import premix_oracle

        mech, dt, opts = "LiDryer", 1e-5, dict(rtol=1e-10, atol=1e-10, max_order=5)
        rY, src, rX, rXs = premix_oracle(po, mech, 48, 3, 1000.0, 500.0, 0.5, 1.5)
        # the single-process answer for every cell
        ref, xr = rY.copy(), rX.copy()
        _, _, ref_stats = po.react_flat_stats(mech, 1, ref, src, xr, rXs, dt, **opts)
        sr = ShardedReactor(OracleReactor(po, mech, opts), rY.shape[0], dist)
        res = []
        for call in range(2):
            y, x = rY.copy(), rX.copy()
            (nfe, steps, failed), ranges = sr.react(y, src, x, rXs, dt)
            a, b = ranges[rank]
            ok = (np.array_equal(y[a:b], ref[a:b]) and np.array_equal(x[a:b], xr[a:b]) and
                  nfe == int(ref_stats[:, 1].sum()) and steps == int(ref_stats[:, 0].sum()) and failed == 0)
            res.append((call, ranges, bool(ok)))
        # the second call's ranges are balanced by the first call's costs
        costs = ref_stats[:, 1].astype(float)
        expect = balanced_ranges(costs, world)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([res[0][2], res[1][2], res[1][1] == expect, res[0][1] == balanced_ranges(
                    np.zeros(rY.shape[0]), world)]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_one_batch(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for rank in range(world):
        flags = np.load(tmp_path / f"rank{rank}.npy")
        assert flags.all(), (rank, flags)
