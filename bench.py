#!/usr/bin/env python
"""Benchmark of the B200 chemistry engine: drm19 on a 64^3 field.

One step = one react() call advancing every cell of the field by dt = 1e-5 s
(constant-volume reactor, BDF orders <= 5, rtol = atol = 1e-10) -- the
drm19 64^3 workload (262144 cells: T = 1100 + 1100 s(x) from an 8-mode
seed-1 Fourier field, phi = 0.6 + 0.8 U, 1 atm, burnt cells at the
composition of a 1 ms pre-integration).  Metric: cells advanced per second
of device time (cells/s per dt), for the tuned engine (warp per cell,
persistent work queue, CUDA graph).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank integrates its own 64^3 field (weak scaling; the
cells are independent, so there is no data-path collective); the time is the
max over ranks.  --impl reference times the reference's CPU chemistry on the
host cores (the CVODE-algorithm BDF of oracle/ over the reference's own
compiled mechanism kernels) on a bounded sample of the same cells.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MECH = "drm19"
DT = 1e-5
OPTS = dict(rtol=1e-10, atol=1e-10, max_order=5)
METRIC = "cells/s per dt (drm19 64^3, tuned engine)"
# FP64 floating-point operations of one reactor RHS and one reactor Jacobian
# evaluation for drm19 (dadd + dmul + 2 dfma, exp/log included), counted with
# ncu on single-cell launches of the pointwise kernels; see
# profiles/drm19_flops_per_evaluation.md for the command and raw counts.
FLOPS_RHS = {"drm19": 12023.0}
FLOPS_JAC = {"drm19": 22908.0}
CPU_SAMPLE = 8192  # cells of the field integrated by the CPU baseline
# DRAM bytes (read + write) per cell of one launch of the tuned kernel,
# from an ncu capture of the same kernel (16 warps per block, rendezvous on)
# on the 16^3 field (4096 cells: 1.890 MB + 0.462 MB);
# profiles/k_react_team_drm19_16cubed.md has the command.  Scaled by the
# cells of a launch (the traffic grows with them).
TRAFFIC_PER_CELL = (1.889536e6 + 0.462336e6) / 4096


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def oracle_eos(po, mech):
    M = po.Mech(mech)

    def eos(T, Y, P, rtype):
        rho = np.array([M.ckrhoy(P, t, y) for t, y in zip(T, Y)])
        e = np.array([(M.ckubms if rtype == 1 else M.ckhbms)(t, y) for t, y in zip(T, Y)])
        return rho, rho * e

    return eos, M.species(), M.mw()


def cpu_sample_index(ncells, n):
    return np.sort(np.random.default_rng(7).permutation(ncells)[:n])


def run_cpu(po, cells, idx, nthreads=0):
    """The oracle (reference kernels) on cells[idx]; returns (seconds, rY,
    flag, per-cell counters [steps, RHS, Jacobians, factorisations, Newton
    iterations, error-test failures, convergence failures])."""
    po.load_ref(MECH)
    rY = cells.rY[idx].copy()
    rX = cells.rX[idx].copy()
    src = np.ascontiguousarray(cells.rYsrc[idx])
    rXs = cells.rX_src[idx].copy()
    t0 = time.perf_counter()
    flag, st, stats = po.react_flat_stats(MECH, 1, rY, src, rX, rXs, DT, use_ref_kernels=1, nthreads=nthreads, **OPTS)
    return time.perf_counter() - t0, rY, flag, stats


def reference_arm(args):
    ws, rank, _ = dist_info()
    if rank != 0:
        return 0
    from oracle import pyoracle as po
    from pelephysics_b200 import workloads as wl

    eos, species, mw = oracle_eos(po, MECH)
    cells = wl.drm19_field(64, eos=eos, species=species, mw=mw)
    idx = cpu_sample_index(cells.ncells, CPU_SAMPLE)
    cores = os.cpu_count()
    for _ in range(args.warmup):
        run_cpu(po, cells, idx[:1024])
    times = []
    for _ in range(args.steps):
        dt, _, flag, _ = run_cpu(po, cells, idx)
        times.append(dt)
    tot = sum(times)
    value = len(idx) * args.steps / tot
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "cells/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "drm19 64^3 field, dt 1e-5 s, BDF q<=5, rtol=atol=1e-10",
                   "sample_cells_per_step": int(len(idx))},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "reference",
                         "sample": f"{len(idx)} seeded cells of the 64^3 field per step; CVODE-algorithm BDF "
                                   "(oracle/reactor.c) over the reference's own compiled drm19 mechanism "
                                   "kernels (oracle/_ref), OpenMP over all host threads; SUNDIALS is absent so "
                                   "ReactorCvode itself cannot be built"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_flops(stats, n):
    """FP64 work of the CVODE algorithm from per-cell counters: RHS and
    Jacobian evaluations, (2/3) n^3 + n^2 per factorisation of I - gamma J,
    2 n^2 per Newton solve."""
    fr, fj = FLOPS_RHS.get(MECH), FLOPS_JAC.get(MECH)
    if fr is None or fj is None:
        return None
    nfe, nje, nset, nni = (stats[:, i].astype(np.float64).sum() for i in (1, 2, 3, 4))
    return nfe * fr + nje * fj + nset * (2.0 / 3.0 * n ** 3 + n * n) + nni * 2.0 * n * n


def our_arm(args):
    import torch

    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        pg = dist

    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor, probe_fp64_peak

    cells = wl.drm19_field(args.edge, device=dev)
    n = cells.ncells
    N = cells.rY.shape[1] - 1
    # device-resident species-major state and a pristine copy
    y0 = torch.as_tensor(cells.rY.T.copy(), device=dev)
    s0 = torch.as_tensor(cells.rYsrc.T.copy(), device=dev)
    x0 = torch.as_tensor(cells.rX, device=dev)
    xs = torch.as_tensor(cells.rX_src, device=dev)
    y = y0.clone()
    x = x0.clone()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    r = Reactor(MECH)
    launch = {}
    if args.launch:
        w_, t_, g_ = (int(v) for v in args.launch.split(","))
        launch = dict(warps_per_block=w_, team_lanes=t_, register_budget=g_)
    r.init(1, n, engine=1, **OPTS, **launch)
    stream = torch.cuda.current_stream(dev)

    def step():
        y.copy_(y0)
        x.copy_(x0)
        r.react_soa(y, s0, x, xs, DT, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()  # evict L2 between timed steps (outside the events)
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    ms = [a.elapsed_time(b) for a, b in ev]
    t_dev = sum(ms) / 1e3
    if pg:
        tt = torch.tensor([t_dev], device=dev, dtype=torch.float64)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        t_dev = float(tt.item())
    value = n * ws * args.steps / t_dev
    y_gpu = y.cpu().numpy().T.copy()
    stats = r.cell_stats(n)
    wpb, team, regs, tune_ms = r.launch_config()
    rv_cycles = r.rendezvous_cycles()
    status, _ = r.cell_status(n)

    # end to end through the public flat API on pinned host buffers
    hy = torch.empty((n, N + 1), dtype=torch.float64).pin_memory().numpy()
    hs = torch.empty((n, N), dtype=torch.float64).pin_memory().numpy()
    hx = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    hxs = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    hs[:] = cells.rYsrc
    hxs[:] = cells.rX_src
    re2e = Reactor(MECH)
    re2e.init(1, n, engine=1, **OPTS, **launch)
    hy[:] = cells.rY
    hx[:] = cells.rX
    re2e.react(hy, hs, hx, hxs, DT)  # warm
    e2e_t = 0.0
    for k in range(args.steps):
        hy[:] = cells.rY
        hx[:] = cells.rX
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        re2e.react(hy, hs, hx, hxs, DT)
        e2e_t += time.perf_counter() - t0
    if pg:
        tt = torch.tensor([e2e_t], device=dev, dtype=torch.float64)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        e2e_t = float(tt.item())
    e2e = n * ws * args.steps / e2e_t
    h2d = n * (N + 1) * 8 + n * N * 8 + 2 * n * 8
    d2h = n * (N + 1) * 8 + 2 * n * 4
    re2e.close()

    out = {}
    if rank == 0:
        # the plain per-cell FP64 engine on the same full field (equal work)
        rp = Reactor(MECH)
        rp.init(1, n, engine=0, **OPTS)
        yp = y0.clone()
        xp = x0.clone()
        # one untimed call first: module load, scratch and graph capture stay
        # outside the timed call
        rp.react_soa(yp, s0, xp, xs, DT)
        yp.copy_(y0)
        xp.copy_(x0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rp.react_soa(yp, s0, xp, xs, DT, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        plain_value = n / (a.elapsed_time(b) / 1e3)
        y_plain = yp.cpu().numpy().T
        dT_plain = float(np.max(np.abs(y_plain[:, N] - y_gpu[:, N]) / y_gpu[:, N]))
        rp.close()
        # the FP32-factor engine (FP32 LU of I - gamma J, one FP64
        # refinement sweep) on the same field
        rf = Reactor(MECH)
        rf.init(1, n, engine=1, lu_fp32=1, refine_sweeps=1, **OPTS)
        yf = y0.clone()
        xf = x0.clone()
        rf.react_soa(yf, s0, xf, xs, DT)
        ms_f = []
        for _ in range(args.steps):
            yf.copy_(y0)
            xf.copy_(x0)
            flush.zero_()
            a.record(stream)
            rf.react_soa(yf, s0, xf, xs, DT, stream=stream)
            b.record(stream)
            torch.cuda.synchronize()
            ms_f.append(a.elapsed_time(b))
        fp32_value = n * len(ms_f) / (sum(ms_f) / 1e3)
        y_fp32 = yf.cpu().numpy().T.copy()
        fw, ft, fr, _ = rf.launch_config()
        frv = rf.rendezvous_cycles()
        rf.close()
        if not args.no_adjoint:
            out["adjoint"] = adjoint_measure(dev, args.adjoint_cells)
        peak = probe_fp64_peak()
        out.update(plain_value=plain_value, dT_plain=dT_plain, fp64_peak_gflops=peak, fp32_value=fp32_value,
                   fp32_launch={"warps_per_block": fw, "lanes_per_cell": ft, "register_budget": fr,
                                "rendezvous_cycles": frv})

    cpu = None
    acc = None
    flops = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import pyoracle as po

        idx = cpu_sample_index(n, CPU_SAMPLE)
        secs, y_cpu, flag, ostats = run_cpu(po, cells, idx)
        cpu = {"value": len(idx) / secs, "unit": "cells/s", "cores": os.cpu_count(), "kind": "reference",
               "sample": f"{len(idx)} seeded cells of the same 64^3 field, one react; CVODE-algorithm BDF "
                         "(oracle/reactor.c) over the reference's own compiled drm19 kernels (oracle/_ref), "
                         "OpenMP over all host threads (ReactorCvode needs the absent SUNDIALS)"}
        # algorithmic work per cell from the oracle's counters on the sample
        # (implementation-independent), times the cells of the field
        flops = algorithmic_flops(ostats, N + 1) / len(idx) * n
        inputs = (cells.rY[idx], cells.rYsrc[idx], cells.rX[idx], cells.rX_src[idx])
        acc = po.compare_to_reference(MECH, 1, *inputs, DT, y_gpu[idx], y_cpu, use_ref_kernels=1, **OPTS)
        acc["fp32_factor"] = po.compare_to_reference(MECH, 1, *inputs, DT, y_fp32[idx], y_cpu, use_ref_kernels=1,
                                                     **OPTS)
        acc["plain"] = po.compare_to_reference(MECH, 1, *inputs, DT, y_plain[idx], y_cpu, use_ref_kernels=1, **OPTS)
        # against a converged solution (the oracle at rtol = atol = 1e-13):
        # the error of the GPU and of the oracle itself at 1e-10
        yconv = cells.rY[idx].copy()
        po.react_flat(MECH, 1, yconv, np.ascontiguousarray(cells.rYsrc[idx]), cells.rX[idx].copy(),
                      cells.rX_src[idx].copy(), DT, use_ref_kernels=1, rtol=1e-13, atol=1e-13, max_order=5)
        Yv = po.mass_fraction_rows(yconv, N)
        err = lambda yy: {"max_rel_T": float(np.max(np.abs(yy[:, N] - yconv[:, N]) / yconv[:, N])),
                          "max_abs_Y": float(np.abs(po.mass_fraction_rows(yy, N) - Yv).max())}
        acc["vs_converged_oracle_1e-13"] = {"gpu_tuned": err(y_gpu[idx]), "gpu_fp32_factor": err(y_fp32[idx]),
                                            "oracle_1e-10": err(y_cpu)}
        acc["oracle_counts_per_cell"] = dict(zip(["steps", "rhs", "jac", "lu", "newton", "err_fail", "conv_fail"],
                                                 [round(float(v), 3) for v in ostats.mean(axis=0)]))

    configs = None
    if rank == 0 and ws == 1 and not args.no_configs:
        from oracle import pyoracle as po

        configs = {"lidryer_16cubed": measure_lidryer(po, dev), "ch4_lean_qss": measure_qss(po, dev)}
        for cfg in ("dodecane", "heptane"):
            configs[cfg] = measure_config(cfg, 1, 256)

    if rank == 0:
        t_step = t_dev / args.steps
        roof = None
        if flops is not None:
            achieved = flops / t_step / 1e12
            peak_t = out["fp64_peak_gflops"] / 1e3
            roof = {"bound": "fp64", "achieved": achieved, "peak": peak_t, "unit": "TFLOP/s",
                    "frac": achieved / peak_t, "traffic": TRAFFIC_PER_CELL * n,
                    "work_note": "FP64 work per cell = n_RHS F_rhs + n_Jac F_jac + n_LU ((2/3) n^3 + n^2) + "
                                 "n_Newton 2 n^2 with the counts of the CPU oracle on the 8192-cell sample "
                                 "(accuracy_vs_fp64_oracle.oracle_counts_per_cell), times the cells",
                    "traffic_note": "DRAM bytes per launch, per cell from the 16^3 ncu capture times the cells",
                    "peak_source": "measured FP64 FMA probe on this GPU (ppb_probe_fp64_peak)"}
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "cells/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": 1e3 * t_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "drm19 64^3 field (262144 cells/GPU), dt 1e-5 s, constant-volume, BDF q<=5, "
                                   "rtol=atol=1e-10", "cells_per_gpu": n, "l2": "flushed between timed steps",
                       "engine": "tuned: team of lanes per cell, persistent work queue, CUDA graph, FP64 LU",
                       "autotuned_launch": {"warps_per_block": wpb, "lanes_per_cell": team,
                                            "register_budget": "<=128 regs" if regs == 2 else "<=255 regs",
                                            "rendezvous_cycles": rv_cycles, "sample_ms": tune_ms}},
            "e2e": {"value": e2e, "unit": "cells/s", "h2d_bytes_per_step": h2d * ws, "d2h_bytes_per_step": d2h * ws},
            "gpu_launches": 2 * args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "tuned_vs_plain": {"plain_value": out["plain_value"], "ratio": value / ws / out["plain_value"],
                               "plain_sample": "the full field, one react after one untimed warm-up react",
                               "max_rel_T_tuned_vs_plain": out["dT_plain"]},
            "fp32_factor": {"value": out["fp32_value"], "ratio_vs_plain": out["fp32_value"] / out["plain_value"],
                            "ratio_vs_fp64_lu": out["fp32_value"] / (value / ws),
                            "engine": "tuned, FP32 LU of I - gamma J + one FP64 refinement sweep",
                            "launch": out["fp32_launch"]},
            "accuracy_vs_fp64_oracle": acc,
            "adjoint": out.get("adjoint"),
            "configs": configs,
            "cell_failures": int(np.sum(status < 0)),
            "per_cell_mean": dict(zip(["steps", "rhs", "jac", "lu", "newton", "err_fail", "conv_fail"],
                                      [round(float(v), 3) for v in stats.mean(axis=0)])),
            "wall_s": wall,
        }
        print(json.dumps(line), flush=True)
    r.close()
    if pg:
        pg.destroy_process_group()
    return 0


def adjoint_measure(dev, ncells):
    """Adjoint workload: forward react() and the discrete adjoint of the loss
    sum(w_T T + w_OH Y_OH) on drm19 h/c_p reactors over 5e-4 s; device time
    of each (CUDA events) and their ratio."""
    import torch

    from pelephysics_b200 import adjoint as adj
    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor

    cells = wl.drm19_adjoint(ncells, device=dev)
    n = cells.rY.shape[0]
    t_end = cells.dt
    ioh = [s.upper() for s in wl._lib.species_names(MECH)].index("OH")
    g = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    y0, s, x0, xs = g(cells.rY), g(cells.rYsrc), g(cells.rX), g(cells.rX_src)
    r = Reactor(MECH)
    r.init(2, n, engine=1, **OPTS)
    # warm-up: the full batch once forward (autotuner, graph capture) and
    # once through the adjoint (its checkpoint, tape and item scratch grows
    # to the batch there, outside the timed calls)
    yw, xw = y0.clone(), x0.clone()
    r.react(yw, s, xw, xs, t_end)
    r.adjoint(y0, s, x0, xs, t_end, torch.zeros_like(y0))
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    y, x = y0.clone(), x0.clone()
    a.record()
    r.react(y, s, x, xs, t_end)
    b.record()
    torch.cuda.synchronize()
    t_fwd = a.elapsed_time(b) / 1e3
    fwd_stats = r.cell_stats(n)
    fw, ft, fr, _ = r.launch_config()
    fwd_launch = {"warps_per_block": fw, "lanes_per_cell": ft, "register_budget": fr,
                  "rendezvous_cycles": r.rendezvous_cycles()}
    w = g(cells.meta["w"])
    L, lam = adj.loss_T_OH(y, ioh, w[0], w[1])
    t_adjs = []
    for _ in range(3):
        a.record()
        y_adj, lam_y0, lam_e, grad = r.adjoint(y0, s, x0, xs, t_end, lam.contiguous())
        b.record()
        torch.cuda.synchronize()
        t_adjs.append(a.elapsed_time(b) / 1e3)
    t_adj = float(np.median(t_adjs))
    st, _ = r.cell_status(n)
    R = r.nrxn
    gr = grad.cpu().numpy()
    dT = float(((y_adj[:, -1] - y[:, -1]).abs() / y[:, -1]).max())
    r.close()
    return {"workload": f"drm19 {n} h/cp reactors, T 1100+500U, phi 0.5+1.5U, 1 atm, t_end 5e-4 s, "
                        "rtol=atol=1e-10; L = sum(w_T T + w_OH Y_OH), w ~ N(0,1) seed 4",
            "cells": n, "forward_ms": 1e3 * t_fwd, "forward_launch": fwd_launch, "adjoint_ms": 1e3 * t_adj,
            "adjoint_ms_runs": [1e3 * v for v in t_adjs], "ratio": t_adj / t_fwd,
            "target_ratio": 5.0, "checkpoint_interval": 16, "loss": float(L),
            "grad_norm": {"lnA": float(np.linalg.norm(gr[:R])), "beta": float(np.linalg.norm(gr[R:2 * R])),
                          "EaR": float(np.linalg.norm(gr[2 * R:])),
                          "y0": float(lam_y0.norm()), "rhoe": float(lam_e.norm())},
            "failed_cells": int(np.sum(st < 0)), "max_rel_T_adjoint_forward_vs_react": dT,
            "mean_steps": float(fwd_stats[:, 0].mean())}


def measure_config(config, steps, sample):
    """One of the larger configurations, as a dict: dodecane_lu 128x128x64
    (FP64 LU vs FP32 factor + FP64 refinement) or heptane_lu_88sk 64^3 (the
    same two, plus RK64); per arm cells/s over `steps` timed react calls after
    one warm-up call, and errors against the FP64 CPU oracle on a seeded
    sample of `sample` cells."""
    import torch

    from oracle import pyoracle as po
    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor

    dev = torch.device("cuda", torch.cuda.current_device())
    if config == "dodecane":
        mech = "dodecane_lu"
        cells = wl.dodecane_field(device=dev)
        opts = dict(rtol=1e-10, atol=1e-10, max_order=5)
        arms = [("bdf_fp64_lu", "ReactorCvode", dict(lu_fp32=0)),
                ("bdf_fp32_lu_fp64_refine", "ReactorCvode", dict(lu_fp32=1, refine_sweeps=1))]
        workload = "dodecane_lu 128x128x64 (1048576 cells), 40 atm, T 700+600 s(x), dt 2e-6 s, advective sources"
    else:
        mech = "heptane_lu_88sk"
        cells = wl.heptane_cells(device=dev)
        opts = dict(rtol=1e-8, atol=1e-12, max_order=5)
        arms = [("bdf_fp64_lu", "ReactorCvode", dict(lu_fp32=0)),
                ("bdf_fp32_lu_fp64_refine", "ReactorCvode", dict(lu_fp32=1, refine_sweeps=1)),
                ("rk64", "ReactorRK64", dict())]
        workload = "heptane_lu_88sk 262144 cells, 20 atm, T 750+650 U, phi 0.3+1.7 U, dt 1e-5 s"
    n = cells.ncells
    N = cells.rY.shape[1] - 1
    y0 = torch.as_tensor(cells.rY.T.copy(), device=dev)
    s0 = torch.as_tensor(cells.rYsrc.T.copy(), device=dev)
    x0 = torch.as_tensor(cells.rX, device=dev)
    xs = torch.as_tensor(cells.rX_src, device=dev)
    idx = np.sort(np.random.default_rng(9).permutation(n)[:sample])
    yc = cells.rY[idx].copy()
    t0 = time.perf_counter()
    flag, _, _ = po.react_flat(mech, 1, yc, np.ascontiguousarray(cells.rYsrc[idx]), cells.rX[idx].copy(),
                               cells.rX_src[idx].copy(), cells.dt, use_ref_kernels=1, **opts)
    cpu_s = time.perf_counter() - t0
    out = {}
    for name, integ, extra in arms:
        r = Reactor(mech, integ)
        r.init(1, n, engine=1, **opts, **extra)
        y = y0.clone()
        x = x0.clone()
        r.react_soa(y, s0, x, xs, cells.dt)  # warm-up (autotuner, allocations, graph)
        ms = []
        for _ in range(steps):
            y.copy_(y0)
            x.copy_(x0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            r.react_soa(y, s0, x, xs, cells.dt)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        yall = y.cpu().numpy()
        finite = np.all(np.isfinite(yall), axis=0)
        yg = yall.T[idx]
        st, _ = r.cell_status(n)
        ok = np.all(np.isfinite(yg), axis=1)
        dT = np.abs(yg[ok, N] - yc[ok, N]) / yc[ok, N]
        Yg = yg[ok, :N] / yg[ok, :N].sum(1, keepdims=True)
        Yc = yc[ok, :N] / yc[ok, :N].sum(1, keepdims=True)
        stats = r.cell_stats(n)
        wpb, team, regs, _ = r.launch_config()
        out[name] = {"cells_per_s": n * len(ms) / (sum(ms) / 1e3), "ms_per_react": sum(ms) / len(ms),
                     "autotuned_launch": {"warps_per_block": wpb, "team_lanes": team, "register_budget": regs},
                     "max_rel_T_vs_fp64_oracle": float(dT.max()) if ok.any() else None,
                     "max_abs_Y_vs_fp64_oracle": float(np.abs(Yg - Yc).max()) if ok.any() else None,
                     "nonfinite_cells": int(np.sum(~finite)),
                     "failed_cells": int(np.sum(st < 0)),
                     "per_cell_mean": dict(zip(["steps", "rhs", "jac", "lu", "newton", "err_fail", "conv_fail"],
                                               [round(float(v), 3) for v in stats.mean(axis=0)]))}
        if integ == "ReactorRK64":
            # the oracle's RK64 on the sample: the explicit scheme's own answer
            yk = cells.rY[idx].copy()
            po.react_flat(mech, 1, yk, np.ascontiguousarray(cells.rYsrc[idx]), cells.rX[idx].copy(),
                          cells.rX_src[idx].copy(), cells.dt, method=1, use_ref_kernels=1, **opts)
            okk = np.all(np.isfinite(yk), axis=1)
            both = okk & ok
            out[name]["oracle_rk64_nonfinite_in_sample"] = int(np.sum(~okk))
            out[name]["gpu_rk64_nonfinite_in_sample"] = int(np.sum(~ok))
            if both.any():
                out[name]["max_rel_T_vs_oracle_rk64"] = float(np.max(np.abs(yg[both, N] - yk[both, N]) / yk[both, N]))
        r.close()
    return {"workload": workload, "cells": n, "opts": opts, "arms": out,
            "oracle_sample": {"cells": int(len(idx)), "seconds": cpu_s, "flag": int(flag),
                              "kind": "oracle BDF over the reference's compiled kernels (oracle/_ref), OpenMP"}}


def measure_lidryer(po, dev):
    """Configuration 1: LiDryer 16^3 = 4096 cells (T 1000 + 400 U, phi 0.5 +
    1.5 U, seed 0, 1 atm), dt 1e-4 s, rtol = atol = 1e-10, BDF orders <= 5;
    tuned and plain engines, one timed react each after a warm-up react, and
    every cell against the oracle over the reference's compiled kernels."""
    import torch

    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor

    cells = wl.lidryer_16(device=dev)
    n = cells.ncells
    opts = dict(rtol=1e-10, atol=1e-10, max_order=5)
    yc = cells.rY.copy()
    t0 = time.perf_counter()
    flag, _, _ = po.react_flat("LiDryer", 1, yc, np.ascontiguousarray(cells.rYsrc), cells.rX.copy(),
                               cells.rX_src.copy(), cells.dt, use_ref_kernels=1, **opts)
    cpu_s = time.perf_counter() - t0
    out = {"workload": "LiDryer 16^3 (4096 cells), 1 atm, T 1000+400 U, phi 0.5+1.5 U, dt 1e-4 s, "
                       "rtol=atol=1e-10, BDF q<=5", "cells": n,
           "oracle": {"cells_per_s": n / cpu_s, "cores": os.cpu_count(), "flag": int(flag)}}
    y0 = torch.as_tensor(cells.rY.T.copy(), device=dev)
    s0 = torch.as_tensor(cells.rYsrc.T.copy(), device=dev)
    x0 = torch.as_tensor(cells.rX, device=dev)
    xs = torch.as_tensor(cells.rX_src, device=dev)
    for name, engine in (("tuned", 1), ("plain", 0)):
        r = Reactor("LiDryer")
        r.init(1, n, engine=engine, **opts)
        y, x = y0.clone(), x0.clone()
        r.react_soa(y, s0, x, xs, cells.dt)
        y.copy_(y0)
        x.copy_(x0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        r.react_soa(y, s0, x, xs, cells.dt)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        yg = y.cpu().numpy().T.copy()
        acc = po.compare_to_reference("LiDryer", 1, cells.rY, cells.rYsrc, cells.rX, cells.rX_src, cells.dt, yg, yc,
                                      use_ref_kernels=1, **opts)
        out[name] = {"cells_per_s": n / (ms / 1e3), "ms_per_react": ms, "accuracy_vs_fp64_oracle": acc}
        r.close()
    out["tuned_vs_plain"] = out["tuned"]["cells_per_s"] / out["plain"]["cells_per_s"]
    return out


def measure_qss(po, dev, sample=1024):
    """A QSS mechanism: CH4_lean_qss, 65536 e-reactors (T 1100 + 1000 U,
    phi 0.5 + 0.5 U, 1 atm), dt 1e-5 s, rtol = atol = 1e-10, BDF orders <= 5
    with a difference-quotient Jacobian (the reference's dense_direct
    solve); one timed react after a warm-up react, and a seeded sample of
    cells against the oracle over the reference's compiled kernels (the
    oracle's time on the sample is the CPU baseline)."""
    import torch

    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor

    mech = "CH4_lean_qss"
    cells = wl.ch4_lean_qss(device=dev)
    n = cells.ncells
    opts = dict(rtol=1e-10, atol=1e-10, max_order=5)
    idx = np.sort(np.random.default_rng(7).permutation(n)[:sample])
    yc = np.ascontiguousarray(cells.rY[idx])
    t0 = time.perf_counter()
    flag, _, _ = po.react_flat(mech, 1, yc, np.ascontiguousarray(cells.rYsrc[idx]), cells.rX[idx].copy(),
                               cells.rX_src[idx].copy(), cells.dt, use_ref_kernels=1, **opts)
    cpu_s = time.perf_counter() - t0
    out = {"workload": f"{mech} {n} e-reactors, 1 atm, T 1100+1000 U, phi 0.5+0.5 U, dt 1e-5 s, rtol=atol=1e-10, "
                       "BDF q<=5, difference-quotient Jacobian", "cells": n,
           "oracle_sample": {"cells": int(sample), "cells_per_s": sample / cpu_s, "cores": os.cpu_count(),
                             "flag": int(flag)}}
    y0 = torch.as_tensor(cells.rY.T.copy(), device=dev)
    s0 = torch.as_tensor(cells.rYsrc.T.copy(), device=dev)
    x0 = torch.as_tensor(cells.rX, device=dev)
    xs = torch.as_tensor(cells.rX_src, device=dev)
    r = Reactor(mech)
    r.init(1, n, **opts)
    y, x = y0.clone(), x0.clone()
    r.react_soa(y, s0, x, xs, cells.dt)
    y.copy_(y0)
    x.copy_(x0)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    r.react_soa(y, s0, x, xs, cells.dt)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    yg = y.cpu().numpy().T.copy()[idx]
    acc = po.compare_to_reference(mech, 1, cells.rY[idx], cells.rYsrc[idx], cells.rX[idx], cells.rX_src[idx],
                                  cells.dt, yg, yc, use_ref_kernels=1, **opts)
    wpb, team, regs, _ = r.launch_config()
    out["tuned"] = {"cells_per_s": n / (ms / 1e3), "ms_per_react": ms, "accuracy_vs_fp64_oracle": acc,
                    "launch": {"warps_per_block": wpb, "lanes_per_cell": team}}
    out["tuned_vs_oracle_sample"] = out["tuned"]["cells_per_s"] / out["oracle_sample"]["cells_per_s"]
    r.close()
    return out


def config_arm(args):
    """--config dodecane|heptane: the larger configuration on its own line."""
    import torch

    torch.cuda.set_device(0)
    line = {"config": args.config, **measure_config(args.config, args.steps, args.sample),
            "dtype": "f64 state; LU as named"}
    print(json.dumps(line), flush=True)
    return 0


def arkode_arm(args):
    """ReactorArkode (the batch-coupled explicit reactor) on the drm19 64^3
    field: the whole field as one integration on the GPU (cells/s per
    dt_react), and on a 4096-cell batch of the field the GPU against the
    oracle's restatement (same step and RHS counts, state differences) and the
    oracle's CPU time (OpenMP over the host cores)."""
    import torch

    from oracle import pyoracle as po
    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    dt, opts = 1e-6, dict(rtol=1e-6, atol=1e-10)  # ode.rtol / ode.atol defaults
    cells = wl.drm19_field(args.edge, device=dev)
    n = cells.ncells
    N = cells.rY.shape[1] - 1
    r = Reactor(MECH, "ReactorArkode")
    r.init(1, n, **opts)
    y0 = torch.as_tensor(cells.rY, device=dev).contiguous()
    s0 = torch.as_tensor(cells.rYsrc, device=dev).contiguous()
    x0 = torch.as_tensor(cells.rX, device=dev)
    xs = torch.as_tensor(cells.rX_src, device=dev)
    y = y0.clone()
    x = x0.clone()
    for _ in range(max(args.warmup, 1)):
        y.copy_(y0)
        x.copy_(x0)
        r.react(y, s0, x, xs, dt)
    ms = []
    for _ in range(args.steps):
        y.copy_(y0)
        x.copy_(x0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        cost, _, _, _ = r.react(y, s0, x, xs, dt)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    stats = r.cell_stats(n)[0]
    full = {"cells_per_s": n * len(ms) / (sum(ms) / 1e3), "ms_per_react": sum(ms) / len(ms),
            "steps": int(stats[0]), "rhs_evals": int(stats[1]), "err_test_fails": int(stats[5]),
            "cell_rhs_per_s": n * int(stats[1]) * len(ms) / (sum(ms) / 1e3)}
    r.close()
    # a 4096-cell batch: GPU vs the oracle, and the oracle's CPU time
    nb = min(4096, n)
    rb = Reactor(MECH, "ReactorArkode")
    rb.init(1, nb, **opts)
    yb = cells.rY[:nb].copy()
    xb = cells.rX[:nb].copy()
    gcost, _, _, _ = rb.react(yb, cells.rYsrc[:nb].copy(), xb, cells.rX_src[:nb].copy(), dt)
    gst = rb.cell_stats(nb)[0]
    rb.close()
    yc = cells.rY[:nb].copy()
    t0 = time.perf_counter()
    flag, st = po.react_arkode(MECH, 1, yc, np.ascontiguousarray(cells.rYsrc[:nb]), cells.rX[:nb].copy(),
                               cells.rX_src[:nb].copy(), dt, **opts)
    cpu_s = time.perf_counter() - t0
    dT = np.abs(yb[:, N] - yc[:, N]) / yc[:, N]
    Yg = yb[:, :N] / yb[:, :N].sum(1, keepdims=True)
    Yc = yc[:, :N] / yc[:, :N].sum(1, keepdims=True)
    line = {"config": "arkode", "workload": f"drm19 {args.edge}^3 field ({n} cells), dt {dt} s, rtol 1e-6, "
                                            "atol 1e-10, ZONNEVELD_5_3_4 + PID (the flat path's defaults), "
                                            "one batch-coupled integration",
            "gpu": full,
            "batch_4096": {"gpu_steps": int(gst[0]), "oracle_steps": st["nst"], "gpu_rhs_evals": int(gcost),
                           "oracle_rhs_evals": st["nfe"], "oracle_flag": int(flag),
                           "max_rel_T_vs_oracle": float(dT.max()),
                           "max_abs_Y_vs_oracle": float(np.abs(Yg - Yc).max()),
                           "oracle_cpu_s": cpu_s, "oracle_cells_per_s": nb / cpu_s, "cores": os.cpu_count()},
            "dtype": "f64"}
    print(json.dumps(line), flush=True)
    return 0


def transport_arm(args):
    """Mixture-averaged transport (ppb_transport, the reference's
    SimpleTransport) on the drm19 edge^3 field and on edge^3 heptane_lu_88sk
    cells (edge 64 by default): cells/s, the binary-diffusion pairs per
    second, the HBM traffic the call needs, the oracle's agreement on a
    sample and its CPU time."""
    import torch

    from oracle import pyoracle as po
    from pelephysics_b200 import transport as tr
    from pelephysics_b200 import workloads as wl

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    out = {}
    for mech, cells in (("drm19", wl.drm19_field(args.edge, device=dev)),
                        ("heptane_lu_88sk", wl.heptane_cells(args.edge ** 3, device=dev))):
        n = cells.ncells
        N = cells.rY.shape[1] - 1
        rho = cells.rY[:, :N].sum(1)
        Y = cells.rY[:, :N] / rho[:, None]
        T = cells.rY[:, N]
        Td = torch.as_tensor(T, device=dev)
        rd = torch.as_tensor(rho, device=dev)
        Yd = torch.as_tensor(np.ascontiguousarray(Y.T), device=dev)
        res = None
        for _ in range(max(args.warmup, 1)):
            res = tr.transport(mech, Td, rd, Yd, tr.TR_ALL)
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            res = tr.transport(mech, Td, rd, Yd, tr.TR_ALL)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        t_ms = sum(ms) / len(ms)
        # bytes the call must move: Y, T, rho in; D, chi, mu, xi, lam out
        hbm = n * 8.0 * (N + 2 + 2 * N + 3)
        idx = cpu_sample_index(n, 512)
        D = res["D"].cpu().numpy().T
        worst = 0.0
        for c in idx[:64]:
            Dr, _, mur, _, lamr = po.transport(mech, po.TR_ALL, T[c], rho[c], Y[c])
            worst = max(worst, float(np.max(np.abs(D[c] - Dr) / np.abs(Dr))),
                        abs(res["mu"][c].item() - mur) / mur, abs(res["lam"][c].item() - lamr) / lamr)
        ns = min(n, 20000)
        t0 = time.perf_counter()
        po.transport_batch(mech, po.TR_ALL, T[:ns], rho[:ns], Y[:ns])
        cpu_s = time.perf_counter() - t0
        out[mech] = {"cells": n, "ms_per_call": t_ms, "cells_per_s": n / (t_ms / 1e3),
                     "dbin_pairs_per_s": n * N * (N - 1) / 2 / (t_ms / 1e3), "hbm_gb_s": hbm / (t_ms / 1e3) / 1e9,
                     "max_rel_vs_oracle_64_cells": worst,
                     "oracle_cpu_cells_per_s": ns / cpu_s, "oracle_cores": os.cpu_count()}
    print(json.dumps({"config": "transport", "workload": "SimpleTransport (D, chi, mu, xi, lam) on the drm19 "
                      f"{args.edge}^3 field and {args.edge ** 3} heptane_lu_88sk cells", "results": out,
                      "dtype": "f64"}),
          flush=True)
    return 0


def srk_arm(args):
    """The SRK real-gas e-reactor (ReactorCvode, eos = SRK) on the drm19
    edge^3 field compressed to 50 atm (rho scaled by 50; rho*e from the SRK
    EOS): cells/s against the ideal-gas reactor on the same cells, and the
    oracle's SRK BDF on a 256-cell sample (agreement and CPU time)."""
    import torch

    from oracle import pyoracle as po
    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cells = wl.drm19_field(args.edge, device=dev)
    n = cells.ncells
    N = cells.rY.shape[1] - 1
    rY = cells.rY.copy()
    rY[:, :N] *= 50.0
    rho = rY[:, :N].sum(1)
    Y = rY[:, :N] / rho[:, None]
    s = po.Srk(MECH)
    rX = np.array([rho[c] * s.rty2e(rho[c], rY[c, N], Y[c]) for c in range(n)])
    dt, opts = DT, dict(rtol=1e-10, atol=1e-10, max_order=5)
    y0 = torch.as_tensor(rY, device=dev).contiguous()
    s0 = torch.as_tensor(cells.rYsrc, device=dev).contiguous()
    x0 = torch.as_tensor(rX, device=dev)
    xs = torch.as_tensor(cells.rX_src, device=dev)
    out = {}
    for name, eos in (("srk", 1), ("ideal_same_cells", 0)):
        r = Reactor(MECH)
        r.init(1, n, **opts, eos=eos)
        y, x = y0.clone(), x0.clone()
        r.react(y, s0, x, xs, dt)  # warm-up (and the autotuner for the ideal gas)
        ms = []
        for _ in range(args.steps):
            y.copy_(y0)
            x.copy_(x0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            r.react(y, s0, x, xs, dt)
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        st = r.cell_stats(n).mean(axis=0)
        out[name] = {"cells_per_s": n * len(ms) / (sum(ms) / 1e3), "ms_per_react": sum(ms) / len(ms),
                     "mean_steps": float(st[0]), "mean_rhs": float(st[1]), "mean_jac": float(st[2])}
        if eos == 1:
            ysrk = y.cpu().numpy()
        r.close()
    idx = cpu_sample_index(n, 256)
    yc = rY[idx].copy()
    t0 = time.perf_counter()
    flag, _, _ = po.react_flat(MECH, 1, yc, np.ascontiguousarray(cells.rYsrc[idx]), rX[idx].copy(),
                               cells.rX_src[idx].copy(), dt, eos=1, **opts)
    cpu_s = time.perf_counter() - t0
    dT = np.abs(ysrk[idx, N] - yc[:, N]) / yc[:, N]
    out["oracle_sample"] = {"cells": 256, "flag": int(flag), "max_rel_T_vs_gpu": float(dT.max()),
                            "cpu_cells_per_s": 256 / cpu_s, "cores": os.cpu_count()}
    print(json.dumps({"config": "srk", "workload": f"drm19 {args.edge}^3 field at 50 atm (SRK energies), "
                      f"dt {dt} s, rtol = atol = 1e-10", "results": out, "dtype": "f64"}), flush=True)
    return 0


def layout_arm(args, reps=5):
    """Device time of ReactorBase::flatten and unflatten (ppb_flatten /
    ppb_unflatten) on the drm19 --edge^3 box, with their algorithmic HBM
    bytes: flatten reads rhoY, frcExt (N each), T, rhoE, frcEExt and writes
    y_vect (N+1), src_vect (N), the energy and its source; unflatten reads
    y_vect (N+1), the energy, frcEExt, FCunt (int64) and writes rhoY (N), T,
    rhoE, FC (int32).  flatten also solves T from the energy per cell."""
    import torch

    from pelephysics_b200 import workloads as wl
    from pelephysics_b200.reactor import Reactor

    e = args.edge
    cells = wl.drm19_field(e)
    nc = cells.ncells
    N = cells.rY.shape[1] - 1
    box = lambda a, k: torch.as_tensor(np.ascontiguousarray(a.T.reshape(k, e, e, e)), device="cuda")
    rY = box(cells.rY[:, :N], N)
    rYs = box(cells.rYsrc, N)
    T = box(cells.rY[:, N:], 1)
    rE = box(cells.rX[:, None], 1)
    rEs = box(cells.rX_src[:, None], 1)
    FC = torch.zeros((1, e, e, e), dtype=torch.int32, device="cuda")
    yv = torch.empty((N + 1) * nc, dtype=torch.float64, device="cuda")
    sv = torch.empty(N * nc, dtype=torch.float64, device="cuda")
    ev = torch.empty(nc, dtype=torch.float64, device="cuda")
    esv = torch.empty(nc, dtype=torch.float64, device="cuda")
    fcu = torch.ones(nc, dtype=torch.int64, device="cuda")
    r = Reactor(MECH)
    r.init(cells.reactor_type, nc)
    lo, hi = (0, 0, 0), (e - 1, e - 1, e - 1)
    ops = {"flatten": (lambda: r.flatten(lo, hi, rY, rYs, T, rE, rEs, yv, sv, ev, esv), 8 * (2 * N + 3) + 8 * (2 * N + 3)),
           "unflatten": (lambda: r.unflatten(lo, hi, rY, T, rE, rEs, FC, yv, ev, fcu, cells.dt),
                         8 * (N + 1) + 8 + 8 + 8 + 8 * N + 8 + 8 + 4)}
    out = {}
    for name, (fn, bpc) in ops.items():
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        s_ = a.elapsed_time(b) / 1e3 / reps
        out[name] = {"ms": round(1e3 * s_, 4), "bytes_per_cell": bpc, "GB_per_s": round(bpc * nc / s_ / 1e9, 1)}
    r.close()
    print(json.dumps({"config": "layout", "mech": MECH, "cells": nc, "kernels": out,
                      "note": "inputs (83 MB per array set at 64^3) larger than L2 only in total; "
                              "repeated launches on the same arrays"}), flush=True)
    return 0


def pointwise_arm(args, reps=5):
    """Device time of the pointwise kernels -- reactor RHS (fKernelSpec),
    productionRate and aJacobian -- on the drm19 field's first --cells cells,
    thread-per-cell and warp-per-cell (one JSON line; with --cells 1 the
    launches are the single-cell ones whose FP64 operations ncu counts)."""
    ncells = args.cells
    import torch

    from pelephysics_b200 import _lib, workloads as wl

    cells = wl.drm19_field(64)
    N = cells.rY.shape[1] - 1
    n = min(ncells, cells.ncells)
    y = torch.as_tensor(cells.rY[:n], device="cuda").contiguous()
    x = torch.as_tensor(cells.rX[:n], device="cuda")
    xs = torch.as_tensor(cells.rX_src[:n], device="cuda")
    s = torch.as_tensor(cells.rYsrc[:n], device="cuda").contiguous()
    f = torch.zeros_like(y)
    mw = torch.as_tensor(_lib.molecular_weights(MECH), device="cuda")
    sc = (y[:, :N] / mw * 1e6).contiguous()
    T = y[:, N].contiguous()
    J = torch.zeros((n, (N + 1) ** 2), dtype=torch.float64, device="cuda")
    L = _lib.lib()
    out = {}
    for team in (1, 32):
        for name, fn in (("rhs", lambda: L.ppb_reactor_rhs(MECH.encode(), 1, 0.0, y.data_ptr(), x.data_ptr(),
                                                               xs.data_ptr(), s.data_ptr(), f.data_ptr(), n, team, None)),
                         ("jac", lambda: L.ppb_ajacobian(MECH.encode(), sc.data_ptr(), T.data_ptr(), 0, J.data_ptr(),
                                                             n, team, None)),
                         ("rates", lambda: L.ppb_production_rate(MECH.encode(), sc.data_ptr(), T.data_ptr(),
                                                                 f.data_ptr(), n, team, None))):
            _lib.check(fn())
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                fn()
            b.record()
            torch.cuda.synchronize()
            us = a.elapsed_time(b) * 1e3 / reps
            out[f"{name}_team{team}"] = {"us_per_launch": round(us, 2), "ns_per_cell": round(us * 1e3 / n, 3)}
    print(json.dumps({"config": "pointwise", "mech": MECH, "kernels": out, "cells": n}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-workload measurement")
    ap.add_argument("--adjoint-cells", type=int, default=65536)
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (LiDryer 16^3, dodecane_lu, heptane_lu_88sk) in the line")
    ap.add_argument("--config", default="drm19", choices=["drm19", "dodecane", "heptane", "arkode", "transport", "srk", "pointwise", "layout"],
                    help="drm19: the headline line; dodecane / heptane: the larger configurations; arkode: "
                         "the ReactorArkode integrator on the drm19 field")
    ap.add_argument("--sample", type=int, default=256, help="oracle sample cells for --config dodecane/heptane")
    ap.add_argument("--launch", default="", help="W,T,R: fixed warps per block, lanes per cell, register budget "
                                                 "instead of the autotuner (profiling runs)")
    ap.add_argument("--edge", type=int, default=64, help="field edge (profiling runs use a smaller box)")
    ap.add_argument("--cells", type=int, default=16384, help="cells of the field for --config pointwise")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.config == "arkode":
        return arkode_arm(args)
    if args.config == "transport":
        return transport_arm(args)
    if args.config == "srk":
        return srk_arm(args)
    if args.config == "pointwise":
        return pointwise_arm(args)
    if args.config == "layout":
        return layout_arm(args)
    if args.config != "drm19":
        return config_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
