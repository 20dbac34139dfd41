"""The C++ drop-in class (pelephysics_b200/csrc/ReactorB200.H) compiled with
g++ and driven like the reference's ReactEval driver drives a reactor
(Testing/Exec/ReactEval/main.cpp): one object, created once, for the flat
react on host arrays, concurrent flat reacts from two host threads on the
one object (the reference's OpenMP tiles, main.cpp:478-520), the box react
on device Array4 planes with a mask, flatten / unflatten, set_typ_vals_ode
and print_final_stats.  The driver's outputs are compared bit for bit with
the Python binding of the same C ABI on the same cells and launch."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from tests.helpers import premix_oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LAUNCH = dict(rtol=1e-10, atol=1e-10, max_order=5, warps_per_block=8, team_lanes=32, register_budget=2)


def build_driver(out_dir):
    exe = os.path.join(out_dir, "reactor_b200_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "pelephysics_b200", "csrc"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "reactor_b200_driver.cpp"), "-o", exe,
           "-L", os.path.join(ROOT, "pelephysics_b200"), "-lppb200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           "-lpthread", "-Wl,-rpath," + os.path.join(ROOT, "pelephysics_b200")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(os.path.join(ROOT, "pelephysics_b200",
                                                                                    "libppb200.so")),
                    reason="needs g++ and the built engine")
def test_driver_compiles_against_the_c_abi(tmp_path):
    """ReactorB200.H and its driver compile and link with g++ (no GPU)."""
    assert os.path.exists(build_driver(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_drop_in_matches_the_python_binding(cuda, oracle, tmp_path):
    torch = cuda
    from pelephysics_b200.reactor import Reactor

    mech, dt = "drm19", 1e-5
    nx, ny, nz = 8, 6, 4
    nc = nx * ny * nz
    rY, src, rX, rXs = premix_oracle(oracle, mech, nc, 17, 1100.0, 1000.0, 0.6, 0.8)
    N = rY.shape[1] - 1
    n = N + 1
    mask = np.ones(nc, np.int32)
    mask[[3, 50, 101]] = -1
    Tstore = rY[:, N] + 20.0  # the box path recomputes T from the energy
    rY_in = rY.copy()
    rY_in[:, N] = Tstore
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(np.array([nc, N, nx, ny, nz], np.int32).tobytes())
        f.write(rY_in.tobytes())
        f.write(rX.tobytes())
        f.write(mask.tobytes())
    exe = build_driver(str(tmp_path))
    run = subprocess.run([exe, str(tmp_path), mech, repr(dt)], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "-- Final stats: nSteps" in run.stdout

    def read(name, *sizes):
        a = np.fromfile(tmp_path / name, dtype=np.float64)
        out, o = [], 0
        for s in sizes:
            out.append(a[o:o + s])
            o += s
        assert o == a.size
        return out

    # 1. flat react on host arrays: the Python binding on the same cells
    fy, fx, fcost = read("out_flat.bin", nc * n, nc, 1)
    r = Reactor(mech)
    r.init(1, nc, **LAUNCH)
    y, x = rY_in.copy(), rX.copy()
    cost, _, _, code = r.react(y, np.zeros((nc, N)), x, np.zeros(nc), dt)
    assert code == 0
    assert np.array_equal(fy.reshape(nc, n), y) and np.array_equal(fx, x)
    assert int(fcost.view(np.int64)[0]) == cost

    # 2. two threads on one object: every cell as in the one-thread call
    h = nc // 2
    ya, yb, xa, xb = read("out_threads.bin", h * n, (nc - h) * n, h, nc - h)
    assert np.array_equal(np.r_[ya, yb].reshape(nc, n), y)
    assert np.array_equal(np.r_[xa, xb], x)

    # 3. the box path with the mask: the Python binding's box call
    bY, bT, bE, bFC = read("out_box.bin", N * nc, nc, nc, nc)
    rb = Reactor(mech)
    rb.init(1, nc, **LAUNCH)

    def box(a, k):
        return torch.as_tensor(np.ascontiguousarray(a.T.reshape(k, nz, ny, nx)), device="cuda")

    dY, dS, dT = box(rY[:, :N], N), box(np.zeros((nc, N)), N), box(Tstore[:, None], 1)
    dE, dEs = box(rX[:, None], 1), box(np.zeros((nc, 1)), 1)
    dFC = torch.zeros((1, nz, ny, nx), dtype=torch.float64, device="cuda")
    dM = torch.as_tensor(mask.reshape(1, nz, ny, nx), device="cuda")
    rb.react_box((0, 0, 0), (nx - 1, ny - 1, nz - 1), dY, dS, dT, dE, dEs, dFC, dM, dt_react=dt)
    torch.cuda.synchronize()
    assert np.array_equal(bY, dY.cpu().numpy().reshape(-1))
    assert np.array_equal(bT, dT.cpu().numpy().reshape(-1))
    assert np.array_equal(bE, dE.cpu().numpy().reshape(-1))
    assert np.array_equal(bFC, dFC.cpu().numpy().reshape(-1))
    assert np.all(bFC[mask == -1] == 0) and np.all(bFC[mask == 1] > 0)

    # 4. flatten: component-major vectors, T from the energy; unflatten with
    # dt = 0 writes the same state back and FC = FCunt
    M = oracle.Mech(mech)
    yv, sv, ev, esv = read("out_flatten.bin", n * nc, N * nc, nc, nc)
    yv = yv.reshape(n, nc)
    assert np.array_equal(yv[:N], rY[:, :N].T)
    assert np.array_equal(sv, np.zeros(N * nc)) and np.array_equal(ev, rX) and np.array_equal(esv, np.zeros(nc))
    for c in range(0, nc, 17):
        rho = rY[c, :N].sum()
        Tr, _ = M.t_given_ey(rX[c] / rho, rY[c, :N] / rho, Tstore[c])
        assert abs(yv[N, c] - Tr) <= 1e-9 * Tr
    uY, uT, uE, uFC = read("out_unflatten.bin", N * nc, nc, nc, nc)
    assert np.array_equal(uY, rY[:, :N].T.reshape(-1))
    assert np.array_equal(uE, rX) and np.all(uFC == 7.0)
    assert np.max(np.abs(uT - yv[N]) / yv[N]) <= 1e-9

    # 5. typical values are forwarded: the Python binding with the same ones
    ty, tx = read("out_typ.bin", nc * n, nc)
    rt = Reactor(mech)
    rt.init(1, nc, **LAUNCH)
    rt.set_typ_vals_ode(np.full(n, 2.0))  # atol_i = 2 atol
    y2, x2 = rY_in.copy(), rX.copy()
    rt.react(y2, np.zeros((nc, N)), x2, np.zeros(nc), dt)
    assert np.array_equal(ty.reshape(nc, n), y2) and np.array_equal(tx, x2)
    assert not np.array_equal(y2, y)  # the looser tolerance integrated differently
