"""Build the engine's shared library for sm_100a: pelephysics_b200/libppb200.so.

The kernels are compiled once per species count of the shipped mechanisms
(ppb_engine_ns.cu with -DPPB_NS=<N>, in five kernel groups -DPPB_PART=0..4),
in parallel, then linked with the
common kernels and the C-ABI layer.  Objects are rebuilt only when a source
or header is newer.  Usage: ``python -m pelephysics_b200.build [-j N]``.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libppb200.so")
NVCC = os.environ.get("NVCC", "nvcc")
SPECIES_COUNTS = (9, 13, 21, 22, 39, 53, 88)
# species counts of the QSS mechanisms, compiled for their QSS kernel only
# (no adjoint, no ReactorArkode)
QSS_ONLY_COUNTS = (13, 22, 39)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-diag-suppress", "177,550"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(
        os.path.join(CSRC, "mech", "*.h")
    ) + [os.path.join(os.path.dirname(HERE), "include", "pelephysics_b200.h")]


def _units():
    units = [
        ("ppb_engine.o", "ppb_engine.cu", []),
        ("ppb_abi.o", "ppb_abi.cu", []),
        ("ppb_noalloc.o", "ppb_noalloc.cu", []),
        ("ppb_transport.o", "ppb_transport.cu", []),
    ]
    for ns in SPECIES_COUNTS:
        for part in range(5):  # the kernel groups of one species count, compiled in parallel
            units.append((f"ppb_engine_ns{ns}_p{part}.o", "ppb_engine_ns.cu", [f"-DPPB_NS={ns}", f"-DPPB_PART={part}"]))
    for ns in SPECIES_COUNTS:
        if ns not in QSS_ONLY_COUNTS:
            units.append((f"ppb_adjoint_ns{ns}.o", "ppb_adjoint_ns.cu", [f"-DPPB_NS={ns}"]))
    for ns in SPECIES_COUNTS:
        if ns not in QSS_ONLY_COUNTS:
            units.append((f"ppb_ark_ns{ns}.o", "ppb_ark_ns.cu", [f"-DPPB_NS={ns}"]))
    return units


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(unit, extra_flags, objdir=OBJ):
    obj, src, defs = unit
    out = os.path.join(objdir, obj)
    srcp = os.path.join(CSRC, src)
    if not _stale(out, [srcp] + _headers()):
        return None
    cmd = [NVCC] + ARCH + FLAGS + extra_flags + defs + ["-c", srcp, "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {obj}:\n{r.stdout}\n{r.stderr}")
    os.replace(out + ".tmp", out)
    return obj


def build(jobs: int | None = None, verbose: bool = False, extra_flags=()) -> str:
    """Compile (incrementally) and link the engine; returns the library path."""
    objdir, lib = OBJ, LIB
    flags = list(extra_flags)
    os.makedirs(objdir, exist_ok=True)
    units = _units()
    # the per-species kernel groups are the long poles: start them first
    units.sort(key=lambda u: 0 if "_ns" in u[0] and "engine" in u[0] else 1)
    jobs = jobs or min(len(units), os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        done = list(ex.map(lambda u: _compile(u, flags, objdir), units))
    objs = [os.path.join(objdir, u[0]) for u in units]
    if any(done) or _stale(lib, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib + ".tmp"] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(lib + ".tmp", lib)
    if verbose:
        print("built", lib, "recompiled:", [d for d in done if d])
    return lib


if __name__ == "__main__":
    j = None
    if "-j" in sys.argv:
        j = int(sys.argv[sys.argv.index("-j") + 1])
    try:
        build(j, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
