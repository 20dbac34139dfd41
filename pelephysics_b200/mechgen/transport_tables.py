"""Transport and SRK tables (mixture-averaged transport, real-gas EOS).

The reference's SimpleTransport (Source/Transport/Simple.H) reads every
coefficient from the mechanism's generated header: the CEPTR transport fits
and molecular data behind egtransetWT / EPS / SIG / DIP / POL / ZROT / NLIN /
COFETA / COFLAM / COFD / NLITE / KTDIF / COFTD (loaded by
Source/Transport/TransportParams.H:228-258), and, for the bulk viscosity,
CKCVMS's R / W_k factors; and the SRK equation of state's per-species
parameters of GET_CRITPARAMS_SRK (Source/Eos/SRK.H).  These are the
mechanism's transport and critical-point data, fitted by
CEPTR from the mechanism's Lennard-Jones parameters; this script reads them
from Mechanisms/<mech>/mechanism.H (the values only) and writes
csrc/mech/trans_<mech>.h for the engine and the oracle.

Usage: python -m pelephysics_b200.mechgen.transport_tables [REFERENCE_ROOT]
"""

from __future__ import annotations

import os
import re
import sys

MECHS = ("LiDryer", "drm19", "dodecane_lu", "heptane_lu_88sk")

_NUM = r"([-+]?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?)"


def _body(src: str, fname: str) -> str:
    m = re.search(r"\b" + fname + r"\s*\([^)]*\)\s*\{", src)
    if not m:
        raise KeyError(fname)
    depth, i = 1, m.end()
    while depth:
        c = src[i]
        depth += c == "{"
        depth -= c == "}"
        i += 1
    return src[m.end():i - 1]


def _array(src: str, fname: str, var: str, conv=float):
    body = _body(src, fname)
    vals = {}
    for m in re.finditer(r"\b" + var + r"\s*\[\s*(\d+)\s*\]\s*=\s*" + _NUM + r"\s*;", body):
        vals[int(m.group(1))] = conv(m.group(2))
    n = max(vals) + 1 if vals else 0
    if sorted(vals) != list(range(n)):
        raise ValueError(f"{fname}: missing entries")
    return [vals[i] for i in range(n)]


def _scaled(src: str, fname: str, var: str):
    body = _body(src, fname)
    vals = {}
    for m in re.finditer(r"\b" + var + r"\s*\[\s*(\d+)\s*\]\s*\*=\s*" + _NUM + r"\s*;", body):
        vals[int(m.group(1))] = float(m.group(2))
    return [vals[i] for i in range(len(vals))]


def build(mech_dir: str, name: str):
    with open(os.path.join(mech_dir, "mechanism.H")) as fh:
        src = fh.read()
    nsp = int(re.search(r"#define\s+NUM_GAS_SPECIES\s+(\d+)", src).group(1))
    assert int(re.search(r"#define\s+NUM_SURFACE_SPECIES\s+(\d+)", src).group(1)) == 0
    nfit = int(re.search(r"#define\s+NUM_FIT\s+(\d+)", src).group(1))
    assert nfit == 4
    T = {"name": name, "nsp": nsp}
    for key in ("WT", "EPS", "SIG", "DIP", "POL", "ZROT"):
        T[key.lower()] = _array(src, "egtranset" + key, key)
    T["nlin"] = _array(src, "egtransetNLIN", "NLIN", int)
    T["fitmu"] = _array(src, "egtransetCOFETA", "COFETA")
    T["fitlam"] = _array(src, "egtransetCOFLAM", "COFLAM")
    T["fitdbin"] = _array(src, "egtransetCOFD", "COFD")
    T["nlite"] = int(re.search(r"\*\s*NLITE\s*=\s*(\d+)\s*;", _body(src, "egtransetNLITE")).group(1))
    T["ktdif"] = _array(src, "egtransetKTDIF", "KTDIF", int)
    T["fittdrat"] = _array(src, "egtransetCOFTD", "COFTD")
    T["cvms"] = _scaled(src, "CKCVMS", "cvms")
    # SRK parameters (GET_CRITPARAMS_SRK), used by Source/Eos/SRK.H
    for key in ("sqrtOneOverTc", "sqrtAsti", "Bi", "Fomega"):
        T["srk_" + key] = _array(src, "GET_CRITPARAMS_SRK", key)
        assert len(T["srk_" + key]) == nsp, (name, key)
    for key in ("wt", "eps", "sig", "dip", "pol", "zrot", "nlin", "cvms"):
        assert len(T[key]) == nsp, (name, key)
    assert len(T["fitmu"]) == len(T["fitlam"]) == 4 * nsp
    assert len(T["fitdbin"]) == 4 * nsp * nsp
    assert len(T["ktdif"]) == T["nlite"] and len(T["fittdrat"]) == 4 * nsp * T["nlite"]
    return T


def _carr(ctype, name, vals, per_line=4):
    f = (lambda v: repr(float(v))) if ctype == "double" else (lambda v: str(int(v)))
    body = ",\n  ".join(", ".join(f(v) for v in vals[i:i + per_line]) for i in range(0, len(vals), per_line))
    return f"static const {ctype} {name}[] = {{\n  {body}\n}};\n"


FIELDS = ("wt", "eps", "sig", "dip", "pol", "zrot", "nlin", "fitmu", "fitlam", "fitdbin", "ktdif", "fittdrat",
          "cvms")


def emit_header(T, path):
    name = T["name"]
    P = f"ppbt_{name}_"
    out = [f"// Generated by pelephysics_b200/mechgen/transport_tables.py from the transport\n",
           f"// data of Mechanisms/{name}/mechanism.H of the reference. Do not edit.\n",
           "#pragma once\n#include \"trans_tables.h\"\n\n"]
    for key in FIELDS:
        ctype = "int" if key in ("nlin", "ktdif") else "double"
        out.append(_carr(ctype, P + key, T[key], 4 if ctype == "double" else 16))
    out.append(f"\nstatic const PPBTransTables ppbt_{name} = {{\n  \"{name}\", {T['nsp']}, {T['nlite']},\n")
    out.append("".join(f"  {P}{k},\n" for k in FIELDS))
    out.append("};\n")
    # SRK: [sqrtOneOverTc | sqrtAsti | Bi | Fomega], N each
    srk = T["srk_sqrtOneOverTc"] + T["srk_sqrtAsti"] + T["srk_Bi"] + T["srk_Fomega"]
    out.append("\n// SRK parameters (GET_CRITPARAMS_SRK): sqrt(1/Tc) | sqrt(a*) | B | F(omega), N each\n")
    out.append(_carr("double", P + "srk", srk))
    with open(path, "w") as fh:
        fh.write("".join(out))


def main(argv):
    ref = argv[1] if len(argv) > 1 else os.environ.get("PPB_REFERENCE_ROOT")
    if not ref:
        sys.exit(f"usage: python {argv[0]} REFERENCE_ROOT  (or set PPB_REFERENCE_ROOT): the PelePhysics tree")
    here = os.path.dirname(os.path.abspath(__file__))
    outdir = os.path.join(os.path.dirname(here), "csrc", "mech")
    for m in MECHS:
        T = build(os.path.join(ref, "Mechanisms", m), m)
        emit_header(T, os.path.join(outdir, f"trans_{m}.h"))
        sym = max(abs(T["fitdbin"][4 * (i + T["nsp"] * j) + q] - T["fitdbin"][4 * (j + T["nsp"] * i) + q])
                  for i in range(T["nsp"]) for j in range(T["nsp"]) for q in range(4))
        print(f"{m}: {T['nsp']} species, {T['nlite']} light species, max |COFD_ij - COFD_ji| = {sym}")


if __name__ == "__main__":
    main(sys.argv)
