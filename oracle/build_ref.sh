#!/usr/bin/env bash
# Builds the reference's own mechanism kernels into oracle/_ref/libref_<mech>.so
# (test infrastructure: used by tests, tests/golden/make_golden.py and the CPU
# baseline only).  Reads the reference sources where they lie; copies nothing.
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (else $PPB_REFERENCE_ROOT, else
# the reference's mount point in the build container, /root/reference).  The
# root it used is recorded in _ref/reference_root for the tests that read the
# reference tree (oracle/pyoracle.py: reference_root).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${PPB_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -d "$REF/Mechanisms" ]; then
  echo "build_ref: no reference tree at $REF; keeping prebuilt $OUT" >&2
  exit 0
fi
printf '%s\n' "$REF" > "$OUT/reference_root"
for mech in LiDryer drm19 dodecane_lu heptane_lu_88sk CH4_lean_qss C1-C2-NO_qss LuEthylene_qss grimech30 FFCM1_Red chem-H; do
  src="$REF/Mechanisms/$mech/mechanism.H"
  lib="$OUT/libref_${mech}.so"
  if [ -f "$lib" ] && [ "$lib" -nt "$src" ] && [ "$lib" -nt "$HERE/ref_wrap.cpp" ]; then
    continue
  fi
  g++ -std=c++17 -O3 -march=x86-64-v3 -fPIC -shared -fvisibility=hidden \
      -I"$HERE/amrex_stub" -I"$REF/Mechanisms/$mech" \
      "$HERE/ref_wrap.cpp" -o "$lib.tmp"
  mv "$lib.tmp" "$lib"
done
# the reference's SimpleTransport (Source/Transport/Simple.H) per mechanism
for mech in LiDryer drm19 dodecane_lu heptane_lu_88sk; do
  src="$REF/Mechanisms/$mech/mechanism.H"
  lib="$OUT/libreftr_${mech}.so"
  if [ -f "$lib" ] && [ "$lib" -nt "$src" ] && [ "$lib" -nt "$HERE/ref_transport.cpp" ]; then
    continue
  fi
  g++ -std=c++17 -O3 -march=x86-64-v3 -fPIC -shared -fvisibility=hidden \
      -I"$HERE/amrex_stub" -I"$REF/Mechanisms/$mech" -I"$REF/Source" \
      "$HERE/ref_transport.cpp" -o "$lib.tmp"
  mv "$lib.tmp" "$lib"
done
# the reference's SRK equation of state (Source/Eos/SRK.H) per mechanism
for mech in LiDryer drm19 dodecane_lu heptane_lu_88sk; do
  src="$REF/Mechanisms/$mech/mechanism.H"
  lib="$OUT/librefsrk_${mech}.so"
  if [ -f "$lib" ] && [ "$lib" -nt "$src" ] && [ "$lib" -nt "$HERE/ref_srk.cpp" ]; then
    continue
  fi
  g++ -std=c++17 -O3 -march=x86-64-v3 -fPIC -shared -fvisibility=hidden \
      -I"$HERE/amrex_stub" -I"$REF/Mechanisms/$mech" -I"$REF/Source" \
      "$HERE/ref_srk.cpp" -o "$lib.tmp"
  mv "$lib.tmp" "$lib"
done
