#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/liboracle.so"
SRC=("$HERE/mech_eval.c" "$HERE/reactor.c" "$HERE/arkode.c" "$HERE/transport.c" "$HERE/srk.c")
newest=0
for f in "${SRC[@]}" "$HERE/oracle.h" "$HERE"/../pelephysics_b200/csrc/mech/*.h "$HERE"/../pelephysics_b200/csrc/ppb_erk_tables.h; do
  t=$(stat -c %Y "$f"); [ "$t" -gt "$newest" ] && newest=$t
done
if [ -f "$OUT" ] && [ "$(stat -c %Y "$OUT")" -ge "$newest" ]; then exit 0; fi
gcc -std=gnu11 -O3 -march=x86-64-v3 -fopenmp -fPIC -shared -o "$OUT.tmp" "${SRC[@]}" -lm -ldl
mv "$OUT.tmp" "$OUT"
