#!/usr/bin/env bash
# Builds the reference's own example executables (its drivers/*.cpp, compiled where they lie)
# for the CPU into oracle/_ref/drivers/<app>_p<problem> -- test infrastructure only: the
# fixtures of tests/golden/drivers.json come from them.  Each driver is compiled once per test
# problem (-DPROBLEMn selects src/problem_definition.cpp's plug-ins, as the reference's
# Makefile does) with the reference's g++ flags minus -ffast-math, and linked with
# oracle/omp_devices_shim.c (one device; target regions fall back to the host).  Nothing from
# the reference is copied into the repository.
set -euo pipefail
REF_DIR="${1:-${REF_DIR:-}}"
if [ -z "$REF_DIR" ]; then
    echo "usage: build_ref_drivers.sh <reference source dir> (or set REF_DIR)" >&2
    exit 2
fi
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref/drivers"
if [ ! -d "$REF_DIR/drivers" ]; then
    echo "reference drivers not found at $REF_DIR; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
gcc -O2 -c "$HERE/omp_devices_shim.c" -o "$OUT/omp_devices_shim.o"
for p in 1 2 3; do
    for app in fcycle vcycle mixed dirichlet neumann gaussseidel; do
        g++ -O2 -fopenmp -std=c++17 -ffp-contract=off -w -DPROBLEM$p \
            -I"$REF_DIR/include" \
            "$REF_DIR/drivers/$app.cpp" \
            "$REF_DIR/src/parser.cpp" "$REF_DIR/src/settings.cpp" \
            "$REF_DIR/src/domainsettings.cpp" "$REF_DIR/src/grid.cpp" \
            "$REF_DIR/src/problem_definition.cpp" \
            "$OUT/omp_devices_shim.o" \
            -o "$OUT/${app}_p$p.tmp"
        mv "$OUT/${app}_p$p.tmp" "$OUT/${app}_p$p"
    done
done
echo "built $OUT"
