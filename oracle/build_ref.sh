#!/usr/bin/env bash
# Builds the reference's own CPU path into oracle/_ref/ref_oracle (test infrastructure only).
# Compiles oracle/ref_harness.cpp against the reference's unmodified include/ and src/ where
# they lie: the reference's source directory is the first argument (or REF_DIR); nothing from
# the reference is copied into the repository.  Flags follow the reference's g++ configuration (config/g++.mkf) minus
# -ffast-math, so the CPU arithmetic is plain IEEE double with no contraction.
set -euo pipefail
REF_DIR="${1:-${REF_DIR:-}}"
if [ -z "$REF_DIR" ]; then
    echo "usage: build_ref.sh <reference source dir> (or set REF_DIR)" >&2
    exit 2
fi
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF_DIR/include" ]; then
    echo "reference sources not found at $REF_DIR; skipping oracle/_ref build" >&2
    exit 0
fi
mkdir -p "$OUT"
g++ -O2 -fopenmp -std=c++17 -ffp-contract=off -w \
    -I"$REF_DIR/include" \
    "$HERE/ref_harness.cpp" \
    "$REF_DIR/src/parser.cpp" "$REF_DIR/src/settings.cpp" \
    "$REF_DIR/src/domainsettings.cpp" "$REF_DIR/src/grid.cpp" \
    -o "$OUT/ref_oracle.tmp"
mv "$OUT/ref_oracle.tmp" "$OUT/ref_oracle"
echo "built $OUT/ref_oracle"
