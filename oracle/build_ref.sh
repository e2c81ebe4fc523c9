#!/bin/bash
# Builds the reference swifttn93 (solver/swifttn93.cpp, refkernel.cpp, argparse.cpp of the reference
# checkout) into oracle/_ref/ as a black-box oracle and CPU baseline. Nothing here is copied into the
# repository: the sources are compiled where they lie, and oracle/_ref/ is git-ignored.
#
# Two builds, both with the reference's own flags (solver/build.sh: -O3 -ffp-contract=off -std=c++17
# -fopenmp -static) except for the target ISA:
#   swifttn93       -march=icelake-server: the AVX-512 paths the reference ships (CPU baseline).
#   swifttn93_libm  -march=x86-64-v3: no AVX-512, so every logarithm is a plain libm log() call and the
#                   formatting/tail paths are the portable scalar ones (the parity oracle; the reference
#                   states both builds write identical bytes).
# An explicit ISA instead of -march=native keeps the binaries runnable on other x86-64 hosts (AVX-512 for the first).
#
# usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
SRC="$REF/solver"
if [ ! -f "$SRC/swifttn93.cpp" ]; then
  echo "build_ref.sh: reference sources not found under $SRC" >&2
  exit 2
fi
mkdir -p "$OUT"
COMMON=(-O3 -ffp-contract=off -std=c++17 -fopenmp -static -DVERSION_NUMBER=\"v1.1.0\")
FILES=("$SRC/swifttn93.cpp" "$SRC/refkernel.cpp" "$SRC/argparse.cpp")
g++ -march=icelake-server "${COMMON[@]}" -o "$OUT/swifttn93.tmp" "${FILES[@]}" 2> "$OUT/build.log"
mv "$OUT/swifttn93.tmp" "$OUT/swifttn93"
g++ -march=x86-64-v3 "${COMMON[@]}" -o "$OUT/swifttn93_libm.tmp" "${FILES[@]}" 2>> "$OUT/build.log"
mv "$OUT/swifttn93_libm.tmp" "$OUT/swifttn93_libm"
echo "built $OUT/swifttn93 and $OUT/swifttn93_libm"
