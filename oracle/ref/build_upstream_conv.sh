#!/usr/bin/env bash
# Builds the upstream RayTraceDicom CPU convolution (the only CPU arithmetic the
# reference ships: RayTraceDicom-main/src/cpu_convolution_1d.cpp, read in place from
# the reference checkout) with the C shim beside this script into
# oracle/_ref/librtd_cpuconv.so. The checkout is $REFERENCE_DIR, else a sibling of
# this repository named `reference`; without either the script stops with a message.
# Test infrastructure only: bench.py times it as a stage-level CPU baseline.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF=${REFERENCE_DIR:-"$HERE/../../../reference"}
OUT="$HERE/../_ref"
SRC="$REF/RayTraceDicom-main (1)/RayTraceDicom-main/src"
if [ ! -f "$SRC/cpu_convolution_1d.cpp" ]; then echo "upstream sources not found at $SRC" >&2; exit 1; fi
mkdir -p "$OUT"
# An optimised host build (-O3); the upstream CMake sets only the language standard.
g++ -O3 -std=c++17 -fPIC -shared -w -I"$SRC" "$SRC/cpu_convolution_1d.cpp" "$HERE/cpuconv_shim.cpp" \
    -o "$OUT/librtd_cpuconv.so"
echo "$OUT/librtd_cpuconv.so"
