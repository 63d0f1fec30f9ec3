#!/usr/bin/env bash
# Builds the reference's dose library from its own CUDA/C++ sources (read in place
# from the reference checkout) plus the C shim beside this script, into oracle/_ref/.
# The checkout is $REFERENCE_DIR, else a sibling of this repository named
# `reference` (<repo>/../reference); without either the script stops with a message.
# Test infrastructure only: the result is run on the GPU box to pin the oracle.
# Usage: bash oracle/ref/build_ref.sh [NUCLEAR_CORR value, e.g. GAUSS_FIT | OFF] [profile]
# With `profile` the wrapper is compiled from a copy (made under oracle/_ref/, the
# checkout is never written) in which the CarbonPBS lateral profile model's two
# switches (useCarbonProfileSigmaOverride, useCarbonProfileOverallWeight,
# raytracedicom_wrapper.cu:2813-2814) are turned on: oracle/_ref/librtd_profile.so.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF=${REFERENCE_DIR:-"$HERE/../../../reference"}
OUT="$HERE/../_ref"
NUC="${1:-OFF}"
PROFILE="${2:-}"
mkdir -p "$OUT"
if [ ! -d "$REF/src" ]; then echo "reference sources not found at $REF" >&2; exit 1; fi
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
TAG=rtd
DEFS="-DSOUKUP=0 -DFLUKA=1 -DGAUSS_FIT=2"
if [ "$NUC" != "OFF" ]; then DEFS="$DEFS -DNUCLEAR_CORR=$NUC"; TAG="rtd_nuc"; fi
WRAPPER_SRC="$REF/src/core/raytracedicom_wrapper.cu"
if [ "$PROFILE" = "profile" ]; then
  TAG="${TAG}_profile"
  mkdir -p "$OUT/profile_src"
  WRAPPER_SRC="$OUT/profile_src/raytracedicom_wrapper.cu"
  sed -e 's/const bool useCarbonProfileSigmaOverride = false;/const bool useCarbonProfileSigmaOverride = true;/' \
      -e 's/const bool useCarbonProfileOverallWeight = false;/const bool useCarbonProfileOverallWeight = true;/' \
      "$REF/src/core/raytracedicom_wrapper.cu" > "$WRAPPER_SRC.tmp"
  if [ "$(grep -c 'useCarbonProfile[A-Za-z]* = true;' "$WRAPPER_SRC.tmp")" != "2" ]; then
    echo "profile switches not found in raytracedicom_wrapper.cu" >&2; exit 1
  fi
  if [ ! -f "$WRAPPER_SRC" ] || ! cmp -s "$WRAPPER_SRC.tmp" "$WRAPPER_SRC"; then mv "$WRAPPER_SRC.tmp" "$WRAPPER_SRC"; else rm "$WRAPPER_SRC.tmp"; fi
fi
INC="-I$REF/include -I$REF/include/core -I$REF/include/algorithms -I$REF/include/utils"
# The reference's own compile options (CMakeLists.txt:180-187, separable compilation).
FLAGS="-O3 -use_fast_math -std=c++17 -rdc=true -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -w"
SRCS="src/core/raytracedicom_wrapper.cu src/core/bev_ray_tracing.cu src/algorithms/convolution.cu
src/algorithms/superposition.cu src/algorithms/complete_superposition.cu src/algorithms/idd_sigma.cu
src/algorithms/cuda_final_dose.cu src/algorithms/prim_transf_kernel.cu src/algorithms/transfer_param_struct_div3_impl.cu
src/algorithms/transfer_param_helper.cu src/utils/utils.cu src/utils/texture_ultra_optimized.cu
src/utils/advanced_memory_pool.cu src/utils/precompiled_texture_manager.cu src/utils/backward_compatibility.cu"
OBJ="$OUT/obj_$TAG"
mkdir -p "$OBJ"
objs=()
for s in $SRCS; do
  o="$OBJ/$(echo "$s" | tr '/' '_').o"
  src="$REF/$s"
  if [ "$s" = "src/core/raytracedicom_wrapper.cu" ]; then src="$WRAPPER_SRC"; fi
  if [ ! -f "$o" ] || [ "$src" -nt "$o" ]; then
    "$NVCC" $FLAGS $DEFS $INC -c "$src" -o "$o"
  fi
  objs+=("$o")
done
o="$OBJ/energy_reader.o"
g++ -O2 -std=c++17 -fPIC -w $DEFS $INC -I/usr/local/cuda/include -c "$REF/src/utils/energy_reader.cpp" -o "$o"
objs+=("$o")
o="$OBJ/ref_shim.o"
"$NVCC" $FLAGS $DEFS $INC -c "$HERE/ref_shim.cu" -o "$o"
objs+=("$o")
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/lib${TAG}.so" "${objs[@]}"
echo "$OUT/lib${TAG}.so"
