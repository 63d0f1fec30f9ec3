#!/usr/bin/env bash
# Builds the reference's dose library from its own CUDA/C++ sources (read in place
# from the reference checkout) plus the C shim beside this script, into oracle/_ref/.
# The checkout is $REFERENCE_DIR, else a sibling of this repository named
# `reference` (<repo>/../reference); without either the script stops with a message.
# Test infrastructure only: the result is run on the GPU box to pin the oracle.
# Usage: bash oracle/ref/build_ref.sh [NUCLEAR_CORR value, e.g. GAUSS_FIT]
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF=${REFERENCE_DIR:-"$HERE/../../../reference"}
OUT="$HERE/../_ref"
NUC="${1:-OFF}"
mkdir -p "$OUT"
if [ ! -d "$REF/src" ]; then echo "reference sources not found at $REF" >&2; exit 1; fi
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
TAG=rtd
DEFS="-DSOUKUP=0 -DFLUKA=1 -DGAUSS_FIT=2"
if [ "$NUC" != "OFF" ]; then DEFS="$DEFS -DNUCLEAR_CORR=$NUC"; TAG="rtd_nuc"; fi
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
  if [ ! -f "$o" ] || [ "$REF/$s" -nt "$o" ]; then
    "$NVCC" $FLAGS $DEFS $INC -c "$REF/$s" -o "$o"
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
