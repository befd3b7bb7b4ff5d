#!/usr/bin/env bash
# Compiles the reference's own CPU/OpenMP path, unmodified, from the sources where they lie,
# into oracle/_ref/libdgtref.so (test infrastructure: the parity checker and the timed CPU
# baseline; git-ignored, travels to the GPU box as a built file).
#
# Sources used (paths inside the reference project):
#   src/model/DelaunayGPU.cu, src/model/DelaunayGPU.cpp,
#   src/utilities/cellListGPU.cu, src/utilities/cellListGPU.cpp, src/utilities/utilities.cu,
#   src/utilities/hilbert_curve.cpp
# The reference's CMake build is not used (it pins gcc-6 and sm_35, CMakeLists.txt:2-18);
# -DNVCC is needed so HOSTDEVICE keeps __device__ (src/utilities/indexer.h:20-24) and the
# nvtx3 include dir because inc/std_include.h:41 includes nvToolsExt.h.
# The reference's sources: $DGT_REFERENCE_DIR, else a checkout named "reference" beside this
# repository.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${DGT_REFERENCE_DIR:-$(dirname "$(dirname "$HERE")")/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/model/DelaunayGPU.cu" ]; then
    echo "reference sources not found at $REF" >&2
    exit 2
fi
CUDA="${CUDA_HOME:-/usr/local/cuda}"
mkdir -p "$OUT/obj"
INC="-I$REF/inc -I$REF/src -I$REF/src/utilities -I$REF/src/model -I$CUDA/include -I$CUDA/include/nvtx3"
NVFLAGS="-O3 -std=c++14 -DNVCC -DENABLE_CUDA --expt-relaxed-constexpr -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC,-fopenmp,-ffp-contract=off -w"
CXXFLAGS="-O3 -std=c++14 -DENABLE_CUDA -fPIC -fopenmp -ffp-contract=off -w"
set -x
nvcc $NVFLAGS $INC -c "$REF/src/model/DelaunayGPU.cu"       -o "$OUT/obj/DelaunayGPU_cu.o"
nvcc $NVFLAGS $INC -c "$REF/src/utilities/cellListGPU.cu"   -o "$OUT/obj/cellListGPU_cu.o"
nvcc $NVFLAGS $INC -c "$REF/src/utilities/utilities.cu"     -o "$OUT/obj/utilities_cu.o"
g++ $CXXFLAGS $INC -c "$REF/src/model/DelaunayGPU.cpp"      -o "$OUT/obj/DelaunayGPU_cpp.o"
g++ $CXXFLAGS $INC -c "$REF/src/utilities/cellListGPU.cpp"  -o "$OUT/obj/cellListGPU_cpp.o"
g++ $CXXFLAGS $INC -c "$REF/src/utilities/hilbert_curve.cpp" -o "$OUT/obj/hilbert_curve_cpp.o"
nvcc $NVFLAGS $INC -c "$HERE/ref_harness.cu"                -o "$OUT/obj/ref_harness.o"
nvcc -shared -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp -o "$OUT/libdgtref.so" \
    "$OUT/obj/DelaunayGPU_cu.o" "$OUT/obj/cellListGPU_cu.o" "$OUT/obj/utilities_cu.o" \
    "$OUT/obj/DelaunayGPU_cpp.o" "$OUT/obj/cellListGPU_cpp.o" "$OUT/obj/hilbert_curve_cpp.o" \
    "$OUT/obj/ref_harness.o" \
    -L"$CUDA/lib64" -lcudart -lgomp
