#!/usr/bin/env bash
# Builds the reference solver's own CUDA kernels, compiled from its sources
# where they lie in the reference tree, together with oracle/ref_wrapper.cu
# into oracle/_ref/libfundem_ref.so (sm_100a). Test infrastructure only:
# the library produces golden vectors on a B200 and is never part of the
# product path. The reference tree is read, never written.
set -euo pipefail
REF=${REF:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
K="$REF/FunDEM/kernel"
if [ ! -d "$K" ]; then
  echo "reference tree not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
SRCS=(
  "$K/CUDAKernelFunction/myUtility/mySpatialGrid.cu"
  "$K/CUDAKernelFunction/myUtility/buildHashStartEnd.cu"
  "$K/CUDAKernelFunction/LSParticleContactDetectionKernel.cu"
  "$K/CUDAKernelFunction/contactKernel.cu"
  "$K/CUDAKernelFunction/particleIntegrationKernel.cu"
  "$HERE/ref_wrapper.cu"
)
# Release flags as the reference's CMake Release build (-O3 -DNDEBUG), sm_100a.
nvcc -std=c++17 -O3 -DNDEBUG -Xcompiler -fPIC -shared \
  -gencode arch=compute_100a,code=sm_100a \
  -I"$K" -I"$K/CUDAKernelFunction" \
  "${SRCS[@]}" -o "$OUT/libfundem_ref.so"
echo "built $OUT/libfundem_ref.so"

# The config-0 benchmark app (tests/apps/c0_bench.cpp, written against the
# LSSolver API only) built against the reference solver itself: its
# kernel/LSSolver.h and the same kernel sources, Release flags, sm_100a. The
# same app source is built against this repository's drop-in LSSolver by
# tests/test_fundem_same_gpu.py.
nvcc -std=c++17 -O3 -DNDEBUG \
  -gencode arch=compute_100a,code=sm_100a \
  -I"$REF/FunDEM" -I"$K" -I"$K/CUDAKernelFunction" \
  "$HERE/../tests/apps/c0_bench.cpp" "${SRCS[@]:0:5}" -o "$OUT/c0_bench_fundem"
echo "built $OUT/c0_bench_fundem"

# Golden-vector driver for the level-set grid builder: the reference's host-only
# generator header (kernel/helper/LevelSetObjectGenerator.h) driven by
# oracle/ref_mesh_grid.cpp. Host code; g++ with the CUDA include path for the
# vector types, no device code.
g++ -std=c++17 -O3 -DNDEBUG -ffp-contract=off \
  -I/usr/local/cuda/include -I"$K" -I"$K/CUDAKernelFunction" \
  "$HERE/ref_mesh_grid.cpp" -o "$OUT/mesh_grid_ref"
echo "built $OUT/mesh_grid_ref"

# The bonded-workload app (tests/apps/c2_bench.cpp, LSSolver API only) against the
# reference solver, as the config-0 app above.
nvcc -std=c++17 -O3 -DNDEBUG \
  -gencode arch=compute_100a,code=sm_100a \
  -I"$REF/FunDEM" -I"$K" -I"$K/CUDAKernelFunction" \
  "$HERE/../tests/apps/c2_bench.cpp" "${SRCS[@]:0:5}" -o "$OUT/c2_bench_fundem"
echo "built $OUT/c2_bench_fundem"
