#!/usr/bin/env bash
# Builds oracle/_ref/libgsref.so: the reference's own CUDA stage kernels
# (core/gaussian_render.cu of RobinSongx/3DGaussianRenderer) plus the C-ABI
# harness in oracle/ref/ref_harness.cu.  Test infrastructure only.
#
# The reference is an MSVC/OpenGL desktop program; its kernel file does not
# compile headless with nvcc as-is.  This recipe copies the handful of files
# the kernels need into a temporary directory, applies four syntax-only
# edits, compiles, writes only the .so into oracle/_ref/, and deletes the
# temporary copy.  No reference source is kept in the repository.
#   1. gaussian_render.cuh: "utilities.h" (OpenGL wrappers + CudaTimer) ->
#      oracle/ref/ref_timer_shim.h (CudaTimer only, same blocking semantics).
#   2. gaussian_render.cu:372,478  `auto ellipse = struct Ellipse();`
#      (MSVC-only syntax)  -> `Ellipse ellipse;`  (same default constructor).
#   3. gaussian_render.cu:470  glm member swizzle `tilesRect.xy` ->
#      `glm::ivec2(tilesRect.x, tilesRect.y)`.
#   4. gaussian_render.cu:735  glm member swizzle `splatColor.rgb` ->
#      `glm::vec3(splatColor)`.
# None of the edits touches an arithmetic expression.
#
# Usage: build_ref.sh <reference-root> [<repo-root>]
set -euo pipefail
if [ $# -lt 1 ]; then
  echo "usage: build_ref.sh <reference-root> [<repo-root>]" >&2
  exit 2
fi
REF=$1
REPO=${2:-$(cd "$(dirname "$0")/../.." && pwd)}
OUT="$REPO/oracle/_ref"
if [ ! -f "$REF/core/gaussian_render.cu" ]; then
  echo "build_ref: reference sources not found under $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
TMP=$(mktemp -d)
trap 'rm -rf "$TMP"' EXIT
for f in gaussian_render.cu gaussian_render.cuh consts.h device_buffer.cu device_buffer.h cuda_error_check.cpp cuda_error_check.h; do
  cp "$REF/core/$f" "$TMP/$f"
done
sed -i 's|#include "utilities.h"|#include "ref_timer_shim.h"|' "$TMP/gaussian_render.cuh"
sed -i 's|auto ellipse = struct Ellipse();|Ellipse ellipse;|' "$TMP/gaussian_render.cu"
sed -i 's|auto globalTileCoords = tilesRect.xy + localTileCoords;|auto globalTileCoords = glm::ivec2(tilesRect.x, tilesRect.y) + localTileCoords;|' "$TMP/gaussian_render.cu"
sed -i 's|color += splatColor.rgb \* transmittance \* alpha;|color += glm::vec3(splatColor) * transmittance * alpha;|' "$TMP/gaussian_render.cu"
# every edit must have applied exactly as described
grep -q 'ref_timer_shim.h' "$TMP/gaussian_render.cuh"
[ "$(grep -c 'Ellipse ellipse;' "$TMP/gaussian_render.cu")" = 2 ]
grep -q 'glm::ivec2(tilesRect.x, tilesRect.y)' "$TMP/gaussian_render.cu"
grep -q 'glm::vec3(splatColor)' "$TMP/gaussian_render.cu"
cp "$REPO/oracle/ref/ref_harness.cu" "$TMP/ref_harness.cu"
nvcc -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -lineinfo \
  -Xcompiler -fPIC -shared \
  -I"$TMP" -I"$REPO/oracle/ref" -I"$REF/external/glm" \
  -include cstdio -include cassert -include cstdlib \
  -diag-suppress 20012,20014,20011,20013,177,550,2361,3012,1444 \
  "$TMP/ref_harness.cu" -o "$OUT/libgsref.so"
echo "build_ref: wrote $OUT/libgsref.so"

# The same harness with the stage functions of include/gs_stage_compat.hpp
# (gs_b200 behind the reference's declarations) in place of the reference's
# kernels: the stage-API drop-in test.  Links the product library.
if [ -f "$REPO/3dgaussianrenderer_b200/libgs_b200.so" ]; then
  nvcc -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -lineinfo \
    -Xcompiler -fPIC -shared -DGS_HARNESS_STAGE_COMPAT \
    -I"$TMP" -I"$REPO/oracle/ref" -I"$REPO/include" -I"$REF/external/glm" \
    -include cstdio -include cassert -include cstdlib \
    -diag-suppress 20012,20014,20011,20013,177,550,2361,3012,1444 \
    "$TMP/ref_harness.cu" -o "$OUT/libgscompat.so" \
    -L"$REPO/3dgaussianrenderer_b200" -lgs_b200 -Xlinker -rpath -Xlinker '$ORIGIN/../../3dgaussianrenderer_b200'
  echo "build_ref: wrote $OUT/libgscompat.so"
fi

# parsePly compiles as it lies (plain C++; glm and CUDA's vector_types.h);
# -ffp-contract=off keeps its float arithmetic uncontracted, as MSVC's
# default /fp:precise does.
g++ -std=c++20 -O2 -fPIC -shared -ffp-contract=off \
  -I"$REF/core" -I"$REF/external/glm" -I/usr/local/cuda/include \
  -include cassert -include limits \
  "$REPO/oracle/ref/ply_ref_harness.cpp" "$REF/core/ply_parser.cpp" -o "$OUT/libplyref.so"
echo "build_ref: wrote $OUT/libplyref.so"
