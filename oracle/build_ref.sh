#!/usr/bin/env bash
# Builds the reference's own CUDA kernel libraries and integration strategies, unmodified,
# from the reference sources where they lie, against the stand-in headers in ref_shim/ (the
# reference's RR-CUDA, spdlog and tl submodules are empty), plus ref_harness.cu.
# Output only into oracle/_ref/ (git-ignored; it travels to the GPU box with the tree).
# Test infrastructure only: nothing in the product links it.
set -euo pipefail
# RRG_REFERENCE: the reference project's root (the directory holding solver/); without it the
# prebuilt library, if any, is kept
REF=${RRG_REFERENCE:-}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-nvcc}
if [ -z "$REF" ] || [ ! -d "$REF/solver" ]; then
  echo "reference sources not found at $REF; keeping any prebuilt $OUT/librrgref.so" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
INC=(-I"$HERE/ref_shim" -I"$REF/solver/extern/tl/include"
     -I"$REF/solver/lib/rrgsim_common/include" -I"$REF/solver/lib/rrgsim_nbody/include"
     -I"$REF/solver/lib/rrgsim_rect_mesh/include" -I"$REF/solver/lib/rrgsim_wave/include"
     -I"$REF/solver/app/include")
FLAGS=(-std=c++20 -rdc=true -O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC
       --expt-relaxed-constexpr -w)
SRCS=(lib/rrgsim_common/src/co_device_structs.cu lib/rrgsim_common/src/co_particles_context.cu
      lib/rrgsim_common/src/co_grid_context.cu lib/rrgsim_nbody/src/nbody.cu
      lib/rrgsim_rect_mesh/src/rm_p2mesh.cu lib/rrgsim_rect_mesh/src/rm_mesh2p.cu
      lib/rrgsim_wave/src/wave.cu lib/rrgsim_wave/src/wave_steady_checker.cu)
pids=()
for s in "${SRCS[@]}"; do
  "$NVCC" "${FLAGS[@]}" "${INC[@]}" -c "$REF/solver/$s" -o "$OUT/obj/$(basename "$s").o" &
  pids+=($!)
done
"$NVCC" "${FLAGS[@]}" "${INC[@]}" -c "$HERE/ref_harness.cu" -o "$OUT/obj/ref_harness.o" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" -shared -rdc=true -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC \
  "$OUT"/obj/*.o -o "$OUT/librrgref.so"
echo "$OUT/librrgref.so"
