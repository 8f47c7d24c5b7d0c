#!/usr/bin/env bash
# Builds the reference's own CUDA frame path (headless) for sm_100a from its sources where
# they lie, into oracle/_ref/<variant>/ref_harness.  Three variants:
#   compressed : the reference's default build (config.h defines USE_COMPRESSED_GAUSSIANS)
#   fp32       : the same sources with a shadow config.h that drops that one define
#   immediate  : fp32 with the config.h toggle ENABLE_IMMEDIATE_SPLATTING switched on
# Test infrastructure only: the outputs are checkers, never linked into the library.
set -euo pipefail
REF=${GPS_REFERENCE_ROOT:-/root/reference}
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/../_ref"
if [ ! -d "$REF/src" ]; then echo "reference sources not found at $REF" >&2; exit 1; fi
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
COMMON="-std=c++17 -O3 -use_fast_math --expt-extended-lambda --expt-relaxed-constexpr -rdc=true -lineinfo $ARCH -w"
COMMON="$COMMON -include $HERE/stub/msvc_shim.h -DPROJECT_ROOT=\"/\""

build_variant() {
  local variant=$1
  local dir="$OUT/$variant"
  mkdir -p "$dir/cfg" "$dir/obj"
  if [ "$variant" = fp32 ]; then
    sed '/^#define USE_COMPRESSED_GAUSSIANS/d' "$REF/src/config.h" > "$dir/cfg/config.h"
  elif [ "$variant" = immediate ]; then
    sed -e '/^#define USE_COMPRESSED_GAUSSIANS/d' -e 's|^//#define ENABLE_IMMEDIATE_SPLATTING|#define ENABLE_IMMEDIATE_SPLATTING|' \
      "$REF/src/config.h" > "$dir/cfg/config.h"
    grep -q '^#define ENABLE_IMMEDIATE_SPLATTING' "$dir/cfg/config.h"
  else
    cp "$REF/src/config.h" "$dir/cfg/config.h"
  fi
  # render_settings.cuh sits next to the original config.h and includes it by a quoted
  # path, which would pull the original back in; an unmodified build-time copy placed
  # beside the shadow config.h makes every include resolve to the shadow.
  cp "$REF/src/render_settings.cuh" "$dir/cfg/render_settings.cuh"
  local INC="-I$HERE/stub -I$dir/cfg -I$REF/src -I$REF/packages -I$REF/packages/glm -I$REF/packages/stb -I$REF/packages/tinybvh"
  local srcs=(
    "$HERE/ref_harness.cu"
    "$REF/src/core/random/workload/workload_distributor.cu"
    "$REF/src/core/rendering/occlusion/depth_mip_chain.cu"
    "$REF/src/core/rendering/occlusion/gaussian_bvh.cu"
    "$REF/src/core/gaussians/gaussian_loader.cu"
    "$REF/src/utils/camera_loader.cu"
    "$REF/src/timings/stochastic_timings.cu"
    "$REF/src/world/camera.cpp"
    "$REF/src/world/transform.cpp"
    "$REF/src/world/node.cpp"
  )
  local objs=()
  local pids=()
  for s in "${srcs[@]}"; do
    local o="$dir/obj/$(basename "$s").o"
    objs+=("$o")
    if [ ! -f "$o" ] || [ "$s" -nt "$o" ] || [ "$HERE/build_ref.sh" -nt "$o" ]; then
      $NVCC $COMMON $INC -x cu -c "$s" -o "$o" &
      pids+=($!)
    fi
  done
  for p in "${pids[@]}"; do wait "$p"; done
  $NVCC $ARCH -rdc=true "${objs[@]}" -o "$dir/ref_harness" -lcudart
  echo "built $dir/ref_harness"
}

for v in ${GPS_REF_VARIANTS:-compressed fp32 immediate}; do build_variant "$v"; done
