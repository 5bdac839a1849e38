#!/usr/bin/env bash
# Builds the reference CUDA backend (TrueKuehli/FoveatedHTGSCudaBackend) from its own
# sources, where they lie, into oracle/_ref/.  Test infrastructure only: the product never
# links or loads anything built here.
#
# Recipe (instead of the reference's setup.py, which globs and builds four modules):
#   _C             = bindings.cpp + inference_api.cu + inference.cu + torch_utils.cpp
#                    nvcc flags: -std=c++20 -rdc=true -lineinfo                (setup.py:55-77)
#   _C_benchmarking = bindings_benchmarking.cpp + fast_inference_api.cu + inference.cu
#                    + torch_utils.cpp, plus -O3 -use_fast_math               (setup.py:63-88)
#   _C_stereo      = bindings_stereo.cpp + inference_stereo_api.cu + inference_stereo.cu
#                    + torch_utils.cpp, plus -O3 -use_fast_math               (setup.py:63-99)
#   _C_visualization = bindings_visualization.cpp + visualization_api.cu + visualization.cu
#                    + torch_utils.cpp, plus -O3 -use_fast_math               (setup.py:32-50,101-110)
# Only the architecture is added: -gencode arch=compute_100a,code=sm_100a.
#
# Usage: oracle/build_ref.sh [module ...]   (default: _C _C_benchmarking _C_stereo _C_visualization)
set -euo pipefail
REF=${REF_ROOT:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref/FoveatedHTGSCudaBackend"
OBJ="$HERE/_ref/obj"
mkdir -p "$OUT" "$OBJ"
[ -f "$OUT/__init__.py" ] || : > "$OUT/__init__.py"
if [ ! -d "$REF/FoveatedHTGSCudaBackend" ]; then
  echo "reference sources not found under $REF; nothing to build" >&2; exit 0
fi
FHB="$REF/FoveatedHTGSCudaBackend"
PY=${PYTHON:-python}
TORCH_DIR=$($PY -c 'import torch,os;print(os.path.dirname(torch.__file__))' 2>/dev/null | tail -1)
PYINC=$($PY -c 'import sysconfig;print(sysconfig.get_paths()["include"])')
EXT=$($PY -c 'import sysconfig;print(sysconfig.get_config_var("EXT_SUFFIX"))')
ARCH="-gencode arch=compute_100a,code=sm_100a"
INC="-I$FHB/utils -I$FHB/rasterization/include -I$FHB/visualization/include \
 -I$TORCH_DIR/include -I$TORCH_DIR/include/torch/csrc/api/include -I$PYINC"
DEFS="-DTORCH_API_INCLUDE_EXTENSION_H -D_GLIBCXX_USE_CXX11_ABI=1"
TORCH_NVCC="-D__CUDA_NO_HALF_OPERATORS__ -D__CUDA_NO_HALF_CONVERSIONS__ \
 -D__CUDA_NO_BFLOAT16_CONVERSIONS__ -D__CUDA_NO_HALF2_OPERATORS__ --expt-relaxed-constexpr"
LIBS="-L$TORCH_DIR/lib -lc10 -lc10_cuda -ltorch -ltorch_cpu -ltorch_cuda -ltorch_python \
 -Xlinker -rpath -Xlinker $TORCH_DIR/lib"

build_module() {
  local name=$1 fast=$2; shift 2
  local srcs=("$@")
  local nv="-std=c++20 -rdc=true -lineinfo"
  local cx="-std=c++20"
  if [ "$fast" = 1 ]; then nv="$nv -O3 -use_fast_math"; cx="$cx -O3"; fi
  local objs=()
  for s in "${srcs[@]}"; do
    local o="$OBJ/${name}_$(basename "$s").o"
    if [[ "$s" == *.cu ]]; then
      nvcc $ARCH $nv $TORCH_NVCC $INC $DEFS -DTORCH_EXTENSION_NAME=$name \
        -Xcompiler -fPIC -c "$s" -o "$o"
    else
      g++ $cx $INC $DEFS -DTORCH_EXTENSION_NAME=$name -fPIC -c "$s" -o "$o"
    fi
    objs+=("$o")
  done
  nvcc $ARCH -rdc=true -shared -Xcompiler -fPIC "${objs[@]}" $LIBS -lcudadevrt \
    -o "$OUT/$name$EXT"
  echo "built $OUT/$name$EXT"
}

MODS=("$@"); [ ${#MODS[@]} -eq 0 ] && MODS=(_C _C_benchmarking _C_stereo _C_visualization)
RS="$FHB/rasterization/src"; TB="$FHB/torch_bindings"
# the modules are independent: build them side by side (about 3 GB of host memory each)
pids=()
for m in "${MODS[@]}"; do
  case $m in
    _C) build_module _C 0 "$TB/bindings.cpp" "$RS/inference_api.cu" "$RS/inference.cu" "$RS/utils/torch_utils.cpp" & ;;
    _C_benchmarking) build_module _C_benchmarking 1 "$TB/bindings_benchmarking.cpp" "$RS/fast_inference_api.cu" "$RS/inference.cu" "$RS/utils/torch_utils.cpp" & ;;
    _C_stereo) build_module _C_stereo 1 "$TB/bindings_stereo.cpp" "$RS/inference_stereo_api.cu" "$RS/inference_stereo.cu" "$RS/utils/torch_utils.cpp" & ;;
    _C_visualization) build_module _C_visualization 1 "$TB/bindings_visualization.cpp" "$FHB/visualization/src/visualization_api.cu" "$FHB/visualization/src/visualization.cu" "$RS/utils/torch_utils.cpp" & ;;
    *) echo "unknown module $m" >&2; exit 2 ;;
  esac
  pids+=($!)
done
status=0
for p in "${pids[@]}"; do wait "$p" || status=1; done
exit $status
