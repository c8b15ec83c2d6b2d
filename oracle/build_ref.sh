#!/usr/bin/env bash
# TEST INFRASTRUCTURE ONLY: compile the reference ChysX cloth path from its
# own sources (read in place from the directory given as the first argument,
# or else $CHYSX_REFERENCE; no default) into oracle/_ref/, for parity runs on a B200.  Nothing here is shipped or
# committed: oracle/_ref/ is git-ignored (it still travels with the tree to
# the GPU box, where the reference sources are absent).
#
# Outputs:
#   oracle/_ref/_chysx_ref.so          reference ClothSimulator, unmodified
#   oracle/_ref/_chysx_ref_springs.so  same, with the three spring call sites
#                                      the reference comments out in step()
#                                      enabled (src/cloth/cloth_simulator.cu
#                                      :785, :921, :1135), so spring parity
#                                      can be checked; the patched translation
#                                      unit is written to oracle/_ref/build/
# Both expose the Python module interface defined in oracle/ref_module.cpp.
#
# The reference's own CMake does not configure here (chysx_scenes needs
# jsoncpp), so this recipe compiles the sources the cloth simulator links
# against directly: nvcc -rdc for sm_100a, -include cstring (two sources miss
# the header), device link, g++ for the binding.
set -euo pipefail
REF=${1:-${CHYSX_REFERENCE:-}}
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh <reference checkout>  (or set CHYSX_REFERENCE)" >&2
  exit 2
fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
CUDA=${CUDA_HOME:-/usr/local/cuda}
JOBS=${JOBS:-8}
if [ ! -d "$REF/src/cloth" ]; then
  echo "build_ref.sh: reference sources not found under $REF" >&2
  exit 2
fi
mkdir -p "$OUT/obj" "$OUT/build"
ARCH="-gencode arch=compute_100a,code=sm_100a"
NVFLAGS="$ARCH -O3 -std=c++17 -rdc=true -Xcompiler -fPIC -include cstring -I $REF/src"

SRCS="memory/cuda_array.cu sparse/block_csr.cu solver/pcg_solver.cu solver/vbd_solver.cu
collision/bvh/lbvh.cu collision/bvh/quant_bvh.cu collision/mesh_topology.cu collision/self_collision.cu
collision/contact_spmv.cu collision/static_contact.cu collision/untangle.cu collision/mesh_contact.cu
collision/sdf/sdf_volume.cu collision/sdf/sdf_contact.cu collision/ef_broadphase.cu
collision/ef_contact_detector.cu collision/simplex_trajectory_filter.cu collision/collision_pipeline.cu
collision/mesh_mesh_contact.cu
constraint/cloth/pin_constraint.cu constraint/cloth/spring_constraint.cu
constraint/cloth/triangle_stretch_constraint.cu constraint/cloth/bending_constraint.cu
constraint/collision/self_collision_constraint.cu constraint/collision/untangle_constraint.cu
constraint/softbody/tet_fem_constraint.cu cloth/cloth_simulator.cu"

compile() {
  local src=$1 obj=$2
  if [ ! -f "$obj" ] || [ "$obj" -ot "$src" ]; then
    "$NVCC" $NVFLAGS -c "$src" -o "$obj"
  fi
}
export -f compile
export NVCC NVFLAGS

for s in $SRCS; do
  echo "$REF/src/$s $OUT/obj/$(echo "$s" | tr / _).o"
done | xargs -P "$JOBS" -n 2 bash -c 'compile "$0" "$1"'

# spring-enabled translation unit of the simulator
PATCHED=$OUT/build/cloth_simulator_springs.cu
sed -e 's#^\( *\)// springs_ disabled.*$#\1springs_.accumulate_gradient(x_n_span, rhs_span, cuda_stream);#' \
    -e 's#^\( *\)pins_.accumulate_hessian(x_n_span, H_, cuda_stream);#&\n\1springs_.accumulate_hessian(x_n_span, H_, cuda_stream);#' \
    -e 's#^\( *\)pins_.bind_hessian_layout(H_);#&\n\1springs_.bind_hessian_layout(H_);#' \
    "$REF/src/cloth/cloth_simulator.cu" > "$PATCHED"
for needle in "springs_.accumulate_gradient" "springs_.accumulate_hessian" "springs_.bind_hessian_layout"; do
  grep -q "$needle" "$PATCHED" || { echo "build_ref.sh: spring patch failed ($needle)" >&2; exit 3; }
done
# the patched file includes "cloth_simulator.h" and "../profile/..." relative
# to the reference's src/cloth directory
if [ ! -f "$OUT/obj/cloth_simulator_springs.o" ] || [ "$OUT/obj/cloth_simulator_springs.o" -ot "$PATCHED" ]; then
  "$NVCC" $NVFLAGS -I "$REF/src/cloth" -c "$PATCHED" -o "$OUT/obj/cloth_simulator_springs.o"
fi

PYINC=$(python3 -c 'import sysconfig; print(sysconfig.get_paths()["include"])')
PBINC=$(python3 -c 'import pybind11; print(pybind11.get_include())')
EXT=$(python3 -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
for name in _chysx_ref _chysx_ref_springs; do
  g++ -O2 -std=c++17 -fPIC -c "$HERE/ref_module.cpp" -o "$OUT/obj/${name}_module.o" -DREF_MODULE_NAME=$name \
      -I "$REF/src" -I "$CUDA/include" -I "$PYINC" -I "$PBINC" -include cstring
done

COMMON=""
for s in $SRCS; do
  [ "$s" = "cloth/cloth_simulator.cu" ] && continue
  COMMON="$COMMON $OUT/obj/$(echo "$s" | tr / _).o"
done

link() {
  local name=$1 sim_obj=$2
  "$NVCC" $ARCH -Xcompiler -fPIC -dlink $COMMON "$sim_obj" -o "$OUT/obj/${name}_dlink.o" -lcudadevrt
  g++ -shared -o "$OUT/${name}${EXT}" "$OUT/obj/${name}_module.o" $COMMON "$sim_obj" "$OUT/obj/${name}_dlink.o" \
      -L "$CUDA/lib64" -lcudadevrt -lcudart_static -lrt -lpthread -ldl
}
link _chysx_ref "$OUT/obj/cloth_cloth_simulator.cu.o"
link _chysx_ref_springs "$OUT/obj/cloth_simulator_springs.o"
echo "build_ref.sh: built $(ls "$OUT"/*.so | tr '\n' ' ')"
