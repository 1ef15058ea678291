#!/bin/bash
# The reference's engine and C API (src/core, src/engine, src/geometry_utils, src/solver,
# c_api/src) built from the reference tree into _ref/factory/, three ways, each one shared
# library that exports the reference's C API (c_api/include/crmpm_c_api.h):
#
#   libcrmpm_factory_ref.so      the reference as it is, its own CUDA solvers included
#   libcrmpm_factory_b200.so     SimulationFactoryImpl::createScene constructing the engine's
#                                adapters (cressim-mpm_b200/adapter/gpu_b200_mpm_solver.h) in
#                                place of GpuMlsMpmSolver, GpuPbMpmSolver and GpuStandardMpmSolver:
#                                the three class names changed, and the adapter header included
#   libcrmpm_factory_b200_rb.so  the same, and SceneImpl::afterAdvance reading back the particles
#                                the scene has allocated instead of all numMaxParticles
#
# Test infrastructure only.  Nothing is copied into the repository: the two changed files are
# edited by sed in build copies under _ref/factory/, and every other file is compiled where it
# lies.  The reference's CMake is not run; the flags are its release flags (-O3 -DNDEBUG, a static
# engine, the debug logger on), with the CUDA solvers built for sm_100a.
#
# usage: build_factory.sh REF_DIR   (run from oracle/; libcrmpm_b200.so must be built first)
set -euo pipefail
REF=${1:?reference directory}
CUDA=${CUDA:-/usr/local/cuda}
NVCC=${NVCC:-$CUDA/bin/nvcc}
OUT=_ref/factory
mkdir -p "$OUT/obj" "$OUT/b200" "$OUT/b200_rb"

INC="-I$REF/include -I$REF/include/math -I$REF/include/utils -I$REF/include/core -I$REF/include/solver \
     -I$REF/include/engine -I$REF/include/geometry_utils -I$REF/src/solver -I$REF/src/core -I$REF/src/utils \
     -I$REF/src/engine -I$REF/c_api/include -I$CUDA/include"
DEFS="-DNDEBUG -DCRMPM_ENGINE_STATIC -DCR_ENABLE_DEBUG_LOGGER -DCRMPM_C_API_EXPORTS"
CXXF="-O3 -std=c++17 -fPIC -w $DEFS $INC"
NVF="-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC -w $DEFS $INC"

# every translation unit but the two that the variants change
SRCS=()
for f in "$REF"/src/core/*.cpp "$REF"/src/engine/*.cpp "$REF"/src/geometry_utils/*.cpp "$REF"/src/solver/*.cpp \
         "$REF"/c_api/src/*.cpp; do
    case "$(basename "$f")" in
        simulation_factory_impl.cpp | scene_impl.cpp) ;;
        *) SRCS+=("$f") ;;
    esac
done
CUS=("$REF"/src/solver/*.cu)

compile() { # source object compiler
    local src=$1 obj=$2
    if [ ! -f "$obj" ] || [ "$src" -nt "$obj" ]; then
        if [[ "$src" == *.cu ]]; then
            $NVCC $NVF -c "$src" -o "$obj"
        else
            g++ $CXXF -c "$src" -o "$obj"
        fi
    fi
}

pids=()
OBJS=()
for f in "${SRCS[@]}" "${CUS[@]}"; do
    o="$OUT/obj/$(basename "$f").o"
    OBJS+=("$o")
    compile "$f" "$o" &
    pids+=($!)
done

# the changed copies: the three GPU solver classes of createScene's switch, the adapter included
sed -e 's/new GpuMlsMpmSolver(/new GpuB200MlsMpmSolver(/' \
    -e 's/new GpuPbMpmSolver(/new GpuB200PbMpmSolver(/' \
    -e 's/new GpuStandardMpmSolver(/new GpuB200StandardMpmSolver(/' \
    -e 's/^#include "gpu_standard_mpm_solver.cuh"$/#include "gpu_standard_mpm_solver.cuh"\n#include "gpu_b200_mpm_solver.h"/' \
    "$REF/src/engine/simulation_factory_impl.cpp" > "$OUT/b200/simulation_factory_impl.cpp"
[ "$(grep -c 'new GpuB200\(Mls\|Pb\|Standard\)MpmSolver(' "$OUT/b200/simulation_factory_impl.cpp")" = 3 ] ||
    { echo "build_factory: the solver switch was not found" >&2; exit 1; }
grep -q '#include "gpu_b200_mpm_solver.h"' "$OUT/b200/simulation_factory_impl.cpp" ||
    { echo "build_factory: the include line was not found" >&2; exit 1; }
# the readback of afterAdvance: the allocated particles only
sed -e 's/dmParticlePositionMass, mMaxNumParticles \* sizeof(float4), cudaMemcpyKind::cudaMemcpyDeviceToHost/dmParticlePositionMass, mNumAllocatedParticles * sizeof(float4), cudaMemcpyKind::cudaMemcpyDeviceToHost/' \
    -e 's/dmParticleVelocity, mMaxNumParticles \* sizeof(Vec3f), cudaMemcpyKind::cudaMemcpyDeviceToHost/dmParticleVelocity, mNumAllocatedParticles * sizeof(Vec3f), cudaMemcpyKind::cudaMemcpyDeviceToHost/' \
    "$REF/src/engine/scene_impl.cpp" > "$OUT/b200_rb/scene_impl.cpp"
[ "$(grep -c 'mNumAllocatedParticles \* sizeof(\(float4\|Vec3f\)), cudaMemcpyKind::cudaMemcpyDeviceToHost' "$OUT/b200_rb/scene_impl.cpp")" = 2 ] ||
    { echo "build_factory: the readback lines were not found" >&2; exit 1; }

ADAPT="-I../include -I../cressim-mpm_b200/adapter"
compile "$REF/src/engine/simulation_factory_impl.cpp" "$OUT/obj/factory_ref.o" &
pids+=($!)
compile "$REF/src/engine/scene_impl.cpp" "$OUT/obj/scene_ref.o" &
pids+=($!)
g++ $CXXF $ADAPT -c "$OUT/b200/simulation_factory_impl.cpp" -o "$OUT/obj/factory_b200.o" &
pids+=($!)
g++ $CXXF -c "$OUT/b200_rb/scene_impl.cpp" -o "$OUT/obj/scene_rb.o" &
pids+=($!)
for p in "${pids[@]}"; do
    wait "$p"
done

$NVCC -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libcrmpm_factory_ref.so" "${OBJS[@]}" \
    "$OUT/obj/factory_ref.o" "$OUT/obj/scene_ref.o" -Xlinker -lpthread
$NVCC -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libcrmpm_factory_b200.so" "${OBJS[@]}" \
    "$OUT/obj/factory_b200.o" "$OUT/obj/scene_ref.o" -L../cressim-mpm_b200 -lcrmpm_b200 \
    -Xlinker -rpath -Xlinker '$ORIGIN/../../../cressim-mpm_b200' -Xlinker -lpthread
$NVCC -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libcrmpm_factory_b200_rb.so" "${OBJS[@]}" \
    "$OUT/obj/factory_b200.o" "$OUT/obj/scene_rb.o" -L../cressim-mpm_b200 -lcrmpm_b200 \
    -Xlinker -rpath -Xlinker '$ORIGIN/../../../cressim-mpm_b200' -Xlinker -lpthread
echo "built $OUT/libcrmpm_factory_{ref,b200,b200_rb}.so"
