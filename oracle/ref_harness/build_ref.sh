#!/usr/bin/env bash
# Builds the reference's own CUDA kernels (from the reference sources, read in
# place and patched in a scratch copy) into oracle/_ref/ as the parity oracle.
# The copy is deleted after the build; only binaries land in oracle/_ref/.
#
# Patches (each a defect of the reference that would make the oracle read out
# of bounds or compute something other than the intended scheme):
#   Transport.cu:88     X[i] -> X[l]  (grid index used as species index)
#   ViscousScheme.cu:317 rho_D(i,j+1,k) -> rho_D(i,j,k+1) on zeta faces
#   Field.cu:216        blockDim.y + blockIdx.y -> blockDim.y * blockIdx.y
# The un-vendored gxl_lib containers and a one-rank mpi.h come from
# oracle/ref_harness/shim (containers only, no arithmetic).
set -euo pipefail
REF=${CC_REFERENCE_DIR:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$(cd "$HERE/.." && pwd)/_ref
if [ ! -f "$REF/Transport.cu" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref build" >&2
  exit 0
fi
mkdir -p "$OUT"
WORK=$(mktemp -d /tmp/ccref.XXXXXX)
trap 'rm -rf "$WORK"' EXIT
cp "$REF"/*.cu "$REF"/*.cuh "$REF"/*.cpp "$REF"/*.h "$WORK"/
sed -i '88s/X\[i\]/X[l]/' "$WORK/Transport.cu"
sed -i '317s/rho_D(i, j + 1, k, l)/rho_D(i, j, k + 1, l)/' "$WORK/ViscousScheme.cu"
sed -i '216s/blockDim.y + blockIdx.y/blockDim.y * blockIdx.y/' "$WORK/Field.cu"
grep -q 'abs(X\[l\]-1)' "$WORK/Transport.cu"
[ "$(sed -n 317p "$WORK/ViscousScheme.cu" | grep -c 'rho_D(i, j, k + 1, l)')" = 1 ]
grep -q 'blockDim.y \* blockIdx.y + threadIdx.y' "$WORK/Field.cu"
TORCH_INC=$(python -c "import torch,os;print(os.path.join(os.path.dirname(torch.__file__),'include'))")
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
SRCS="Field.cu TimeAdvanceFunc.cu InviscidScheme.cu Reconstruction.cu ViscousScheme.cu Thermo.cu Transport.cu TemporalScheme.cu BoundCond.cu BoundCond.cpp ChemData.cpp Element.cpp Parameter.cpp Mesh.cpp"
for MS in 1 0; do
  OBJ="$WORK/obj$MS"
  mkdir -p "$OBJ"
  FLAGS="-std=c++20 -O2 $ARCH -rdc=true -DGPU -DMULTISPECIES=$MS -DFMT_HEADER_ONLY -w -I$HERE/shim -I$HERE/shim/mpi -I$WORK -isystem $TORCH_INC"
  pids=()
  for s in $SRCS; do
    $NVCC $FLAGS -x cu -c "$WORK/$s" -o "$OBJ/${s}.o" &
    pids+=($!)
  done
  $NVCC $FLAGS -x cu -c "$HERE/harness.cu" -o "$OBJ/harness.o" &
  pids+=($!)
  for p in "${pids[@]}"; do wait "$p"; done
  NAME=ref_harness_ms; [ "$MS" = 0 ] && NAME=ref_harness_air
  $NVCC $ARCH -rdc=true "$OBJ"/*.o -o "$OUT/$NAME"
done
echo "built $OUT/ref_harness_ms $OUT/ref_harness_air"
