#!/usr/bin/env bash
# Builds the reference's own RHS/RK3 kernels for sm_100a from the reference
# sources where they lie (read-only), plus oracle/ref_cuda_harness.cu, into
# oracle/_ref/libostc_ref_cuda.so. Test and measurement infrastructure only.
#
# What the reference's CMake build needs and this recipe replaces:
#   - MPI: a single-rank header shim (oracle/ref_shim/mpi.h), no library;
#   - fmt: header-only mode from the reference's vendored headers
#     (depends/include, FMT_HEADER_ONLY); the prebuilt depends/lib/* are not used;
#   - MAX_SPEC_NUMBER=20, MAX_REAC_NUMBER=50, GPU: the reference's CMake defines.
# Objects go to oracle/_ref/obj; rebuilt only when the harness changes.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${OSTC_REFERENCE_DIR:-/root/reference}"
SRC="$REF/src"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
LIB="$OUT/libostc_ref_cuda.so"
if [ ! -d "$SRC" ]; then echo "reference sources not found at $SRC; skipping"; exit 0; fi
if [ -f "$LIB" ] && [ "$LIB" -nt "$HERE/ref_cuda_harness.cu" ] && [ "$LIB" -nt "$HERE/build_ref.sh" ] \
   && [ "$LIB" -nt "$HERE/ref_shim/mpi.h" ] && [ "$LIB" -nt "$HERE/../include/ostc_reference_shim.h" ] \
   && [ "$LIB" -nt "$HERE/../include/ostc.h" ]; then exit 0; fi
mkdir -p "$OBJ"
NVCC="${NVCC:-nvcc}"
FLAGS=(-gencode arch=compute_100a,code=sm_100a -rdc=true -std=c++20 -O3 -Xcompiler -fPIC
       -DMAX_SPEC_NUMBER=20 -DMAX_REAC_NUMBER=50 -DGPU -DFMT_HEADER_ONLY
       -I"$HERE/ref_shim" -I"$REF/depends/include" -I"$SRC" -w)
UNITS=(Thermo.cu Transport.cu FiniteRateChem.cu AusmP.cu HLLC.cu LaxFriedrichs.cu AWENO.cu Reconstruction.cu
       InviscidScheme.cu Roe.cu FieldOperation.cu SST.cu TimeAdvanceFunc.cu Residual.cu DPLUR.cu Parameter.cpp
       gxl_lib/MyString.cpp gxl_lib/Time.cpp Mesh.cpp Parallel.cpp Parallel.cu)
# host-only units go through the host compiler: nvcc's front end rejects the
# consteval format strings of header-only fmt 10
HOSTFLAGS=(-std=c++20 -O2 -fPIC -DMAX_SPEC_NUMBER=20 -DMAX_REAC_NUMBER=50 -DGPU -DFMT_HEADER_ONLY
           -I"$HERE/ref_shim" -I"$REF/depends/include" -I"$SRC" -w)
pids=()
objs=()
for u in "${UNITS[@]}"; do
  o="$OBJ/$(echo "$u" | tr '/' '_').o"
  objs+=("$o")
  if [ -f "$o" ]; then continue; fi
  if [[ "$u" == *.cpp ]]; then
    g++ "${HOSTFLAGS[@]}" -c "$SRC/$u" -o "$o" &
  else
    "$NVCC" "${FLAGS[@]}" -c "$SRC/$u" -o "$o" &
  fi
  pids+=($!)
done
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_cuda_harness.cu" -o "$OBJ/harness.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC -o "$LIB.tmp" "${objs[@]}" "$OBJ/harness.o" -lcudart
mv "$LIB.tmp" "$LIB"
echo "built $LIB"
