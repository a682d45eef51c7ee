#!/bin/bash
# Builds the reference's particle-FMM C interface (src/pvfmm-wrapper.cpp and
# the src/*.cpp it needs) from the read-only reference tree, over the
# stand-ins in shim/ (SCTL subset, single-rank MPI, configuration header),
# into oracle/_ref/libpvfmm_ref_<isa>.so: one library for AVX2+FMA hosts and
# one for AVX-512 hosts.  BLAS/LAPACK: the OpenBLAS that scipy bundles.
# Test infrastructure only (oracle pins, golden fixtures, CPU baseline).
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${PVFMM_REFERENCE:-/root/reference}"
OUT="$HERE/../_ref"
if [ ! -d "$REF/src" ] || [ ! -d "$REF/include" ]; then
  echo "reference sources not found at $REF: checker not built"
  exit 0
fi
PY="${PYTHON:-python3}"
BLAS_DIR="$($PY -c 'import scipy, os; print(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs"))')"
BLAS_LIB="$(ls "$BLAS_DIR"/libscipy_openblas*.so | head -1)"
mkdir -p "$OUT"
SRCS="$REF/src/profile.cpp $REF/src/mem_mgr.cpp $REF/src/tree_node.cpp $REF/src/mortonid.cpp \
      $REF/src/cheb_utils.cpp $REF/src/legendre_rule.cpp $HERE/ref_driver.cpp $HERE/mpi_stub.cpp"
build() {  # isa flags, library suffix
  local flags="$1" tag="$2" obj="$OUT/obj_$2"
  mkdir -p "$obj"
  local objs=""
  for s in $SRCS; do
    local o="$obj/$(basename "$s" .cpp).o"
    if [ ! -f "$o" ] || [ "$s" -nt "$o" ] || [ -n "$(find "$HERE/shim" -newer "$o" 2>/dev/null)" ]; then
      g++ -O3 -std=gnu++17 -fopenmp -fPIC $flags -ffp-contract=fast -w -DNDEBUG \
          -I "$HERE/shim" -I "$REF/include" -I "$REF/src" -c "$s" -o "$o"
    fi
    objs="$objs $o"
  done
  g++ -shared -fopenmp -o "$OUT/libpvfmm_ref_$tag.so" $objs "$BLAS_LIB" -Wl,-rpath,"$BLAS_DIR"
}
build "-march=x86-64-v3" avx2 &
build "-march=x86-64-v4" avx512 &
# periodic boundaries without PVFMM_EXTENDED_BC (the lattice sum of all images)
build "-march=x86-64-v3 -DPVFMM_REF_LATTICE_BC" avx2_lattice &
wait %1 && wait %2 && wait %3
