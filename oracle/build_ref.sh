#!/usr/bin/env bash
# Test infrastructure: compiles the SPAMS reference's own omp / lasso code
# (header-only C++ under the reference checkout) together with
# oracle/ref_driver.cpp into oracle/_ref/libspams_ref.so.  Nothing is copied
# out of the reference tree: the headers are used in place through -I.
#
# BLAS/LAPACK: the reference calls Fortran BLAS symbols (dgemv_, idamax_, ...
# linalg/cblas_alt_template.h:291-365).  This image has no system libblas, so
# the build links SciPy's bundled LP64 OpenBLAS, whose symbols carry a
# "scipy_" prefix; a generated forced-include header renames each symbol.
# The ILP64 numpy OpenBLAS must not be used: the reference's INTT is int.
#
# Usage: oracle/build_ref.sh [REFERENCE_DIR]
#   REFERENCE_DIR: the argument, else $SPAMS_REFERENCE_DIR.  Exits 2 when
#   neither is given or no reference sources are found there.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${SPAMS_REFERENCE_DIR:-}}"
OUT="$HERE/_ref"
if [ -z "$REF" ] || [ ! -d "$REF/decomp" ]; then
  echo "build_ref: reference sources not found at $REF" >&2
  exit 2
fi
PY="${PYTHON:-python}"
SCIPY_LIBS="$("$PY" -c 'import scipy, os; print(os.path.join(os.path.dirname(scipy.__file__), os.pardir, "scipy.libs"))')"
SCIPY_LIBS="$(cd "$SCIPY_LIBS" && pwd)"
BLAS="$(ls "$SCIPY_LIBS"/libscipy_openblas-*.so | grep -v openblas64 | head -1)"
mkdir -p "$OUT"
RENAME="$OUT/blas_rename.h"
{
  echo "/* generated by oracle/build_ref.sh: map Fortran BLAS names to SciPy's OpenBLAS */"
  for s in dasum daxpby daxpy dcopy ddot dgemm dgemv dger dgesvd dlasrt dscal \
           dsyev dsymv dsyr dsyrk dsytrf dsytri dtrmm dtrmv dtrtri idamax \
           isamax sasum saxpby saxpy scopy sdot sgemm sgemv sger sgesvd slasrt \
           sscal ssyev ssymv ssyr ssyrk ssytrf ssytri strmm strmv strtri \
           dnrm2 snrm2; do
    echo "#define ${s}_ scipy_${s}_"
  done
} > "$RENAME"
set -x
g++ -std=c++14 -O3 -fopenmp -DNDEBUG -DUSE_BLAS_LIB -fPIC -shared -w \
  -include "$RENAME" \
  -I"$REF/cpp_library" -I"$REF/linalg" -I"$REF/decomp" -I"$REF/prox" -I"$REF/dictLearn" \
  "$HERE/ref_driver.cpp" -o "$OUT/libspams_ref.so" \
  "$BLAS" -Wl,-rpath,"$SCIPY_LIBS"
