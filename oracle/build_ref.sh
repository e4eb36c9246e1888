#!/usr/bin/env bash
# Build the reference's own CPU FP64 modules (local_kernels, kernelmath,
# fchl19_repr, kitchen_sinks = the random-Fourier-feature module) from their sources under the reference checkout, into
# oracle/_ref/ (git-ignored).  TEST INFRASTRUCTURE ONLY: the result is the
# "reference" CPU arm of bench.py and the generator of tests/golden fixtures.
#
# The reference normally links a system CBLAS/LAPACK through CMake.  This box
# has no BLAS headers, so a small shim maps the CBLAS / LAPACK names the
# reference calls onto the LP64 OpenBLAS that scipy ships (exported names
# scipy_cblas_*, scipy_d*_, scipy_openblas_*).  The reference's -ffast-math is
# dropped so the oracle is strict FP64.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-/root/reference}"
OUT="$HERE/_ref"
SRC="$REF/src"
if [ ! -d "$SRC" ]; then
    echo "reference sources not found at $SRC" >&2
    exit 1
fi
PY="${PYTHON:-python3}"
SCIPY_LIBS="$($PY -c 'import scipy, os; print(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs"))')"
OPENBLAS="$(ls "$SCIPY_LIBS"/libscipy_openblas-*.so | head -1)"
PYINC="$($PY -m pybind11 --includes)"
EXT="$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')"
mkdir -p "$OUT/shim"

cat > "$OUT/shim/cblas.h" <<'EOF'
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER {CblasRowMajor=101, CblasColMajor=102};
enum CBLAS_TRANSPOSE {CblasNoTrans=111, CblasTrans=112, CblasConjTrans=113};
enum CBLAS_UPLO {CblasUpper=121, CblasLower=122};
typedef enum CBLAS_ORDER CBLAS_LAYOUT;
void scipy_cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, int, int, int,
                       double, const double*, int, const double*, int, double, double*, int);
void scipy_cblas_dsyrk(enum CBLAS_ORDER, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, int, int, double,
                       const double*, int, double, double*, int);
void scipy_cblas_dgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, int, int, double, const double*, int,
                       const double*, int, double, double*, int);
void scipy_cblas_dger(enum CBLAS_ORDER, int, int, double, const double*, int, const double*, int,
                      double*, int);
void scipy_cblas_daxpy(int, double, const double*, int, double*, int);
double scipy_cblas_ddot(int, const double*, int, const double*, int);
#ifdef __cplusplus
}
#endif
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dsyrk scipy_cblas_dsyrk
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dger scipy_cblas_dger
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_ddot scipy_cblas_ddot
EOF

cat > "$OUT/shim/glue.cpp" <<'EOF'
extern "C" int scipy_openblas_get_num_threads(void);
extern "C" void scipy_openblas_set_num_threads(int);
extern "C" int openblas_get_num_threads(void) { return scipy_openblas_get_num_threads(); }
extern "C" void openblas_set_num_threads(int n) { scipy_openblas_set_num_threads(n); }
EOF

LAPACK_DEFS=""
for f in dpftrf dpftrs dtrttf dtfttr dpotrf dpotrs dgels dgelsd dgetrf dgecon dlange dsfrk; do
    LAPACK_DEFS="$LAPACK_DEFS -D${f}_=scipy_${f}_"
done
CXXFLAGS="-O3 -fopenmp -std=c++17 -shared -fPIC -w $PYINC -I$OUT/shim -I$SRC $LAPACK_DEFS"
LDFLAGS="$OPENBLAS -Wl,-rpath,$SCIPY_LIBS -fopenmp"

build() {
    local name="$1"; shift
    echo "building $name"
    g++ $CXXFLAGS "$@" "$OUT/shim/glue.cpp" -o "$OUT/$name$EXT" $LDFLAGS
}
build local_kernels "$SRC/local_kernels.cpp" "$SRC/local_kernels_bindings.cpp" &
build kernelmath "$SRC/math.cpp" "$SRC/math_bindings.cpp" &
build fchl19_repr "$SRC/fchl19_repr.cpp" "$SRC/fchl19_repr_bindings.cpp" &
build kitchen_sinks "$SRC/rff_features.cpp" "$SRC/rff_features_bindings.cpp" \
    "$SRC/rff_elemental.cpp" "$SRC/rff_elemental_bindings.cpp" &
wait
echo "reference modules in $OUT"
