#!/usr/bin/env bash
# Compiles the reference's PCG evaluator (methods_cython/backward_error.pyx) from
# the reference source tree into oracle/_ref/ so tests and the CPU baseline can
# run the reference's own code.  Usage: build_ref.sh <reference-root> <out-dir>
set -euo pipefail
REF="${1:-/root/reference}"
OUT="${2:-$(dirname "$0")/_ref}"
SRC="$REF/methods_cython/backward_error.pyx"
if [ ! -f "$SRC" ]; then
  echo "reference source not found: $SRC" >&2
  exit 1
fi
mkdir -p "$OUT"
PY=${PYTHON:-python}
EXT=$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
INC=$($PY -c 'import sysconfig; print(sysconfig.get_paths()["include"])')
$PY -m cython --cplus -3 "$SRC" -o "$OUT/backward_error.cpp"
/usr/bin/g++ -O3 -fPIC -shared -fopenmp -I"$INC" "$OUT/backward_error.cpp" -o "$OUT/backward_error$EXT"
echo "built $OUT/backward_error$EXT"
