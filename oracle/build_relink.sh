#!/usr/bin/env bash
# Compiles the reference's UNMODIFIED Cython binding methods_cython/methods.pyx
# from the reference source tree against this repository's include/methods_c_api.h
# and links it to libspai_b200.so, into oracle/_ref/relinked/.  This is the
# relink a user of the reference makes to switch libraries; the tests import
# the result to replay the reference's recorded runs through it.
# Usage: build_relink.sh <reference-root> <repo-root>
set -euo pipefail
REF="${1:-/root/reference}"
ROOT="${2:-$(cd "$(dirname "$0")/.." && pwd)}"
SRC="$REF/methods_cython/methods.pyx"
PKG="$ROOT/parallellocallyoptimalapproximatesparsematrixinverses_b200"
OUT="$ROOT/oracle/_ref/relinked"
if [ ! -f "$SRC" ]; then
  echo "reference source not found: $SRC" >&2
  exit 1
fi
if [ ! -f "$PKG/libspai_b200.so" ]; then
  echo "libspai_b200.so is not built: $PKG" >&2
  exit 1
fi
mkdir -p "$OUT"
PY=${PYTHON:-python}
EXT=$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
INC=$($PY -c 'import sysconfig; print(sysconfig.get_paths()["include"])')
$PY -m cython --cplus -3 "$SRC" -o "$OUT/methods.cpp"
# $ORIGIN/../../.. is the repository root wherever the tree is copied
/usr/bin/g++ -O2 -fPIC -shared -I"$INC" -I"$ROOT/include" "$OUT/methods.cpp" -o "$OUT/methods$EXT" \
  -L"$PKG" -lspai_b200 -Wl,-rpath,'$ORIGIN/../../../parallellocallyoptimalapproximatesparsematrixinverses_b200'
echo "built $OUT/methods$EXT"
