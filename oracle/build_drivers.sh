#!/usr/bin/env bash
# Compiles the reference's UNMODIFIED experiment drivers (scripts/common.py,
# scripts/methods_convergence.py and scripts/utils/{methods,typst,
# backward_error}.py) with Cython into extension modules under
# oracle/_ref/drivers/, and puts the reference's ten sample matrices and its
# recorded result CSVs (results_sample) beside them.  The drivers import
# `methods_cython`, which the tests resolve to this library's compat shims, so
# the reference's own driver code runs against libspai_b200.so on a GPU box
# that has no reference tree.  Outputs only under oracle/_ref/drivers/.
# Usage: build_drivers.sh <reference-root> <repo-root>
set -euo pipefail
REF="${1:-/root/reference}"
ROOT="${2:-$(cd "$(dirname "$0")/.." && pwd)}"
SCRIPTS="$REF/scripts"
OUT="$ROOT/oracle/_ref/drivers"
if [ ! -f "$SCRIPTS/common.py" ]; then
  echo "reference drivers not found: $SCRIPTS" >&2
  exit 1
fi
PY=${PYTHON:-python}
EXT=$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
INC=$($PY -c 'import sysconfig; print(sysconfig.get_paths()["include"])')
mkdir -p "$OUT/scripts/utils" "$OUT/scripts/sample_datasets" "$OUT/recorded"
# the two package markers are empty in the reference too
: > "$OUT/scripts/__init__.py"
: > "$OUT/scripts/utils/__init__.py"

compile() {  # <source .py> <module name> <output path without suffix>
  local src="$1" name="$2" dst="$3"
  local c="$OUT/c/$name.c"
  mkdir -p "$OUT/c"
  if [ ! -f "$dst$EXT" ] || [ "$src" -nt "$dst$EXT" ]; then
    $PY -m cython -3 --module-name "$name" "$src" -o "$c"
    /usr/bin/gcc -O1 -fPIC -shared -I"$INC" "$c" -o "$dst$EXT"
  fi
}
# common and methods_convergence are imported as top-level modules (the
# scripts directory is on sys.path); the utils as the scripts.utils package
compile "$SCRIPTS/common.py" common "$OUT/scripts/common"
compile "$SCRIPTS/methods_convergence.py" methods_convergence "$OUT/scripts/methods_convergence"
for m in methods typst backward_error; do
  compile "$SCRIPTS/utils/$m.py" "scripts.utils.$m" "$OUT/scripts/utils/$m"
done

# data: the sample matrices (read by the drivers as-is) and the recorded CSVs
for f in "$SCRIPTS"/sample_datasets/*-dataset.mtx; do
  [ -f "$OUT/scripts/sample_datasets/$(basename "$f")" ] || cp "$f" "$OUT/scripts/sample_datasets/"
done
( cd "$SCRIPTS/results/results_sample" && find . -name '*.csv' ) | while read -r rel; do
  mkdir -p "$OUT/recorded/$(dirname "$rel")"
  cp "$SCRIPTS/results/results_sample/$rel" "$OUT/recorded/$rel"
done
# the translated C is an intermediate; only the extension modules are kept
rm -rf "$OUT/c"
echo "built $OUT"
