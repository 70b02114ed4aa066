#!/usr/bin/env bash
# Builds _ref/liboracle_ref.so: the FASP++ reference solvers compiled from their own
# source tree (the first argument, else $FASPXX_REFERENCE, else the default below; read
# only) plus ref_shim.cxx, for use as a test
# oracle and as the timed CPU baseline. Sources are copied to a temporary directory, the
# build-time fixes below are applied there, and only the shared library lands in _ref/.
#   1. GMRES.cxx:214,224,386,396 / FGMRES.cxx:209,219: unsigned back-substitution loops
#      `for (USI k = count - 2; k >= 0; --k)` never end; made signed.
#   2. VEC.cxx:121: VEC::SetValues(size, array) writes into an unsized vector; resize it.
#   3. CG.cxx:213: `pk.SetValues(0.0)` shrinks pk to length 0; give it its length.
#   4. GMRES.cxx:53 / FGMRES.cxx:39: `var` is indexed up to maxRestart; size it for that.
# Compiled with -O2 -ffp-contract=off so that results are bit-comparable with the C
# restatement (fasp_oracle.c), which is built with the same flags.
set -euo pipefail
REF="${1:-${FASPXX_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
    echo "build_ref.sh: no reference tree at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
cp "$REF"/src/*.cxx "$REF"/src/*.hxx "$REF"/include/Faspxx.hxx "$TMP"/
sed -i -e 's/for (USI k = count - 2; k >= 0; --k)/for (INT k = (INT)count - 2; k >= 0; --k)/' \
       -e 's/for (USI j = count - 2; j >= 0; --j)/for (INT j = (INT)count - 2; j >= 0; --j)/' \
       -e 's/var.resize(len);/var.resize(len > maxRestart + 1 ? len : maxRestart + 1);/' \
       "$TMP/GMRES.cxx" "$TMP/FGMRES.cxx"
sed -i -e 's|INT i; // OpenMP only allows INT|INT i; this->values.resize(size); // OpenMP only allows INT|' \
       "$TMP/VEC.cxx"
sed -i -e 's/this->pk.SetValues(0.0);/this->pk.SetValues(len, 0.0);/' "$TMP/CG.cxx"
for f in GMRES.cxx FGMRES.cxx VEC.cxx CG.cxx; do
    if cmp -s "$REF/src/$f" "$TMP/$f"; then echo "build_ref.sh: patch did not apply to $f" >&2; exit 1; fi
done
SRCS=""
for f in "$TMP"/*.cxx; do
    case "$(basename "$f")" in
        Umfpack.cxx|Timing.cxx) ;;   # direct solver stub and wall clock: not on the path
        *) SRCS="$SRCS $f" ;;
    esac
done
g++ -std=c++17 -O2 -ffp-contract=off -fPIC -shared -w -I"$TMP" -I"$HERE" \
    $SRCS "$HERE/ref_shim.cxx" -o "$OUT/liboracle_ref.so.tmp"
mv "$OUT/liboracle_ref.so.tmp" "$OUT/liboracle_ref.so"
echo "built $OUT/liboracle_ref.so"
# The reference's own matrix-free example (example/TestMatFree.cxx, with its Poisson2D.hxx),
# built from the same patched sources; tests/golden/make_golden.py records what it prints.
if [ -f "$REF/example/TestMatFree.cxx" ]; then
    cp "$REF/example/TestMatFree.cxx" "$REF/example/Poisson2D.hxx" "$TMP"/
    g++ -std=c++17 -O2 -ffp-contract=off -w -I"$TMP" $SRCS "$TMP/Timing.cxx" \
        "$TMP/TestMatFree.cxx" -o "$OUT/test_matfree.tmp"
    mv "$OUT/test_matfree.tmp" "$OUT/test_matfree"
    echo "built $OUT/test_matfree"
fi
