#!/usr/bin/env bash
# Builds the XnYZip reference from its own sources, where they lie, into oracle/_ref/:
#   oracle/_ref/xnyzip_ref      the reference CLI (source/main.cpp, unmodified)
#   oracle/_ref/libxnyz_ref.so  oracle/ref_driver.cpp over the unmodified reference headers
# Eigen 3.4 and zstd.h are absent on this image: oracle/shim/ supplies a minimal Eigen
# stand-in and the zstd declarations; the zstd runtime is the libzstd 1.5.7 shared
# library bundled on the image (the version the reference pins in its conanfile).
# Flags follow the reference's Linux conan profile (-O3, no -march, so no FMA).
# Test infrastructure only; never part of the product.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${XNYZ_REFERENCE:-/root/reference}"
if [ ! -d "$REF/source" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
ZSTD_LIB="${XNYZ_ZSTD_LIBRARY:-$(python3 "$HERE/find_zstd.py")}"
ZSTD_DIR="$(dirname "$ZSTD_LIB")"
ZSTD_NAME="$(basename "$ZSTD_LIB")"
OUT="$HERE/_ref"
mkdir -p "$OUT"
CXX="${XNYZ_CXX:-/usr/bin/g++}"  # not $CXX: this image points it at a g++ that links libstdc++ statically
FLAGS=(-O3 -std=c++20 -I"$HERE/shim" -I"$REF/source" -w)
LINK=(-L"$ZSTD_DIR" -l:"$ZSTD_NAME" -Wl,-rpath,"$ZSTD_DIR")
"$CXX" "${FLAGS[@]}" "$REF/source/main.cpp" "$REF/source/quantizer/hilbert-curves-cpp/hilbert.cpp" \
  -o "$OUT/xnyzip_ref" "${LINK[@]}"
"$CXX" "${FLAGS[@]}" -fPIC -shared "$HERE/ref_driver.cpp" "$REF/source/quantizer/hilbert-curves-cpp/hilbert.cpp" \
  -o "$OUT/libxnyz_ref.so" "${LINK[@]}"
echo "built $OUT/xnyzip_ref and $OUT/libxnyz_ref.so (zstd: $ZSTD_LIB)"
