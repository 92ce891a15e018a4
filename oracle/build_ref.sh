#!/bin/sh
# Builds oracle/_ref/libgxref.so from the reference's own hot-path sources,
# compiled in place from a reference checkout (the first argument, else
# $GX_REFERENCE_ROOT, else a directory named `reference` beside the
# repository), through the headers in oracle/refshim.  Test
# infrastructure only: the library pins the oracle and generates the golden
# vectors.  The reference's own build system is not used (it needs cmake and
# its empty VecCore/VecGeom/PTL/timemory submodules).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${GX_REFERENCE_ROOT:-$HERE/../../reference}}
OUT="$HERE/_ref"
SRC="$REF/source/Geant"
if [ ! -d "$SRC" ]; then
  echo "build_ref.sh: no reference checkout at $REF" >&2
  exit 2
fi
mkdir -p "$OUT"
# link the system libstdc++ dynamically: a static copy inside a library that a
# Python process loads next to another libstdc++ crashes in iostream set-up
STDCXX=$(${CXX:-g++} -print-file-name=libstdc++.so.6)
case "$STDCXX" in /*) ;; *) STDCXX=/usr/lib/x86_64-linux-gnu/libstdc++.so.6 ;; esac
${CXX:-g++} -std=c++14 -O2 -fPIC -shared -w -x c++ \
  -I"$HERE/refshim" -I"$REF/source" \
  "$HERE/refshim/ref_capi.cpp" \
  "$SRC/random/src/MRG32k3a.cpp" \
  "$SRC/proxy/src/Proxy2DVector.cpp" \
  "$SRC/proxy/src/ProxyPhysicsVector.cu" \
  "$SRC/proxy/src/ProxyPhysicsTable.cu" \
  "$SRC/proxy/src/ProxyDataManager.cu" \
  "$SRC/proxy/src/ProxyEgammaGun.cpp" \
  "$SRC/proxy/src/ProxyHepEvtGenerator.cpp" \
  -x none "$STDCXX" -lm -o "$OUT/libgxref.so"
# the production-cut converter, with its own material shims (oracle/refshim_cuts)
${CXX:-g++} -std=c++14 -O2 -fPIC -shared -w -x c++ \
  -I"$HERE/refshim_cuts" -I"$HERE/refshim" -I"$REF/source" \
  "$HERE/refshim_cuts/cut_capi.cpp" \
  "$SRC/cuts/src/CutConverter.cpp" \
  "$SRC/cuts/src/CutConverterForGamma.cpp" \
  "$SRC/cuts/src/CutConverterForElectron.cpp" \
  "$SRC/cuts/src/CutConverterForPositron.cpp" \
  "$SRC/cuts/src/Spline.cpp" \
  -x none "$STDCXX" -lm -o "$OUT/libgxref_cuts.so"
# the CMS field-map reader of the reference's field example, with its own shims
${CXX:-g++} -std=c++14 -O2 -fPIC -shared -w -x c++ \
  -I"$HERE/refshim_field" -I"$REF/examples/magneticfield/simplifiedCMS/inc" \
  "$HERE/refshim_field/field_capi.cpp" \
  -x none "$STDCXX" -lm -o "$OUT/libgxref_field.so"
echo "built $OUT/libgxref.so $OUT/libgxref_cuts.so $OUT/libgxref_field.so"
