#!/bin/sh
# Build oracle/_ref/libref.so: RBMD's own force-path code compiled from the reference tree
# (read in place, never copied into the repository) against the VTK-m stand-in in
# oracle/ref_shim, driven by oracle/ref_harness.cpp.  Test infrastructure.
#
# The reference location is the first argument, else $RBMD_REFERENCE, else /root/reference.
# Outputs go to oracle/_ref/ only (git-ignored): two line ranges of the reference's sources that
# hold class definitions outside any header (the worklet structs of RunWorklet.cpp and the
# BinPointsWorklet of ContPointLocator.cxx) are extracted there, then compiled with the harness.
# -ffp-contract=off keeps every float operation rounded as written, as VTK-m's host build does.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${RBMD_REFERENCE:-/root/reference}}"
FW="$REF/rbmd/framework"
if [ ! -f "$FW/run/worklet/RunWorklet.cpp" ]; then
  echo "build_ref.sh: no reference tree at $REF" >&2
  exit 2
fi
OUT="$HERE/_ref"
mkdir -p "$OUT"
# RunWorklet.cpp:40-1913 are the worklet structs of namespace RunWorklet (the dispatch
# functions that follow need VTK-m's control environment and are not compiled)
{ echo 'namespace RunWorklet {'; sed -n '40,1913p' "$FW/run/worklet/RunWorklet.cpp"; echo '}'; } > "$OUT/run_worklets.inc"
# ContPointLocator.cxx:35-68: namespace internal { class BinPointsWorklet }
sed -n '35,68p' "$FW/locator/ContPointLocator.cxx" > "$OUT/bin_points.inc"
g++ -O2 -std=c++17 -ffp-contract=off -fopenmp -fPIC -shared -w \
  -I "$HERE/ref_shim" -I "$FW" -I "$OUT" \
  -o "$OUT/libref.so.tmp" "$HERE/ref_harness.cpp"
mv "$OUT/libref.so.tmp" "$OUT/libref.so"
