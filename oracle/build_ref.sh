#!/usr/bin/env bash
# Builds oracle/_ref/libflsref.so: the reference's own CPU codecs
# (src/fls/*.cpp, src/alp/falp.cpp, src/alp/alp-bindings.cu, compiled from
# where they lie in the reference checkout) plus oracle/ref_shim.cu.
# TEST INFRASTRUCTURE ONLY: used to pin the oracle and as the timed CPU
# baseline.  Flags follow the reference's CPU build without -march=native
# (src/alp/encoder.hpp:342-350 does not compile under AVX-512) and with
# -ffp-contract=off (the ALP encoder's rounding trick must not become an FMA).
set -euo pipefail
REF="${1:-${FLSGPU_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF/src/fls" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
CXXFLAGS="-std=c++17 -O3 -fPIC -ffp-contract=off -w"
pids=()
for f in pack unpack ffor unffor; do
  if [ ! -f "$OUT/obj/fls-$f.o" ] || [ "$REF/src/fls/$f.cpp" -nt "$OUT/obj/fls-$f.o" ]; then
    g++ $CXXFLAGS -c "$REF/src/fls/$f.cpp" -o "$OUT/obj/fls-$f.o" & pids+=($!)
  fi
done
if [ ! -f "$OUT/obj/alp-falp.o" ]; then
  g++ $CXXFLAGS -c "$REF/src/alp/falp.cpp" -o "$OUT/obj/alp-falp.o" & pids+=($!)
fi
NVFLAGS="-Wno-deprecated-gpu-targets -std=c++17 -O3 --expt-relaxed-constexpr -Xcompiler -fPIC,-ffp-contract=off -w -I$REF -diag-suppress 3033,3356"
nvcc $NVFLAGS -c "$REF/src/alp/alp-bindings.cu" -o "$OUT/obj/alp-bindings.o" & pids+=($!)
nvcc $NVFLAGS -c "$HERE/ref_shim.cu" -o "$OUT/obj/ref_shim.o" & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
nvcc -shared -o "$OUT/libflsref.so" "$OUT"/obj/*.o
echo "built $OUT/libflsref.so"
