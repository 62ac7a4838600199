#!/usr/bin/env bash
# Builds the reference (carlidel/henon_map_cpp) pybind11 module from its own
# sources, unmodified, into oracle/_ref/<variant>/ -- the checker for parity
# tests and the CPU baseline of bench.py.  Nothing here is part of the
# library.  The reference's CMake build is not used: the four sources are
# compiled directly, with cuFFTW standing in for FFTW3 (oracle/shim/fftw3.h).
#
# Variants:
#   fmad_off : CUDA code built with --fmad=false (no FMA contraction), so the
#              reference GPU path does the same arithmetic as its CPU path
#   default  : CUDA code built as shipped (nvcc's default --fmad=true)
# Host code: g++ -O3 without -march (plain SSE2 binary64, no FMA).
#
# REF must name the reference checkout (its src/ directory is compiled).
set -euo pipefail
: "${REF:?set REF to the reference checkout (the directory holding src/henon.cu)}"
HERE=$(cd "$(dirname "$0")" && pwd)
CUDA=${CUDA_HOME:-/usr/local/cuda}
PY=${PYTHON:-python3}
if [ ! -d "$REF/src" ]; then
  echo "reference sources not found at $REF/src" >&2
  exit 2
fi
PYINC=$($PY -m pybind11 --includes)
SUFFIX=$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
ARCH="-gencode arch=compute_100a,code=sm_100a"
VARIANTS=${VARIANTS:-"fmad_off default"}
for v in $VARIANTS; do
  OUT="$HERE/_ref/$v"
  OBJ="$OUT/obj"
  mkdir -p "$OBJ"
  FMAD=""
  [ "$v" = "fmad_off" ] && FMAD="--fmad=false"
  # modulation.cpp uses std::runtime_error without including <stdexcept>.
  g++ -O3 -std=c++17 -fPIC -DPYBIND -include stdexcept -I"$HERE/shim" -I"$CUDA/include" \
      -I"$REF/src" $PYINC -c "$REF/src/modulation.cpp" -o "$OBJ/modulation.o"
  g++ -O3 -std=c++17 -fPIC -DPYBIND -include stdexcept -I"$HERE/shim" -I"$CUDA/include" \
      -I"$REF/src" $PYINC -c "$REF/src/dynamic_indicator.cpp" -o "$OBJ/dynamic_indicator.o"
  "$CUDA/bin/nvcc" -O3 -std=c++17 -DPYBIND -Xcompiler -fPIC $ARCH $FMAD -I"$HERE/shim" \
      -I"$REF/src" $PYINC -c "$REF/src/henon.cu" -o "$OBJ/henon.o"
  "$CUDA/bin/nvcc" -O3 -std=c++17 -DPYBIND -Xcompiler -fPIC $ARCH $FMAD -I"$HERE/shim" \
      -I"$REF/src" $PYINC -x cu -c "$REF/src/bind.cpp" -o "$OBJ/bind.o"
  "$CUDA/bin/nvcc" -shared $ARCH -o "$OUT/henon_map_engine$SUFFIX" "$OBJ"/*.o \
      -lcufftw -lcufft -lcurand -lpthread
  echo "built $OUT/henon_map_engine$SUFFIX"
done
