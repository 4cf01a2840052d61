#!/bin/sh
# Builds the oracle's reference pins from the reference's own sources, where
# they lie under the read-only reference tree (nothing is copied).  Output goes
# only to oracle/_ref/.  Needs the reference tree, so it runs only where that
# tree is present; elsewhere the prebuilt files are used as they are.
#   _ref/libctref.so   the vendored cryptoTools AES and PRNG
#                      (silent/lib/cryptoTools/Crypto/{AES,PRNG}.cpp)
#   _ref/libempref.so  emp-ot's Ferret GGM / SPCOT / LPN headers
#                      (ferret/emp-ot/emp-ot/ferret/{twokeyprp,spcot_sender,
#                      spcot_recver,lpn_f2}.h) over the emp-tool shim in
#                      oracle/emp_shim
set -e
REF=${CUOT_REFERENCE:-/root/reference}
CT=$REF/silent/lib
EMPOT=$REF/ferret/emp-ot
HERE=$(cd "$(dirname "$0")" && pwd)
[ -d "$CT/cryptoTools" ] || { echo "reference tree not found; skipping"; exit 0; }
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++20 -w -fPIC -shared -maes -msse4.1 -mpclmul -I"$CT" \
  "$HERE/ref_driver.cpp" "$CT/cryptoTools/Crypto/AES.cpp" \
  "$CT/cryptoTools/Crypto/PRNG.cpp" "$CT/cryptoTools/Common/block.cpp" \
  -o "$HERE/_ref/libctref.so"
echo "built $HERE/_ref/libctref.so"
# The shim directory comes first so that "emp-tool/emp-tool.h" and
# "emp-ot/emp-ot.h" resolve to it, while "emp-ot/ferret/*.h" resolve to the
# reference tree.
g++ -O2 -std=c++17 -fPIC -shared -maes -msse4.1 -Wall -Wno-unused-parameter \
  -Wno-unused-variable -Wno-ignored-attributes -I"$HERE/emp_shim" -I"$EMPOT" \
  "$HERE/emp_ref.cpp" -o "$HERE/_ref/libempref.so"
echo "built $HERE/_ref/libempref.so"
# The drop-in check: emp-ot's own MpcotReg / OTPre / LpnF2 callers
# (ferret/emp-ot/emp-ot/ferret/{mpcot_reg,preot,lpn_f2}.h and the real
# dev_layer.h) compiled against include/cuot_dev_layer.h and linked to
# libcuot.so; tests/cpp/dl_shim maps dev_layer.h's gpu/ includes onto the
# adapter.  Needs libcuot.so, so it is skipped until the library is built.
ROOT=$(dirname "$HERE")
CUDA=${CUDA_HOME:-/usr/local/cuda}
if [ -f "$ROOT/cuot_b200/libcuot.so" ]; then
  g++ -O2 -std=c++17 -maes -msse4.1 -Wall -Wno-unused-parameter -Wno-unused-variable \
    -Wno-ignored-attributes -Wno-sign-compare -Wno-unused-but-set-variable \
    -I"$HERE/emp_shim" -I"$ROOT/tests/cpp/dl_shim" -I"$ROOT/include" -I"$EMPOT" -I"$CUDA/include" \
    "$ROOT/tests/cpp/test_emp_callers.cpp" "$ROOT/cuot_b200/libcuot.so" \
    -L"$CUDA/lib64" -lcudart -lpthread \
    -Wl,-rpath,'$ORIGIN/../../cuot_b200':"$CUDA/lib64" \
    -o "$HERE/_ref/test_emp_callers"
  echo "built $HERE/_ref/test_emp_callers"
fi
# The reference's own GPU path (gpu/*.cu, silent/quasi_cyclic.cu,
# ferret/emp-ot/emp-ot/ferret/dev_layer.cu) for sm_100a at -O2, with the
# timing / transpose harness oracle/ref_gpu_driver.cu: speed context and the
# transpose pin only.  Only the ref_gpu_* entry points are exported
# (refgpu.map), so its Mat / dev_layer names stay private.
if command -v nvcc >/dev/null 2>&1; then
  OBJ="$HERE/_ref/refgpu_obj"
  mkdir -p "$OBJ"
  NVF="-gencode arch=compute_100a,code=sm_100a -O2 -std=c++20 -w -Xcompiler -fPIC"
  INC="-I$REF/gpu -I$REF/silent -I$EMPOT/emp-ot/ferret"
  pids=""
  for f in "$REF"/gpu/aes_expand.cu "$REF"/gpu/aes_op.cu "$REF"/gpu/gpu_data.cu "$REF"/gpu/gpu_matrix.cu \
           "$REF"/gpu/gpu_ops.cu "$REF"/gpu/gpu_span.cu "$REF"/gpu/gpu_tests.cu "$REF"/gpu/logger.cu \
           "$REF"/silent/quasi_cyclic.cu "$EMPOT"/emp-ot/ferret/dev_layer.cu "$HERE"/ref_gpu_driver.cu; do
    nvcc $NVF $INC -c "$f" -o "$OBJ/$(basename "$f" .cu).o" &
    pids="$pids $!"
  done
  for p in $pids; do wait "$p"; done
  nvcc -shared -gencode arch=compute_100a,code=sm_100a "$OBJ"/*.o -o "$HERE/_ref/librefgpu.so" \
    -lcufft -lcurand -L"${CUDA:-/usr/local/cuda}/lib64/stubs" -lcuda -Xlinker --version-script="$HERE/refgpu.map" -Xlinker -Bsymbolic \
    -Xlinker -rpath="${CUDA:-/usr/local/cuda}/lib64"
  echo "built $HERE/_ref/librefgpu.so"
fi
