#!/bin/sh
# Builds oracle/_ref/libctref.so from the reference's own vendored cryptoTools
# sources, where they lie under the read-only reference tree (nothing is
# copied).  Output goes only to oracle/_ref/.  Needs the reference tree, so it
# runs in the build container only; the GPU box uses the prebuilt file.
set -e
REF=${CUOT_REFERENCE:-/root/reference}
CT=$REF/silent/lib
HERE=$(cd "$(dirname "$0")" && pwd)
[ -d "$CT/cryptoTools" ] || { echo "reference tree not found; skipping"; exit 0; }
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++20 -w -fPIC -shared -maes -msse4.1 -mpclmul -I"$CT" \
  "$HERE/ref_driver.cpp" "$CT/cryptoTools/Crypto/AES.cpp" \
  "$CT/cryptoTools/Crypto/PRNG.cpp" "$CT/cryptoTools/Common/block.cpp" \
  -o "$HERE/_ref/libctref.so"
echo "built $HERE/_ref/libctref.so"
