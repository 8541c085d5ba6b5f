#!/usr/bin/env bash
# Build oracle/_ref/ref_harness and oracle/_ref/tuple_text_to_bin from the
# reference's own sources, where they lie: the reference directory is the
# first argument (or $REF).  Outputs go to oracle/_ref/ only.  The
# reference's GPU code targets sm_35 and does not compile for sm_100a; the
# headers are compiled here for sm_52 only so that their host functions can
# run on the CPU -- no kernel of theirs is ever launched.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${REF:-}}"
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh <reference-dir> (or REF=<dir>)" >&2
  exit 2
fi
OUT="$HERE/_ref"
if [ ! -f "$REF/graph.h" ]; then
  echo "reference sources not present; keeping any prebuilt $OUT"
  exit 0
fi
mkdir -p "$OUT"
# the reference's edge-list converter, one standalone C++ file
CONV="$REF/tuple_text_to_binary_csr/tuple_text_to_bin.cpp"
if [ -f "$CONV" ] && ! [ "$OUT/tuple_text_to_bin" -nt "$CONV" ]; then
  g++ -O2 -w "$CONV" -o "$OUT/tuple_text_to_bin"
  echo "built $OUT/tuple_text_to_bin"
fi
if [ -x "$OUT/ref_harness" ] && [ "$OUT/ref_harness" -nt "$HERE/ref_harness.cu" ]; then
  echo "up to date"
  exit 0
fi
nvcc -arch=sm_52 -O2 -w -Wno-deprecated-gpu-targets -I"$REF" -Xcompiler -fopenmp \
  "$HERE/ref_harness.cu" -o "$OUT/ref_harness"
echo "built $OUT/ref_harness"
