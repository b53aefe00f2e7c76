#!/usr/bin/env bash
# Builds the hilbertJoin reference from its own sources (read in place under
# REF_DIR, default: the directory `reference` beside this repository) into
# oracle/_ref/, for use as a parity oracle and as the CPU baseline. Nothing
# from the reference is copied into this repository; only the binaries land in
# oracle/_ref/ (git-ignored).
#
# The reference needs MKL (only for its default data generator) and Boost
# lockfree (only for its dead pair-queue path); oracle/shim/ stands in for both.
# Flags follow the reference's CMakeLists.txt:24 (-march=skylake-avx512, so the
# binary runs on any AVX-512 host, not only the one it was built on) with the
# count-only define both of its targets use (CMakeLists.txt:56-57). KBLOCK and
# NUM_THREADS are compile-time in the reference (hilbertjoin/egojoin.h:21-27),
# so one binary per (KBLOCK, NUM_THREADS) pair is built.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_DIR="${REF_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF_DIR/hilbertjoin/egojoin.cpp" ]; then
    echo "reference sources not found under $REF_DIR; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
KBLOCKS="${KBLOCKS:-4 16}"
THREADS="${THREADS:-8 16 32 64 128 256}"
SRCS="hilbertjoin/egojoin.cpp hilbertjoin/hilloop.cpp util/dataIo.cpp util/allocation.cpp util/chrisutil.cpp measure/timer.cpp"
CXXFLAGS="-std=c++11 -march=skylake-avx512 -ffast-math -fassociative-math -O3 -fopenmp -DCOUNT_ONLY -w"
for kb in $KBLOCKS; do
  for nt in $THREADS; do
    exe="$OUT/hj_ref_k${kb}_t${nt}"
    if [ -x "$exe" ] && [ "$exe" -nt "$HERE/ref_driver.cpp" ] && [ "$exe" -nt "$0" ]; then continue; fi
    objdir="$OUT/obj_k${kb}_t${nt}"
    mkdir -p "$objdir"
    objs=""
    for s in $SRCS; do
      o="$objdir/$(echo "$s" | tr '/' '_').o"
      g++ $CXXFLAGS -DKBLOCK=$kb -DNUM_THREADS=$nt -I"$HERE/shim" -I"$REF_DIR" -c "$REF_DIR/$s" -o "$o" &
      objs="$objs $o"
    done
    g++ $CXXFLAGS -DKBLOCK=$kb -DNUM_THREADS=$nt -c "$HERE/ref_driver.cpp" -o "$objdir/driver.o" &
    wait
    g++ $CXXFLAGS -o "$exe" $objs "$objdir/driver.o"
  done
done
echo "reference binaries in $OUT"
