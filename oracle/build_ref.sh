#!/usr/bin/env bash
# build_ref.sh -- TEST INFRASTRUCTURE ONLY.
#
# Builds the reference's own CPU code paths from the sources where they lie
# (read-only reference tree) into oracle/_ref/ (git-ignored; the binaries
# travel with the working tree so the CPU baseline can run them elsewhere).
# No reference source is copied into the repository: the CPU-emulation builds
# rewrite kernel launches into a temporary directory outside the repo, the
# same rewrite the reference Makefile's emul-% rule performs (Makefile:98-141).
#
#   oracle/_ref/sieve_ref             sieve_ref.cpp (CPU Zech-log sieve)
#   oracle/_ref/cantor_ref            cantor_ref.cpp (CPU additive-FFT suite)
#   oracle/_ref/libref_cantor.so      gf2x_fft_mul & friends behind a C ABI
#   oracle/_ref/trinomial_stage2_emul trinomial_stage2.cu kernels run on CPU
#   oracle/_ref/trinomial_scan_emul   trinomial_scan.cu (naive gcd) on CPU
#   oracle/_ref/cert2bin, bin2cert,   certificate <-> found.bin converters and
#   oracle/_ref/check_ref             the sieve-vs-reference cross-check
#
# Flags: the reference uses -O2 -march=native; we use -O2 with PCLMUL/SSE4
# enabled but no host-specific ISA so the binaries also run on the GPU
# hosts' CPUs.
set -euo pipefail
# GF2E_REFERENCE_SRC names the reference's src/ directory; without it (or
# with a directory that does not exist) nothing is built.
REF="${GF2E_REFERENCE_SRC:-}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ -z "$REF" ]; then
    echo "build_ref: set GF2E_REFERENCE_SRC to the reference's src/ directory; skipping" >&2
    exit 0
fi
if [ ! -d "$REF" ]; then
    echo "build_ref: reference sources not present ($REF); skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
CXX="${CXX:-g++}"
FLAGS="-O2 -mpclmul -msse4.1 -w"

"$CXX" $FLAGS -I"$REF" -o "$OUT/sieve_ref" "$REF/sieve_ref.cpp"
"$CXX" $FLAGS -I"$REF" -o "$OUT/cantor_ref" "$REF/cantor_ref.cpp"
"$CXX" $FLAGS -fPIC -shared -I"$REF" -o "$OUT/libref_cantor.so" "$HERE/ref_cantor_driver.cpp"
"${CC:-gcc}" -O2 -w -o "$OUT/cert2bin" "$REF/cert2bin.c"
"${CC:-gcc}" -O2 -w -o "$OUT/bin2cert" "$REF/bin2cert.c"
"$CXX" $FLAGS -o "$OUT/check_ref" "$REF/check_ref.cpp"

TMP="$(mktemp -d /tmp/gf2e_refemul.XXXXXX)"
trap 'rm -rf "$TMP"' EXIT
SEDLAUNCH='s/([A-Za-z_][A-Za-z0-9_]*)<<<([^>]*)>>>/EMUL_LAUNCH(\1, \2)/g; s/__device__ __forceinline__/static inline/'
for h in gf2_small_field.h gf2_field_setup.h gf2_cantor_core.h gf2_cantor_engine.h cuda_emul.h gf2_gcd.h; do
    cp "$REF/$h" "$TMP/"
done
sed -E "$SEDLAUNCH" "$REF/gf2_cantor_cuda.h" > "$TMP/gf2_cantor_cuda.h"
sed -E "$SEDLAUNCH" "$REF/gf2_trinomial_cuda.h" > "$TMP/gf2_trinomial_cuda.h"
printf '#pragma once\n#include "cuda_emul.h"\n' > "$TMP/cuda_runtime.h"
for prog in trinomial_stage2 trinomial_scan; do
    sed -E "$SEDLAUNCH" "$REF/$prog.cu" > "$TMP/$prog.cpp"
    "$CXX" $FLAGS -x c++ -I"$TMP" -pthread -o "$OUT/${prog}_emul" "$TMP/$prog.cpp"
done
echo "build_ref: built $(ls "$OUT" | tr '\n' ' ')" >&2
