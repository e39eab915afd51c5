#!/usr/bin/env bash
# Builds the reference program for the B200 (sm_100a) from its own source
# where it lies ($REF_DIR/collatz_cudav7.cu; REF_DIR defaults to the directory
# "reference" beside this repository), to time the
# reference's own CUDA kernel on the same GPU as the product in cases mode.
# Outputs go only to oracle/_ref/ (git-ignored).  The source is compiled as
# written; the one edit sets MAXBITS (cu:43, a compile-time constant) to each
# N in $NS on a build copy (N = 45 is the source's own value).
# Products: oracle/_ref/ref_gpu_N<N> (stdin 6-tuple, stdout overflow seeds,
# stderr summary, exactly as the reference program).
set -euo pipefail
REF_DIR=${REF_DIR:-$(cd "$(dirname "$0")/../.." && pwd)/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NS=${NS:-"45"}
SRC="$REF_DIR/collatz_cudav7.cu"
[ -r "$SRC" ] || { echo "reference source not found: $SRC" >&2; exit 1; }
mkdir -p "$OUT"
for N in $NS; do
  gen="$OUT/ref_gpu_N$N.cu"
  sed -e "s/^const u32 MAXBITS = 45;/const u32 MAXBITS = $N;/" "$SRC" > "$gen"
  grep -q "^const u32 MAXBITS = $N;" "$gen" || { echo "MAXBITS edit failed" >&2; exit 1; }
  nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -w -o "$OUT/ref_gpu_N$N" "$gen"
done
echo "built: $(ls "$OUT" | grep '^ref_gpu_N[0-9]*$' | tr '\n' ' ')"
