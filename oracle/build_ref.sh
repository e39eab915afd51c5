#!/usr/bin/env bash
# Builds the reference program for the CPU, from its own source where it lies
# ($REF_DIR/collatz_cudav7.cu; REF_DIR defaults to the directory "reference"
# beside this repository), through the fake CUDA runtime
# header in oracle/ref_shim/.  Outputs go only to oracle/_ref/ (git-ignored).
#
# The source is compiled as written except for three mechanical edits that
# sed applies to a build copy under oracle/_ref/:
#   * MAXBITS (cu:43) is set to each N in $NS (it is a compile-time constant);
#   * the launch `compute_kernel<<<blocks, threads_per_block>>>(` (cu:598)
#     becomes SHIM_LAUNCH(...), a sequential loop over blocks and threads;
#   * shim_count_seeds(alength) is inserted before cu:237 to report the
#     number of seeds checked (printed to stderr at exit as "shim seeds = S").
# Products per N: ref_N<N> (the reference program: stdin 6-tuple, stdout
# overflow seeds, stderr summary) and ref_tool_N<N> (oracle/ref_shim/ref_tool.cpp).
set -euo pipefail
REF_DIR=${REF_DIR:-$(cd "$(dirname "$0")/../.." && pwd)/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NS=${NS:-"26 30 36 40 42 45"}
SRC="$REF_DIR/collatz_cudav7.cu"
[ -r "$SRC" ] || { echo "reference source not found: $SRC" >&2; exit 1; }
mkdir -p "$OUT"
for N in $NS; do
  gen="$OUT/ref_N$N.cpp"
  sed -e "s/^const u32 MAXBITS = 45;/const u32 MAXBITS = $N;/" \
      -e 's/compute_kernel<<<blocks, threads_per_block>>>(/SHIM_LAUNCH(blocks, threads_per_block, compute_kernel, /' \
      -e 's/^    if (alength == 0) { return; }/    shim_count_seeds(alength);\n&/' \
      "$SRC" > "$gen"
  grep -q "^const u32 MAXBITS = $N;" "$gen" || { echo "MAXBITS edit failed" >&2; exit 1; }
  grep -q "SHIM_LAUNCH(blocks" "$gen" || { echo "launch edit failed" >&2; exit 1; }
  grep -q "shim_count_seeds(alength)" "$gen" || { echo "counter edit failed" >&2; exit 1; }
  g++ -std=c++17 -O2 -w -I"$HERE/ref_shim" -x c++ "$gen" -o "$OUT/ref_N$N"
  g++ -std=c++17 -O2 -w -I"$HERE/ref_shim" -I"$OUT" -DREF_SOURCE="\"ref_N$N.cpp\"" \
      "$HERE/ref_shim/ref_tool.cpp" -o "$OUT/ref_tool_N$N"
done
echo "built: $(ls "$OUT" | grep -v '\.cpp$' | tr '\n' ' ')"
