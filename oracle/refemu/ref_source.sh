#!/usr/bin/env bash
# TEST INFRASTRUCTURE.  Streams the reference source to stdout with its
# compile-time sizes replaced and main() cut off; nothing is written to disk.
#   usage: ref_source.sh REF_CU X Z L N NT fixed|verbatim
# "fixed" turns the receiver test's assignment into a comparison
# (P-S-seperating.cu:307), making the recorded value the post-update one.
# For N != 6 the six-term coefficient initialisers are replaced by the
# float32 weights of oracle/coeffs.py padded with zero weights, because the
# kernels' stencils are unrolled to six terms.
set -euo pipefail
ref=$1; X=$2; Z=$3; L=$4; N=$5; NT=$6; mode=$7
here=$(cd "$(dirname "$0")" && pwd)
args=(-e "s/^#define L 200\$/#define L $L/"
      -e "s/^#define N 6\$/#define N $N/"
      -e "s/^#define NT 6000\$/#define NT $NT/"
      -e "s/^#define Xn 600\$/#define Xn $X/"
      -e "s/^#define Zn 600\$/#define Zn $Z/")
if [ "$mode" = fixed ]; then
  args+=(-e 's/if (j = Z_receive)/if (j == Z_receive)/')
fi
if [ "$N" != 6 ]; then
  coef=$(python3 "$here/../coeffs.py" "$N")
  args+=(-e "s/float a\[N\] = {[^}]*};/float a[6] = { $coef };/")
fi
sed "${args[@]}" "$ref" | sed -n '/^int main()/q;p'
