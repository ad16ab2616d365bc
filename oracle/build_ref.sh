#!/usr/bin/env bash
# Builds the reference-kernel harness (test infrastructure) into oracle/_ref/:
# the reference's own solvers/smoke/operators.cu and the forward example's
# examples/smoke/forward/simulation.cu, included unmodified from the
# read-only reference checkout, compiled for sm_100a behind the small C ABI
# of oracle/ref_harness.cu.  Nothing is copied out of the reference.
#   oracle/build_ref.sh /path/to/diff-solver      (or REFERENCE=/path/to/diff-solver)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REFERENCE="${1:-${REFERENCE:-}}"
if [ -z "$REFERENCE" ]; then
    echo "no reference checkout given (argument or REFERENCE); skipping the harness build" >&2
    exit 0
fi
SMOKE="$REFERENCE/solvers/smoke"
EXAMPLE="$REFERENCE/examples/smoke/forward"
if [ ! -f "$SMOKE/operators.cu" ]; then
    echo "reference checkout not found at $REFERENCE; skipping the harness build" >&2
    exit 0
fi
mkdir -p "$HERE/_ref"
OUT="$HERE/_ref/libref_smoke.so"
if [ -f "$OUT" ] && [ "$OUT" -nt "$HERE/ref_harness.cu" ] && [ "$OUT" -nt "$SMOKE/operators.cu" ] && [ "$OUT" -nt "$EXAMPLE/simulation.cu" ]; then
    exit 0
fi
/usr/local/cuda/bin/nvcc -std=c++20 -O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -shared \
    -I "$SMOKE" -I "$REFERENCE/solvers" -I "$EXAMPLE" -o "$OUT" "$HERE/ref_harness.cu"
echo "$OUT"
