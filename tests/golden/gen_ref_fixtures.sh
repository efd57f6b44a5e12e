#!/usr/bin/env bash
# Regenerates tests/golden/ref_jacobi2d*.bin + ref_jacobi2d.json by running the
# reference's own jacobi_2d_kernel (oracle/_ref/ref_jacobi_dump, built by
# oracle/ref/Makefile from examples/jacobi-kernel/jacobi_kernel.cu) on a GPU.
# usage: tests/golden/gen_ref_fixtures.sh [outdir]   (default: tests/golden)
set -euo pipefail
ROOT="$(cd "$(dirname "$0")/../.." && pwd)"
OUT="${1:-$ROOT/tests/golden}"
EXE="$ROOT/oracle/_ref/ref_jacobi_dump"
mkdir -p "$OUT"
cases=("16 16 1 1" "37 23 7 2" "128 128 50 3" "130 66 100 4" "64 200 13 5")
json="{\"generator\": \"oracle/_ref/ref_jacobi_dump (reference jacobi_2d_kernel)\", \"cases\": ["
first=1
for c in "${cases[@]}"; do
  read -r nx ny sw seed <<<"$c"
  f="ref_jacobi2d_${nx}x${ny}_s${sw}_seed${seed}.bin"
  "$EXE" "$nx" "$ny" "$sw" "$seed" "$OUT/$f"
  [ $first -eq 1 ] || json+=", "
  first=0
  json+="{\"nx\": $nx, \"ny\": $ny, \"sweeps\": $sw, \"seed\": $seed, \"file\": \"$f\"}"
done
json+="]}"
echo "$json" > "$OUT/ref_jacobi2d.json"

# the reference's 3-D kernel (jacobi_3d_kernel), same generator
EXE3="$ROOT/oracle/_ref/ref_jacobi3d_dump"
cases3=("6 5 4 1 1" "17 9 11 3 2" "33 7 13 5 3")
json="{\"generator\": \"oracle/_ref/ref_jacobi3d_dump (reference jacobi_3d_kernel)\", \"cases\": ["
first=1
for c in "${cases3[@]}"; do
  read -r nx ny nz sw seed <<<"$c"
  f="ref_jacobi3d_${nx}x${ny}x${nz}_s${sw}_seed${seed}.bin"
  "$EXE3" "$nx" "$ny" "$nz" "$sw" "$seed" "$OUT/$f"
  [ $first -eq 1 ] || json+=", "
  first=0
  json+="{\"nx\": $nx, \"ny\": $ny, \"nz\": $nz, \"sweeps\": $sw, \"seed\": $seed, \"file\": \"$f\"}"
done
json+="]}"
echo "$json" > "$OUT/ref_jacobi3d.json"
