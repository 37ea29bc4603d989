#!/usr/bin/env bash
# Builds the reference solver (pawelswoboda/RAMA) from its sources, where they
# lie, together with oracle/ref_harness.cu into oracle/_ref/librama_ref.so.
# Test infrastructure: the result is the parity oracle on the GPU and the
# reference arm of bench.py.  Nothing from the reference is copied into this
# repository.
#
#   oracle/build_ref.sh <reference tree>     (or RAMA_REFERENCE_DIR=<tree>)
#
# Without a reference tree the prebuilt oracle/_ref is kept.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${RAMA_REFERENCE_DIR:-}}"
if [ -z "$REF" ]; then
  echo "usage: $0 <reference tree> (or set RAMA_REFERENCE_DIR); keeping the prebuilt oracle/_ref" >&2
  exit 0
fi
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -d "$REF/src" ]; then
  echo "reference sources not found at $REF; keeping the prebuilt oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OBJ"
NVCC="${NVCC:-nvcc}"
FLAGS=(-gencode arch=compute_100a,code=sm_100a -std=c++17 -O3 -use_fast_math -DNDEBUG
       -Xcompiler -fPIC --expt-relaxed-constexpr -w
       -I"$HERE/ref_shim" -I"$REF/include" -I"$REF/external/ECL-CC" -I"$REF/external/cudaMST/gpuMST" -I"$REF/external/cudaMST/common")
SRCS=("$REF/src/dCOO.cu" "$REF/src/conflicted_cycles_cuda.cu" "$REF/src/multicut_message_passing.cu"
      "$REF/src/dual_solver.cu" "$REF/src/maximum_matching_vertex_based.cu"
      "$REF/src/edge_contractions_woc_thrust.cu" "$REF/src/edge_contractions_woc.cu"
      "$REF/src/rama_cuda.cu" "$REF/external/ECL-CC/ECL-CC_11.cu" "$REF/external/cudaMST/gpuMST/gpuMST.cu"
      "$HERE/ref_harness.cu")
pids=()
objs=()
for s in "${SRCS[@]}"; do
  o="$OBJ/$(basename "${s%.*}").o"
  objs+=("$o")
  if [ ! -f "$o" ] || [ "$s" -nt "$o" ]; then
    "$NVCC" "${FLAGS[@]}" -c "$s" -o "$o" &
    pids+=($!)
  fi
done
for p in "${pids[@]}"; do wait "$p"; done
g++ -std=c++17 -O2 -fPIC -c "$REF/src/multicut_text_parser.cpp" -o "$OBJ/multicut_text_parser.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/librama_ref.so" "${objs[@]}" "$OBJ/multicut_text_parser.o"
echo "built $OUT/librama_ref.so"
