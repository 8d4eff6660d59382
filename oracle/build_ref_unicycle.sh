#!/bin/sh
# Build the reference unicycle program's own propagate + weight kernel
# (src/models/unicycle/particle_filter.cu, straight from the Esthera tree,
# cuRAND build, its main() renamed, the legacy cutil.h replaced by
# oracle/cutil_shim/cutil.h) behind the C-ABI of
# oracle/ref_unicycle_harness.cu into oracle/_ref/libref_unicycle.so.  Test
# infrastructure only.  Needs the reference tree ($ESTHERA_REF, else
# ../reference beside the repository); outputs only into oracle/_ref/.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# the Esthera tree: $ESTHERA_REF, else a checkout named "reference" beside the repository
REF=${ESTHERA_REF:-$HERE/../../reference}
SRC="$REF/src/models/unicycle"
[ -f "$SRC/particle_filter.cu" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
NVCC=${NVCC:-$( [ -x /usr/local/cuda/bin/nvcc ] && echo /usr/local/cuda/bin/nvcc || echo nvcc)}
mkdir -p "$HERE/_ref"
"$NVCC" -O2 -shared -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -w \
    -Dmain=esthera_ref_unicycle_main -I"$SRC" -I"$HERE/cutil_shim" \
    "$HERE/ref_unicycle_harness.cu" -o "$HERE/_ref/libref_unicycle.so" -lcurand
echo "built $HERE/_ref/libref_unicycle.so"
