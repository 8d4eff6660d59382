#!/bin/sh
# Build the reference's own pinhole-camera arm model
# (src/models/robotarm/cuda/pf_model_soa_packed_code.cuh, straight from the
# Esthera tree) behind the C-ABI of oracle/ref_camarm_harness.cu into
# oracle/_ref/libref_camarm.so.  Test infrastructure only.  Needs the
# reference tree ($ESTHERA_REF, else ../reference beside the repository);
# outputs only into oracle/_ref/.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# the Esthera tree: $ESTHERA_REF, else a checkout named "reference" beside the repository
REF=${ESTHERA_REF:-$HERE/../../reference}
SRC="$REF/src/models/robotarm/cuda"
[ -f "$SRC/pf_model_soa_packed_code.cuh" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
NVCC=${NVCC:-$( [ -x /usr/local/cuda/bin/nvcc ] && echo /usr/local/cuda/bin/nvcc || echo nvcc)}
mkdir -p "$HERE/_ref"
"$NVCC" -O2 -shared -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -w -I"$SRC" \
    "$HERE/ref_camarm_harness.cu" -o "$HERE/_ref/libref_camarm.so"
echo "built $HERE/_ref/libref_camarm.so"
