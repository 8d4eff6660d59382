#!/bin/sh
# Build the reference's own CUDA sort / resampling / ring-exchange kernels
# (src/partfilt/cuda/pf_generic_soa.cu with bitonic-sort.cu and the robot-arm
# model header, straight from the Esthera tree, cuRAND build, its main()
# renamed) behind the C-ABI of oracle/ref_kernels_harness.cu into
# oracle/_ref/libref_kernels.so.  Test infrastructure only.  Needs the
# reference tree ($ESTHERA_REF, else ../reference beside the repository);
# outputs only into oracle/_ref/.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# the Esthera tree: $ESTHERA_REF, else a checkout named "reference" beside the repository
REF=${ESTHERA_REF:-$HERE/../../reference}
SRC="$REF/src/partfilt/cuda"
[ -f "$SRC/pf_generic_soa.cu" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
NVCC=${NVCC:-$( [ -x /usr/local/cuda/bin/nvcc ] && echo /usr/local/cuda/bin/nvcc || echo nvcc)}
mkdir -p "$HERE/_ref"
"$NVCC" -O2 -shared -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -w \
    -Dmain=esthera_ref_main -I"$SRC" -I"$REF/src/models/robotarm/cuda" \
    "$HERE/ref_kernels_harness.cu" -o "$HERE/_ref/libref_kernels.so" -lcurand
echo "built $HERE/_ref/libref_kernels.so"
