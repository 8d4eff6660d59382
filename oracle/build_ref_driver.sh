#!/bin/sh
# Build the reference's own filter driver loop (particle_filter() of
# src/partfilt/cuda/pf_generic_soa.cu with the robot-arm model header) with
# its CUDA MTGP32 generator and DEBUG_ESTIMATE output, straight from the
# Esthera tree, behind the C-ABI of oracle/ref_driver_harness.cu into
# oracle/_ref/libref_driver.so.  Its main() is renamed, the legacy cutil.h is
# replaced by oracle/cutil_shim/cutil.h, gettimeofday() by the harness's
# fixed-seed stand-in.  Test infrastructure only.  Needs the reference tree
# ($ESTHERA_REF, else ../reference beside the repository); outputs only into
# oracle/_ref/.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${ESTHERA_REF:-$HERE/../../reference}
SRC="$REF/src/partfilt/cuda"
[ -f "$SRC/pf_generic_soa.cu" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
NVCC=${NVCC:-$( [ -x /usr/local/cuda/bin/nvcc ] && echo /usr/local/cuda/bin/nvcc || echo nvcc)}
mkdir -p "$HERE/_ref"
"$NVCC" -O2 -shared -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -w \
    -DMTGP -DDEBUG_ESTIMATE -Dmain=esthera_ref_main -Dgettimeofday=ref_fixed_gettimeofday \
    -I"$SRC" -I"$SRC/mtgp" -I"$REF/src/models/robotarm/cuda" -I"$HERE/cutil_shim" \
    "$HERE/ref_driver_harness.cu" "$SRC/mtgp/mtgp32-fast.c" "$SRC/mtgp/mtgp32dc-param-11213.c" \
    -o "$HERE/_ref/libref_driver.so"
echo "built $HERE/_ref/libref_driver.so"
