#!/bin/sh
# Build the reference's own Vose alias resampler
# (src/partfilt/opencl/resampling-valias.cl, straight from the Esthera tree,
# compiled as CUDA device code through the self-written OpenCL-name shim
# oracle/opencl_shim/cl_on_cuda.h) behind the C-ABI of
# oracle/ref_valias_harness.cu into oracle/_ref/libref_valias.so.  Test
# infrastructure only.  Needs the reference tree ($ESTHERA_REF, else
# ../reference beside the repository); outputs only into oracle/_ref/.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${ESTHERA_REF:-$HERE/../../reference}
SRC="$REF/src/partfilt/opencl"
[ -f "$SRC/resampling-valias.cl" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
NVCC=${NVCC:-$( [ -x /usr/local/cuda/bin/nvcc ] && echo /usr/local/cuda/bin/nvcc || echo nvcc)}
mkdir -p "$HERE/_ref"
# OpenCL C functions carry no execution-space qualifier, which CUDA reads as
# host code: a build-time copy (an output in _ref/, never committed) marks the
# file's top-level function definitions __device__; every other OpenCL name is
# mapped by the shim header.
sed -E 's/^(float|void|unsigned int|inline void) ([A-Za-z_0-9]+\()/__device__ \1 \2/' \
    "$SRC/resampling-valias.cl" > "$HERE/_ref/resampling-valias-device.cl"
"$NVCC" -O2 -shared -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -w -x cu \
    -I"$HERE/_ref" -I"$HERE/opencl_shim" "$HERE/ref_valias_harness.cu" -o "$HERE/_ref/libref_valias.so"
echo "built $HERE/_ref/libref_valias.so"
