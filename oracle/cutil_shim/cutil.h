/* Test infrastructure only: the one macro of the legacy CUDA SDK header
 * cutil.h that the reference's unicycle program uses (CUDA_SAFE_CALL), so that
 * its kernels compile for oracle/ref_unicycle_harness.cu.  Written for this
 * repository; it is not the SDK header. */
#ifndef ORACLE_CUTIL_SHIM_H
#define ORACLE_CUTIL_SHIM_H
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>
#define CUDA_SAFE_CALL(call)                                                                       \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            fprintf(stderr, "%s:%d: %s\n", __FILE__, __LINE__, cudaGetErrorString(e_));           \
            exit(1);                                                                               \
        }                                                                                          \
    } while (0)
#endif
