/* Test infrastructure only: the few macros and functions of the legacy CUDA
 * SDK header cutil.h that the reference's unicycle program and its CUDA
 * MTGP32 sources use (CUDA_SAFE_CALL; CUT_SAFE_CALL and the cutTimer calls of
 * the MTGP32 sources' own benchmark routines, stubbed: nothing here times
 * anything), so that they compile for the harnesses in oracle/.  Written for
 * this repository; it is not the SDK header. */
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
#define CUT_SAFE_CALL(call) ((void)(call))
static inline int cutCreateTimer(unsigned int* t) { *t = 0u; return 1; }
static inline int cutStartTimer(unsigned int) { return 1; }
static inline int cutStopTimer(unsigned int) { return 1; }
static inline float cutGetTimerValue(unsigned int) { return 0.0f; }
static inline int cutDeleteTimer(unsigned int) { return 1; }
#endif
