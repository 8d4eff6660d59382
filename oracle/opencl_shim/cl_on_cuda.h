/* Test infrastructure only: the OpenCL C names the reference's Vose resampler
 * (src/partfilt/opencl/resampling-valias.cl) uses, mapped onto CUDA so that
 * its device functions compile unchanged as CUDA device code for
 * oracle/ref_valias_harness.cu.  One OpenCL work-group = one CUDA block (1-D).
 * Written for this repository.
 *   __kernel            -> a device function (the harness launches its own kernel)
 *   __global, __local   -> nothing: generic pointers reach global and shared memory
 *                          (the reference's __local arrays are passed in by the harness)
 *   get_*_id / size     -> threadIdx / blockIdx / blockDim / gridDim, dimension 0
 *   barrier(...)        -> __syncthreads()
 *   atomic_inc / dec    -> atomicAdd / atomicSub of 1 (the old value, no wrap)
 *   restrict            -> __restrict__ */
#ifndef ORACLE_CL_ON_CUDA_H
#define ORACLE_CL_ON_CUDA_H
#include <cuda_runtime.h>

#define __kernel static __device__ __forceinline__
#define __global
#define __local
#define restrict __restrict__
#define CLK_LOCAL_MEM_FENCE 0
#define barrier(flags) __syncthreads()

__device__ __forceinline__ unsigned int get_local_id(int) { return threadIdx.x; }
__device__ __forceinline__ unsigned int get_local_size(int) { return blockDim.x; }
__device__ __forceinline__ unsigned int get_group_id(int) { return blockIdx.x; }
__device__ __forceinline__ unsigned int get_num_groups(int) { return gridDim.x; }
__device__ __forceinline__ unsigned int get_global_id(int) { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ unsigned int atomic_inc(unsigned int* p) { return atomicAdd(p, 1u); }
__device__ __forceinline__ unsigned int atomic_dec(unsigned int* p) { return atomicSub(p, 1u); }
#endif
