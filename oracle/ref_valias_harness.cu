// ref_valias_harness.cu -- test infrastructure only: a C-ABI around the
// reference's OWN Vose alias resampler (src/partfilt/opencl/resampling-valias.cl:
// sum_reduce4 :85-104, vose_alias_init :111-195, vose_alias_generate_next
// :198-202), compiled as CUDA device code through the self-written
// oracle/opencl_shim/cl_on_cuda.h and run on a GPU, one block per sub-filter
// of m work-items as the reference's work-group.  Built by
// oracle/build_ref_valias.sh from the reference tree into oracle/_ref/ (its
// build-time copy there only marks the file's top-level functions __device__;
// nothing of the reference is committed).
//
// The wrapper kernel does what the reference's resampling_valias kernel does
// around those functions (:236-290, without the decision uniform and the
// particle copy): scratch <- weight, sum_reduce4, p /= sum (1/m when the sum
// is not positive), prob <- p, vose_alias_init, one draw per work-item from
// the work-item's pair of uniforms.  The work lists are filled with atomic_inc
// / atomic_dec, so the tables' order -- not their distribution -- depends on
// the hardware's ordering of the atomics.
#include <cstdint>

#define TEST_VALIAS 1  // the file then defines its own particle_set for the robot-arm buffers
#include "cl_on_cuda.h"
#include "resampling-valias-device.cl"  // the reference file, top-level functions marked __device__

namespace {

__global__ void k_ref_valias(const float* __restrict__ w, const float* __restrict__ u2, float* scaled, float* prob_out,
                             unsigned* alias_out, unsigned* sel_out)
{
    extern __shared__ unsigned char sm[];
    const unsigned m = blockDim.x, ltid = threadIdx.x, idx = blockIdx.x * m + ltid;
    float* prob = reinterpret_cast<float*>(sm);
    unsigned* alias = reinterpret_cast<unsigned*>(prob + m);
    unsigned* scratch = alias + m;
    __shared__ unsigned tmp[2];
    if (ltid == 0) {
        tmp[0] = 0;
        tmp[1] = m - 1;
    }
    float* scratchf = reinterpret_cast<float*>(scratch);
    float p = w[idx];
    scratchf[ltid] = p;
    __syncthreads();
    const float sum = sum_reduce4(scratchf);
    if (sum > 0.0f) p /= sum;
    else p = 1.0f / (float)m;
    prob[ltid] = p;
    scaled[idx] = p * (float)m;  // what vose_alias_init's first statement makes of it
    __syncthreads();
    vose_alias_init(prob, alias, scratch, &tmp[0], &tmp[1]);
    __syncthreads();
    prob_out[idx] = prob[ltid];
    alias_out[idx] = alias[ltid];
    const float2 r2 = make_float2(u2[2 * idx], u2[2 * idx + 1]);
    sel_out[idx] = vose_alias_generate_next(prob, alias, r2);
}

}  // namespace

// nsub sub-filters of m weights (m a power of two, 32..1024); u2: 2 uniforms
// in [0,1) per particle.  Host arrays.  Returns 0 on success.
extern "C" int ref_valias(const float* w, const float* u2, int m, int nsub, float* scaled, float* prob,
                          unsigned* alias, unsigned* sel)
{
    if (m < 32 || m > 1024 || (m & (m - 1)) || nsub < 1) return 1;
    const size_t n = (size_t)m * nsub;
    float *dw = nullptr, *du = nullptr, *ds = nullptr, *dp = nullptr;
    unsigned *da = nullptr, *dsel = nullptr;
    cudaError_t e = cudaMalloc(&dw, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&du, 2 * n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&ds, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dp, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&da, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dsel, n * 4);
    if (e == cudaSuccess) e = cudaMemcpy(dw, w, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(du, u2, 2 * n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_ref_valias<<<nsub, m, (size_t)m * 12>>>(dw, du, ds, dp, da, dsel);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(scaled, ds, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(prob, dp, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(alias, da, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sel, dsel, n * 4, cudaMemcpyDeviceToHost);
    cudaFree(dw);
    cudaFree(du);
    cudaFree(ds);
    cudaFree(dp);
    cudaFree(da);
    cudaFree(dsel);
    return e == cudaSuccess ? 0 : 2;
}
