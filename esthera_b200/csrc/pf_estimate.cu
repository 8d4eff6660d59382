// pf_estimate.cu -- posterior estimate of a set of particles as a kernel-level
// entry point: per-sub-filter FP64 partials (one CTA each) into a scratch
// array in global memory, then one CTA combining them with log-sum-exp
// rescaling.  The same arithmetic as the filter's own estimate: weights
// exp(key - max) in FP32, sums in FP64, circular means for angular variables,
// the reference's winner (first maximum key, thrust::max_element semantics,
// src/partfilt/cuda/pf_generic_soa.cu:1014-1017).
#include <cstring>
#include <mutex>
#include <string>

#include <cuda.h>

#include "pf_launch.cuh"

namespace pfdev {

constexpr int kEstMaxState = 16;
constexpr int kEstStride = 3 + 2 * kEstMaxState;  // doubles per sub-filter: lmax, W, sums[S], cos[S], best

// Partials of sub-filter blockIdx.x: [0] key max (0 in linear mode), [1] sum w,
// [2+v] sum w x_v (angles: sum w sin x_v), [2+S+v] sum w cos x_v, [2+2S] index of
// the first maximal key within the sub-filter.
__global__ void __launch_bounds__(256) k_est_partials(const float* __restrict__ keys, const float* __restrict__ state,
                                                      int S, int64_t T, int m, uint32_t angle_mask, int log_weights,
                                                      double* __restrict__ part)
{
    __shared__ double red[8][kEstStride];
    __shared__ float rk[8];
    __shared__ int ri[8];
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int64_t base = (int64_t)b * m;
    float bk = -INFINITY;
    int bi = 0x7fffffff;
    for (int i = tid; i < m; i += 256) {
        const float k = keys[base + i];
        if (k > bk || (k == bk && i < bi)) {
            bk = k;
            bi = i;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float ok = __shfl_xor_sync(kFull, bk, o);
        const int oi = __shfl_xor_sync(kFull, bi, o);
        if (ok > bk || (ok == bk && oi < bi)) {
            bk = ok;
            bi = oi;
        }
    }
    if (lane == 0) {
        rk[wp] = bk;
        ri[wp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < 8; ++w)
            if (rk[w] > rk[0] || (rk[w] == rk[0] && ri[w] < ri[0])) {
                rk[0] = rk[w];
                ri[0] = ri[w];
            }
    }
    __syncthreads();
    const float lmax = log_weights ? rk[0] : 0.0f;
    double acc[kEstStride - 1];
#pragma unroll
    for (int j = 0; j < kEstStride - 1; ++j) acc[j] = 0.0;
    for (int i = tid; i < m; i += 256) {
        const float k = keys[base + i];
        const double w = log_weights ? (double)__expf(k - lmax) : (double)k;
        acc[0] += w;
#pragma unroll
        for (int v = 0; v < kEstMaxState; ++v) {
            if (v < S) {
                const float x = state[(int64_t)v * T + base + i];
                if ((angle_mask >> v) & 1u) {
                    float sn, cs;
                    __sincosf(x, &sn, &cs);
                    acc[1 + v] += w * (double)sn;
                    acc[1 + kEstMaxState + v] += w * (double)cs;
                } else {
                    acc[1 + v] += w * (double)x;
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kEstStride - 1; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(kFull, acc[j], o);
        if (lane == 0) red[wp][j] = acc[j];
    }
    __syncthreads();
    double* out = part + (int64_t)b * kEstStride;
    for (int j = tid; j < kEstStride - 1; j += 256) {
        double s = red[0][j];
        for (int w = 1; w < 8; ++w) s += red[w][j];
        // [0] lmax, [1] W, [2..] sums (compacted: sin/linear at 2+v, cos at 2+S+v)
        if (j == 0) out[1] = s;
        else if (j <= kEstMaxState) {
            if (j - 1 < S) out[2 + (j - 1)] = s;
        } else if (j - 1 - kEstMaxState < S) {
            out[2 + S + (j - 1 - kEstMaxState)] = s;
        }
    }
    if (tid == 0) {
        out[0] = (double)lmax;
        out[2 + 2 * S] = (double)ri[0];
    }
}

// Combine nsub partials into one pf_estimate (one CTA of 256 threads).
__global__ void __launch_bounds__(256) k_est_final(const double* __restrict__ part, const float* __restrict__ keys,
                                                   const float* __restrict__ state, int S, int64_t T, int m,
                                                   int nsub, uint32_t angle_mask, int log_weights,
                                                   pf_estimate* __restrict__ out)
{
    __shared__ double red[8][kEstStride];
    __shared__ float rk[8];
    __shared__ int64_t rg[8];
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    double gmax = -INFINITY;
    float bk = -INFINITY;
    int64_t bg = INT64_MAX;
    for (int b = tid; b < nsub; b += 256) {
        const double* p = part + (int64_t)b * kEstStride;
        gmax = fmax(gmax, p[0]);
        const int64_t g = (int64_t)b * m + (int64_t)p[2 + 2 * S];
        const float k = keys[g];
        if (k > bk || (k == bk && g < bg)) {
            bk = k;
            bg = g;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        gmax = fmax(gmax, __shfl_xor_sync(kFull, gmax, o));
        const float ok = __shfl_xor_sync(kFull, bk, o);
        const int64_t og = __shfl_xor_sync(kFull, bg, o);
        if (ok > bk || (ok == bk && og < bg)) {
            bk = ok;
            bg = og;
        }
    }
    if (lane == 0) {
        red[wp][0] = gmax;
        rk[wp] = bk;
        rg[wp] = bg;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < 8; ++w) {
            red[0][0] = fmax(red[0][0], red[w][0]);
            if (rk[w] > rk[0] || (rk[w] == rk[0] && rg[w] < rg[0])) {
                rk[0] = rk[w];
                rg[0] = rg[w];
            }
        }
    }
    __syncthreads();
    const double gm = log_weights ? red[0][0] : 0.0;
    const int64_t best = (rg[0] >= 0 && rg[0] < T) ? rg[0] : 0;
    __syncthreads();
    const int nv = 1 + 2 * S;
    double acc[1 + 2 * kEstMaxState];
#pragma unroll
    for (int j = 0; j < 1 + 2 * kEstMaxState; ++j) acc[j] = 0.0;
    for (int b = tid; b < nsub; b += 256) {
        const double* p = part + (int64_t)b * kEstStride;
        const double sc = log_weights ? exp(p[0] - gm) : 1.0;
#pragma unroll
        for (int j = 0; j < 1 + 2 * kEstMaxState; ++j)
            if (j < nv) acc[j] += sc * p[1 + j];
    }
#pragma unroll
    for (int j = 0; j < 1 + 2 * kEstMaxState; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(kFull, acc[j], o);
        if (lane == 0) red[wp][j] = acc[j];
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < 8; ++w)
            for (int j = 0; j < nv; ++j) red[0][j] += red[w][j];
        const double W = red[0][0];
        pf_estimate e;
        memset(&e, 0, sizeof(e));
        for (int v = 0; v < S; ++v)
            e.mean[v] = ((angle_mask >> v) & 1u) ? atan2(red[0][1 + v], red[0][1 + S + v]) : red[0][1 + v] / W;
        e.log_norm = gm + log(W);
        for (int v = 0; v < S; ++v) e.best[v] = state[(int64_t)v * T + best];
        e.best_key = keys[best];
        e.best_subfilter = (int32_t)(best / m);
        e.step = 0;
        e.flags = (isfinite(gm) && isfinite(W) && W > 0.0) ? 0 : 1;
        *out = e;
    }
}

// Validates the shape and launches partials + final on `st` with the given scratch.
static cudaError_t launch_estimate(const float* keys, const float* state, int S, int64_t T, int m,
                                   uint32_t angle_mask, int log_weights, double* scratch, pf_estimate* out,
                                   cudaStream_t st)
{
    const int nsub = (int)(T / m);
    k_est_partials<<<nsub, 256, 0, st>>>(keys, state, S, T, m, angle_mask, log_weights, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_est_final<<<1, 256, 0, st>>>(scratch, keys, state, S, T, m, nsub, angle_mask, log_weights, out);
    return cudaGetLastError();
}

static bool estimate_shape_ok(int S, int64_t T, int m, std::string* why)
{
    if (S < 1 || S > kEstMaxState) {
        *why = "num_state must be in [1, 16]";
        return false;
    }
    if (m < 1 || T < m || T % m != 0) {
        *why = "num_particles must be a positive multiple of m";
        return false;
    }
    if (T / m > INT32_MAX) {
        *why = "too many sub-filters";
        return false;
    }
    return true;
}

}  // namespace pfdev

using namespace pfdev;

// Error recording shared with pf_api.cu (thread-local message for pf_last_error).
pf_status pfi_fail(pf_status s, const char* msg);

extern "C" pf_status pfk_estimate(const float* keys, const float* state, int32_t num_state, int64_t num_particles,
                                  int32_t m, uint32_t angle_mask, int32_t log_weights, pf_estimate* out)
{
    std::string why;
    if (!keys || !state || !out) return pfi_fail(PF_ERR_INVALID, "null argument");
    if (!estimate_shape_ok(num_state, num_particles, m, &why)) return pfi_fail(PF_ERR_INVALID, why.c_str());
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
        cudaGetLastError();
        return pfi_fail(PF_ERR_CUDA, "no CUDA device available (this engine has no CPU path)");
    }
    const int64_t T = num_particles;
    const int nsub = (int)(T / m);
    float *dk = nullptr, *ds = nullptr;
    double* dp = nullptr;
    pf_estimate* de = nullptr;
    cudaError_t e = cudaMalloc(&dk, (size_t)T * 4);
    if (e == cudaSuccess) e = cudaMalloc(&ds, (size_t)T * num_state * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dp, (size_t)nsub * kEstStride * 8);
    if (e == cudaSuccess) e = cudaMalloc(&de, sizeof(pf_estimate));
    if (e == cudaSuccess) e = cudaMemcpy(dk, keys, (size_t)T * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ds, state, (size_t)T * num_state * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_estimate(dk, ds, num_state, T, m, angle_mask, log_weights, dp, de, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, de, sizeof(pf_estimate), cudaMemcpyDeviceToHost);
    cudaFree(dk);
    cudaFree(ds);
    cudaFree(dp);
    cudaFree(de);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return pfi_fail(PF_ERR_CUDA, cudaGetErrorString(e));
    }
    return PF_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers cannot call cudaMalloc: code running
// inside a memory pool or arena that owns every device allocation, embedded
// hosts whose allocator is locked after start-up, and work that must not
// allocate between stream captures.  pfk_estimate_noalloc computes exactly
// what pfk_estimate computes, from device pointers the caller already owns,
// with its per-sub-filter scratch in the static array below (allocated with
// the module, held by every GPU that loads the library until exit).
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxSubfilters = 4096;  // 4096 * 35 doubles = 1.15 MB per device
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxSubfilters * kEstStride];

static std::mutex g_noalloc_mu;
// Device address of g_noalloc_scratch per device ordinal, valid for the CUDA
// context whose process-unique id is stored beside it: cudaDeviceReset (or a
// caller switching to another context on the same ordinal) loads the module
// afresh, possibly at another address, and the new context has a new id, so
// the next call looks the address up again instead of using a stale one.
static double* g_noalloc_ptr[256];
static unsigned long long g_noalloc_ctx[256];

// The current context's process-unique id (cuCtxGetId; ids are never reused
// within a process), through the runtime's driver entry points so the library
// needs no link against libcuda.  0 when no context is current.
static unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b) {
            cudaGetLastError();
            return 0;
        }
        get_current = reinterpret_cast<GetCurrent>(a);
        get_id = reinterpret_cast<GetId>(b);
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

extern "C" pf_status pfk_estimate_noalloc(const float* d_keys, const float* d_state, int32_t num_state,
                                          int64_t num_particles, int32_t m, uint32_t angle_mask,
                                          int32_t log_weights, pf_estimate* d_out, void* stream)
{
    std::string why;
    if (!d_keys || !d_state || !d_out) return pfi_fail(PF_ERR_INVALID, "null argument");
    if (!estimate_shape_ok(num_state, num_particles, m, &why)) return pfi_fail(PF_ERR_INVALID, why.c_str());
    if (num_particles / m > kNoAllocMaxSubfilters)
        return pfi_fail(PF_ERR_INVALID, "pfk_estimate_noalloc: more than 4096 sub-filters (num_particles / m) "
                                        "exceed its static scratch; use pfk_estimate");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256) {
        cudaGetLastError();
        return pfi_fail(PF_ERR_CUDA, "no current CUDA device");
    }
    double* scratch = nullptr;
    {
        // Once per device (and again after the device's context was replaced),
        // with that device current: the host-side name of the array is only a
        // stand-in, so ask the runtime for its device address.
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        unsigned long long ctx = current_context_id();
        if (!g_noalloc_ptr[dev] || !ctx || ctx != g_noalloc_ctx[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return pfi_fail(PF_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed");
            }
            g_noalloc_ptr[dev] = static_cast<double*>(p);
            g_noalloc_ctx[dev] = current_context_id();  // the lookup made the context current if none was
        }
        scratch = g_noalloc_ptr[dev];
    }
    e = launch_estimate(d_keys, d_state, num_state, num_particles, m, angle_mask, log_weights, scratch, d_out,
                        static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return pfi_fail(PF_ERR_CUDA, cudaGetErrorString(e));
    }
    return PF_OK;
}
