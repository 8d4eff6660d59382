// pf_host.cuh -- host-side helpers shared by the C-ABI translation units
// (pf_api.cu: single filters and kernel entry points; pf_batch.cu: batched
// filters).  Defined in pf_api.cu.
#pragma once
#include <cstddef>
#include <cstdint>

#include "pf_launch.cuh"

namespace pfhost {

using namespace pfdev;

// Records a printf-style message as this thread's last error and returns s.
pf_status fail(pf_status s, const char* fmt, ...);

#define CU(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return ::pfhost::fail(e_ == cudaErrorMemoryAllocation ? PF_ERR_NOMEM : PF_ERR_CUDA,           \
                                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

pf_status require_gpu(int device);

struct ModelInfo {
    int S, K, C, Z;
    size_t psize;
};
bool model_info(int model, ModelInfo* mi);

// Whether to launch the resampling kernel as a programmatic dependent of the
// sampling kernel: measured to pay when the sampling grid runs in more than
// one wave (its CTAs start in the sampling kernel's last wave: 2^20 unicycle
// particles, 67.0 -> 62.2 us per step) and to cost when it fits in one (2^18
// DH-arm particles, 49.8 -> 58.3 us).
bool dependent_launch_pays(int grid, int M, int E, int S, int device);
const float* init_state_of(int model, const ModelParams& mp);
uint32_t angle_mask_of(int model);
int angle_count_of(int model);

// Launch dispatch over the model template.
struct ModelOps {
    cudaError_t (*sample_sort)(int, int, bool, int, cudaStream_t, const FilterDesc*, const int2*, InputRef);
    cudaError_t (*sample_weight)(int, int, int, cudaStream_t, const FilterDesc*, const int2*, InputRef);
    cudaError_t (*block_sort)(int, int, int, cudaStream_t, const FilterDesc*, const int2*);
    cudaError_t (*exchange_resample)(int, int, int, int, cudaStream_t, const FilterDesc*, const int2*, InputRef,
                                     int32_t*, int);
    cudaError_t (*exchange_inplace)(int, int, cudaStream_t, const FilterDesc*, const int2*);
    cudaError_t (*test_model)(const ModelParams&, const pf_step_input*, int, float*, const float*, float*,
                              cudaStream_t);
    cudaError_t (*step)(int, int, int, int, cudaStream_t, const FilterDesc*, const StepState&, InputRef, int32_t*,
                        bool);
};
ModelOps model_ops(int model);

// MTGP32 stream state for parameter set `set` seeded with `seed` (351 words).
void mtgp_init_state_host(uint32_t* st, int set, uint32_t seed);
// Torus dimensions: dx = 2^floor(log2 sqrt N), dy = N / dx.
void torus_dims(int N, int* dx, int* dy);
// Uniforms a sub-filter's resampler draws per step.
int64_t resample_draws(int res, int M);

}  // namespace pfhost
