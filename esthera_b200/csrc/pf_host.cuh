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

// Particles per thread when a configuration leaves it at 0 (the same for
// single filters, batches and the server: the same configuration gives the
// same bits everywhere): 1 for m = 32, 2 for m = 64, else 4 for states of up
// to 3 variables and 2 for larger states (S is the model's state size).
int default_ppt(int M, int S);

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
    cudaError_t (*sample_sort)(int, int, int, bool, int, cudaStream_t, const FilterDesc*, const int2*, InputRef);
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

// The model registry: every model the library can run, built-in or added with
// PF_MODEL (esthera_b200_model.cuh), registered once at load time.
struct ModelEntry {
    int id;
    const char* name;
    ModelInfo info;
    ModelOps ops;
    uint32_t angle_mask;  // bit v: state variable v is an angle (circular means)
    int angle_count;
    size_t init_offset;   // offset of init_state[] in the parameter struct
};
// false (and nothing registered) when the id is taken, negative or the table is full.
bool register_model(const ModelEntry& e);
const ModelEntry* find_model(int id);
int registered_models(int* ids, int cap);

template <class Mdl>
ModelOps ops_of()
{
    return {Launch<Mdl>::sample_sort,       Launch<Mdl>::sample_weight,    Launch<Mdl>::block_sort,
            Launch<Mdl>::exchange_resample, Launch<Mdl>::exchange_inplace, Launch<Mdl>::test_model,
            Launch<Mdl>::step};
}

template <class Mdl, class Params>
ModelEntry model_entry(int id, const char* name, size_t init_offset)
{
    static_assert(sizeof(Params) <= sizeof(ModelParams), "model parameters larger than ModelParams::raw");
    static_assert(Mdl::S >= 1 && Mdl::S <= PF_MAX_STATE && Mdl::K >= 1 && Mdl::NA >= 0 && Mdl::NA <= Mdl::S,
                  "model sizes out of range");
    static_assert(Mdl::C <= PF_MAX_CONTROL && Mdl::Z <= PF_MAX_MEAS, "control / measurement larger than pf_step_input");
    static_assert(2 + Mdl::S + Mdl::NA + 2 <= pfdev::kPartStride,
                  "a sub-filter's estimate row (key max, weight sum, S state sums, NA cosine sums, winner key and "
                  "index) must fit kPartStride doubles: S + NA <= 28");
    uint32_t mask = 0;
    for (int a = 0; a < Mdl::NA; ++a) mask |= 1u << Mdl::angle_var(a);
    return {id, name, {Mdl::S, Mdl::K, Mdl::C, Mdl::Z, sizeof(Params)}, ops_of<Mdl>(), mask, Mdl::NA, init_offset};
}

}  // namespace pfhost

// Registers model struct MDL (with parameter struct PARAMS, which has a
// float init_state[MDL::S] member) under id ID, from one translation unit;
// the kernels themselves are instantiated where Launch<MDL>'s members are.
#define PF_CAT_(a, b) a##b
#define PF_CAT(a, b) PF_CAT_(a, b)
#define PF_REGISTER_MODEL(MDL, ID, PARAMS, NAME)                                                                \
    static const bool PF_CAT(pf_model_registered_, __LINE__) =                                               \
        ::pfhost::register_model(::pfhost::model_entry<MDL, PARAMS>((ID), (NAME), offsetof(PARAMS, init_state)))

namespace pfhost {

// MTGP32 stream state for parameter set `set` seeded with `seed` (351 words).
void mtgp_init_state_host(uint32_t* st, int set, uint32_t seed);
// Torus dimensions: dx = 2^floor(log2 sqrt N), dy = N / dx.
void torus_dims(int N, int* dx, int* dy);
// Uniforms a sub-filter's resampler draws per step.
int64_t resample_draws(int res, int M);

}  // namespace pfhost
