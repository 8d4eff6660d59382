// pf_launch.cuh -- host-side launchers: map runtime (model, m, particles per
// thread, resampler) onto the compiled kernel instantiations.
#pragma once

#include "pf_step_cta.cuh"

namespace pfdev {

// (particles per sub-filter, particles per thread) pairs that are compiled.
#define PF_ME_LIST(X) X(32, 1) X(64, 2) X(128, 2) X(128, 4) X(256, 2) X(256, 4) X(256, 8) X(512, 2) X(512, 4) X(512, 16) X(1024, 2) X(1024, 4)

inline bool me_supported(int M, int E)
{
#define PF_ME_CHECK(m, e) if (M == m && E == e) return true;
    PF_ME_LIST(PF_ME_CHECK)
#undef PF_ME_CHECK
    return false;
}

// Opt a kernel into more than 48 KB of dynamic shared memory (once per instantiation).
template <class F>
inline cudaError_t allow_smem(F* fn, size_t bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes);
}

template <class Mdl>
struct Launch {
    static constexpr int S = Mdl::S;
    static uint32_t angle_mask()
    {
        uint32_t m = 0;
        for (int a = 0; a < Mdl::NA; ++a) m |= 1u << Mdl::angle_var(a);
        return m;
    }
    // tp: threads per particle (1, or 2 with fr)
    static cudaError_t sample_sort(int M, int E, int tp, bool fr, int grid, cudaStream_t st, const FilterDesc* d,
                                   const int2* map, InputRef in);
    static cudaError_t sample_weight(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map,
                                     InputRef in);
    static cudaError_t block_sort(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map);
    static cudaError_t k2_ref(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map,
                              InputRef in, int32_t* ctr, int virt);
    static cudaError_t k2_sys(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map,
                              InputRef in, int32_t* ctr, int virt);
    static cudaError_t k2_vose(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map,
                               InputRef in, int32_t* ctr, int virt);
    static cudaError_t exchange_resample(int M, int E, int res, int grid, cudaStream_t st, const FilterDesc* d,
                                         const int2* map, InputRef in, int32_t* ctr, int virt);
    static cudaError_t exchange_inplace(int grid, int threads, cudaStream_t st, const FilterDesc* d,
                                        const int2* map);
    static cudaError_t step_ref(int M, int E, int N, cudaStream_t st, const FilterDesc* d, const StepState& X,
                                InputRef in, int32_t* ctr, bool ro);
    static cudaError_t step_sys(int M, int E, int N, cudaStream_t st, const FilterDesc* d, const StepState& X,
                                InputRef in, int32_t* ctr, bool ro);
    static cudaError_t step_vose(int M, int E, int N, cudaStream_t st, const FilterDesc* d, const StepState& X,
                                 InputRef in, int32_t* ctr, bool ro);
    static cudaError_t step(int M, int E, int res, int N, cudaStream_t st, const FilterDesc* d, const StepState& X,
                            InputRef in, int32_t* ctr, bool resample_only);
    static cudaError_t test_model(const ModelParams& mp, const pf_step_input* in, int n, float* state,
                                  const float* noise, float* ll, cudaStream_t st);
};

// Members are defined in pf_launch_impl.cuh and instantiated by the pf_inst_*.cu files.

// Model-independent launchers (pf_common.cu).
cudaError_t launch_test_sort(int M, int E, int nsub, float* keys, int32_t* idx, int rank, int32_t* fallbacks,
                             cudaStream_t st);
cudaError_t launch_test_resample(int res, int M, int E, int nsub, const float* w, const float* u, int32_t* sel,
                                 float* prob, uint32_t* alias, cudaStream_t st);
cudaError_t launch_mtgp_blocks(int G, uint32_t* states, uint32_t* out, int64_t size, uint32_t mask, int float_out,
                               int set_base, cudaStream_t st);
cudaError_t launch_boxmuller(float* data, int64_t n, cudaStream_t st);
// Initial words of MTGP32 streams g0 .. g0+n-1 (parameter set g mod 200, seed + g + 1).
cudaError_t launch_mtgp_init(uint32_t* states, int n, int g0, uint32_t seed, cudaStream_t st);
cudaError_t launch_a2a_merge(int nfilters, const FilterDesc* d, cudaStream_t st);
cudaError_t launch_exchange_sources(const FilterDesc* d, int32_t* src, cudaStream_t st);
cudaError_t launch_a2a_merge_step(const FilterDesc* d, const StepState& X, cudaStream_t st);
cudaError_t launch_test_bounded_wait(int limit, int32_t* status, cudaStream_t st);
// shards (pf_shard_*)
cudaError_t launch_shard_pack(const FilterDesc* d, float* out, int S, int P, cudaStream_t st);
cudaError_t launch_shard_rows(const FilterDesc* d, int ng, double* rows, float* states, int S, int NV, cudaStream_t st);
cudaError_t launch_shard_estimate(const FilterDesc& D, int S, const float* best_src, pf_estimate* out, int ng,
                                  int32_t step_no, cudaStream_t st);
constexpr int kMixedWaitSrcBytes = 32768;  // the source buffer launch_test_bounded_wait_mixed copies
cudaError_t launch_test_bounded_wait_mixed(const int32_t* limits, int nthreads, const void* src, int32_t* outcome,
                                           int32_t* copied, cudaStream_t st);
cudaError_t launch_counter_inc(int32_t* ctr, cudaStream_t st);
cudaError_t launch_counter_set(int32_t* ctr, int32_t value, cudaStream_t st);


}  // namespace pfdev
