// pf_launch.cuh -- host-side launchers: map runtime (model, m, particles per
// thread, resampler) onto the compiled kernel instantiations.
#pragma once

#include "pf_kernels.cuh"

namespace pfdev {

// (particles per sub-filter, particles per thread) pairs that are compiled.
#define PF_ME_LIST(X) X(32, 1) X(64, 2) X(128, 2) X(128, 4) X(256, 2) X(256, 4) X(512, 2) X(512, 4) X(1024, 2) X(1024, 4)

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

    static cudaError_t sample_sort(int M, int E, bool fr, int grid, cudaStream_t st, const FilterDesc* d,
                                   const int2* map, InputRef in)
    {
#define PF_K1(m, e)                                                                         \
    if (M == m && E == e) {                                                                 \
        if (fr) {                                                                           \
            auto fn = k_sample_sort<Mdl, m, e, true>;                                       \
            constexpr size_t sm = k1_smem<Mdl, m, true>();                                  \
            cudaError_t r = allow_smem(fn, sm);                                             \
            if (r != cudaSuccess) return r;                                                 \
            fn<<<grid, m / e, sm, st>>>(d, map, in);                                        \
        } else {                                                                            \
            auto fn = k_sample_sort<Mdl, m, e, false>;                                      \
            constexpr size_t sm = k1_smem<Mdl, m, false>();                                 \
            cudaError_t r = allow_smem(fn, sm);                                             \
            if (r != cudaSuccess) return r;                                                 \
            fn<<<grid, m / e, sm, st>>>(d, map, in);                                        \
        }                                                                                   \
        return cudaGetLastError();                                                          \
    }
        PF_ME_LIST(PF_K1)
#undef PF_K1
        return cudaErrorInvalidValue;
    }

    static cudaError_t sample_weight(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map,
                                     InputRef in)
    {
#define PF_SW(m, e)                                                       \
    if (M == m && E == e) {                                               \
        k_sample_weight<Mdl, m, e><<<grid, m / e, 0, st>>>(d, map, in);   \
        return cudaGetLastError();                                        \
    }
        PF_ME_LIST(PF_SW)
#undef PF_SW
        return cudaErrorInvalidValue;
    }

    static cudaError_t block_sort(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map)
    {
#define PF_BS(m, e)                                                     \
    if (M == m && E == e) {                                             \
        auto fn = k_block_sort<Mdl, m, e>;                              \
        constexpr size_t sm = (size_t)S * m * 4 + (size_t)m * 8;        \
        cudaError_t r = allow_smem(fn, sm);                             \
        if (r != cudaSuccess) return r;                                 \
        fn<<<grid, m / e, sm, st>>>(d, map);                            \
        return cudaGetLastError();                                      \
    }
        PF_ME_LIST(PF_BS)
#undef PF_BS
        return cudaErrorInvalidValue;
    }

    template <int RES>
    static cudaError_t exchange_resample_res(int M, int E, int grid, cudaStream_t st, const FilterDesc* d,
                                             const int2* map, int32_t* ctr, int virt)
    {
#define PF_K2(m, e)                                                     \
    if (M == m && E == e) {                                             \
        auto fn = k_exchange_resample<S, m, e, RES>;                    \
        constexpr size_t sm = k2_smem<S, m, e, RES>();                  \
        cudaError_t r = allow_smem(fn, sm);                             \
        if (r != cudaSuccess) return r;                                 \
        fn<<<grid, m / e, sm, st>>>(d, map, ctr, virt);                 \
        return cudaGetLastError();                                      \
    }
        PF_ME_LIST(PF_K2)
#undef PF_K2
        return cudaErrorInvalidValue;
    }

    static cudaError_t exchange_resample(int M, int E, int res, int grid, cudaStream_t st, const FilterDesc* d,
                                         const int2* map, int32_t* ctr, int virt)
    {
        if (res == PF_RESAMPLE_SYSTEMATIC)
            return exchange_resample_res<PF_RESAMPLE_SYSTEMATIC>(M, E, grid, st, d, map, ctr, virt);
        if (res == PF_RESAMPLE_REFERENCE)
            return exchange_resample_res<PF_RESAMPLE_REFERENCE>(M, E, grid, st, d, map, ctr, virt);
        return exchange_resample_res<PF_RESAMPLE_VOSE>(M, E, grid, st, d, map, ctr, virt);
    }

    static cudaError_t exchange_inplace(int grid, int threads, cudaStream_t st, const FilterDesc* d,
                                        const int2* map)
    {
        k_exchange_inplace<S><<<grid, threads, 0, st>>>(d, map);
        return cudaGetLastError();
    }

    static cudaError_t estimate(int nfilters, cudaStream_t st, const FilterDesc* d, InputRef in)
    {
        k_estimate<S><<<nfilters, 256, 0, st>>>(d, in, angle_mask());
        return cudaGetLastError();
    }

    static cudaError_t test_model(const ModelParams& mp, const pf_step_input* in, int n, float* state,
                                  const float* noise, float* ll, cudaStream_t st)
    {
        k_test_model<Mdl><<<(n + 127) / 128, 128, 0, st>>>(mp, in, n, state, noise, ll);
        return cudaGetLastError();
    }
};

extern template struct Launch<Unicycle>;
extern template struct Launch<DhArm>;
extern template struct Launch<RefArm>;

// Model-independent launchers (pf_common.cu).
cudaError_t launch_test_sort(int M, int E, int nsub, float* keys, int32_t* idx, cudaStream_t st);
cudaError_t launch_test_resample(int res, int M, int E, int nsub, const float* w, const float* u, int32_t* sel,
                                 float* prob, uint32_t* alias, cudaStream_t st);
cudaError_t launch_mtgp_blocks(int G, uint32_t* states, uint32_t* out, int64_t size, uint32_t mask, int float_out,
                               int set_base, cudaStream_t st);
cudaError_t launch_boxmuller(float* data, int64_t n, cudaStream_t st);
cudaError_t launch_a2a_merge(int nfilters, const FilterDesc* d, cudaStream_t st);
cudaError_t launch_exchange_sources(const FilterDesc* d, int32_t* src, cudaStream_t st);

}  // namespace pfdev
