// pf_launch_impl.cuh -- out-of-class definitions of Launch<Mdl> members.  Each
// instantiation file defines one PF_PART_* macro so it compiles only the
// kernels it instantiates (keeps translation units small and parallel).
#pragma once

#include "pf_launch.cuh"

namespace pfdev {

#if defined(PF_PART_K1)
template <class Mdl>
cudaError_t Launch<Mdl>::sample_sort(int M, int E, int tp, bool fr, int grid, cudaStream_t st, const FilterDesc* d,
                                     const int2* map, InputRef in)
{
#define PF_K1_ONE(m, e, FR, TP)                                                             \
    {                                                                                       \
        auto fn = k_sample_sort<Mdl, m, e, FR, TP>;                                         \
        constexpr size_t sm = k1_smem<Mdl, m, FR, TP>();                                    \
        cudaError_t r = allow_smem(fn, sm);                                                 \
        if (r != cudaSuccess) return r;                                                     \
        fn<<<grid, TP * m / e, sm, st>>>(d, map, in);                                       \
        return cudaGetLastError();                                                          \
    }
#define PF_K1(m, e)                                                                         \
    if (M == m && E == e) {                                                                 \
        if (tp == 2) {                                                                      \
            if constexpr (2 * m / e <= 1024) {                                              \
                if (fr) PF_K1_ONE(m, e, true, 2)                                            \
            }                                                                               \
            return cudaErrorInvalidValue;                                                   \
        }                                                                                   \
        if (fr) PF_K1_ONE(m, e, true, 1)                                                    \
        PF_K1_ONE(m, e, false, 1)                                                           \
    }
    PF_ME_LIST(PF_K1)
#undef PF_K1
#undef PF_K1_ONE
    return cudaErrorInvalidValue;
}
#endif

#if defined(PF_PART_K2REF) || defined(PF_PART_K2SYS) || defined(PF_PART_K2VOSE)
#define PF_K2_CASE(m, e, RES)                                              \
    if (M == m && E == e) {                                                \
        auto fn = k_exchange_resample<Mdl::S, m, e, RES>;                  \
        constexpr size_t sm = k2_smem<Mdl::S, m, e, RES>();                \
        cudaError_t r = allow_smem(fn, sm);                                \
        if (r != cudaSuccess) return r;                                    \
        if (virt & 2) { /* programmatic dependent of the sampling kernel */ \
            cudaLaunchConfig_t lc = {};                                    \
            lc.gridDim = dim3(grid);                                       \
            lc.blockDim = dim3(m / e);                                     \
            lc.dynamicSmemBytes = sm;                                      \
            lc.stream = st;                                                \
            cudaLaunchAttribute at[1];                                     \
            at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization; \
            at[0].val.programmaticStreamSerializationAllowed = 1;          \
            lc.attrs = at;                                                 \
            lc.numAttrs = 1;                                               \
            return cudaLaunchKernelEx(&lc, fn, d, map, in, ctr, virt & 1); \
        }                                                                  \
        fn<<<grid, m / e, sm, st>>>(d, map, in, ctr, virt & 1);            \
        return cudaGetLastError();                                         \
    }
#define PF_K2_CASE_0(m, e) PF_K2_CASE(m, e, 0)
#define PF_K2_CASE_1(m, e) PF_K2_CASE(m, e, 1)
#define PF_K2_CASE_2(m, e) PF_K2_CASE(m, e, 2)
#define PF_K2_DEF(NAME, RES)                                                                            \
    template <class Mdl>                                                                                \
    cudaError_t Launch<Mdl>::NAME(int M, int E, int grid, cudaStream_t st, const FilterDesc* d,       \
                                  const int2* map, InputRef in, int32_t* ctr, int virt)               \
    {                                                                                                   \
        PF_ME_LIST(PF_K2_CASE_##RES)                                                                    \
        return cudaErrorInvalidValue;                                                                   \
    }
#if defined(PF_PART_K2REF)
PF_K2_DEF(k2_ref, 0)
#endif
#if defined(PF_PART_K2SYS)
PF_K2_DEF(k2_sys, 1)
#endif
#if defined(PF_PART_K2VOSE)
PF_K2_DEF(k2_vose, 2)
#endif
#endif

#if defined(PF_PART_PHASED)
template <class Mdl>
cudaError_t Launch<Mdl>::sample_weight(int M, int E, int grid, cudaStream_t st, const FilterDesc* d,
                                       const int2* map, InputRef in)
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

template <class Mdl>
cudaError_t Launch<Mdl>::block_sort(int M, int E, int grid, cudaStream_t st, const FilterDesc* d, const int2* map)
{
#define PF_BS(m, e)                                                     \
    if (M == m && E == e) {                                             \
        auto fn = k_block_sort<Mdl, m, e>;                              \
        constexpr size_t sm = (size_t)Mdl::S * m * 4 + (size_t)m * 8;   \
        cudaError_t r = allow_smem(fn, sm);                             \
        if (r != cudaSuccess) return r;                                 \
        fn<<<grid, m / e, sm, st>>>(d, map);                            \
        return cudaGetLastError();                                      \
    }
    PF_ME_LIST(PF_BS)
#undef PF_BS
    return cudaErrorInvalidValue;
}

template <class Mdl>
cudaError_t Launch<Mdl>::exchange_resample(int M, int E, int res, int grid, cudaStream_t st, const FilterDesc* d,
                                           const int2* map, InputRef in, int32_t* ctr, int virt)
{
    if (res == PF_RESAMPLE_SYSTEMATIC) return k2_sys(M, E, grid, st, d, map, in, ctr, virt);
    if (res == PF_RESAMPLE_REFERENCE) return k2_ref(M, E, grid, st, d, map, in, ctr, virt);
    return k2_vose(M, E, grid, st, d, map, in, ctr, virt);
}

template <class Mdl>
cudaError_t Launch<Mdl>::exchange_inplace(int grid, int threads, cudaStream_t st, const FilterDesc* d,
                                          const int2* map)
{
    k_exchange_inplace<Mdl::S><<<grid, threads, 0, st>>>(d, map);
    return cudaGetLastError();
}

template <class Mdl>
cudaError_t Launch<Mdl>::step(int M, int E, int res, int N, cudaStream_t st, const FilterDesc* d,
                              const StepState& X, InputRef in, int32_t* ctr, bool resample_only)
{
    if (res == PF_RESAMPLE_SYSTEMATIC) return step_sys(M, E, N, st, d, X, in, ctr, resample_only);
    if (res == PF_RESAMPLE_REFERENCE) return step_ref(M, E, N, st, d, X, in, ctr, resample_only);
    return step_vose(M, E, N, st, d, X, in, ctr, resample_only);
}

template <class Mdl>
cudaError_t Launch<Mdl>::test_model(const ModelParams& mp, const pf_step_input* in, int n, float* state,
                                    const float* noise, float* ll, cudaStream_t st)
{
    k_test_model<Mdl><<<(n + 127) / 128, 128, 0, st>>>(mp, in, n, state, noise, ll);
    return cudaGetLastError();
}
#endif

#if defined(PF_PART_STEPREF) || defined(PF_PART_STEPSYS) || defined(PF_PART_STEPVOSE)
#define PF_STEP_CASE(m, e, RES)                                      \
    if (M == m && E == e) {                                          \
        constexpr size_t sm = step_cta_smem<Mdl, m, e, RES>();       \
        if (ro) {                                                    \
            auto fn = k_resample_only_cta<Mdl, m, e, RES>;           \
            cudaError_t r = allow_smem(fn, sm);                      \
            if (r != cudaSuccess) return r;                          \
            fn<<<N, m / e, sm, st>>>(d, X);                          \
        } else {                                                     \
            auto fn = k_step_cta<Mdl, m, e, RES>;                    \
            cudaError_t r = allow_smem(fn, sm);                      \
            if (r != cudaSuccess) return r;                          \
            fn<<<N, m / e, sm, st>>>(d, X, in, ctr);                 \
        }                                                            \
        return cudaGetLastError();                                   \
    }
#define PF_STEP_CASE_0(m, e) PF_STEP_CASE(m, e, 0)
#define PF_STEP_CASE_1(m, e) PF_STEP_CASE(m, e, 1)
#define PF_STEP_CASE_2(m, e) PF_STEP_CASE(m, e, 2)
#define PF_STEP_DEF(NAME, RES)                                                                                 \
    template <class Mdl>                                                                                       \
    cudaError_t Launch<Mdl>::NAME(int M, int E, int N, cudaStream_t st, const FilterDesc* d, const StepState& X, \
                                  InputRef in, int32_t* ctr, bool ro)                                         \
    {                                                                                                          \
        PF_ME_LIST(PF_STEP_CASE_##RES)                                                                         \
        return cudaErrorInvalidValue;                                                                          \
    }
#if defined(PF_PART_STEPREF)
PF_STEP_DEF(step_ref, 0)
#endif
#if defined(PF_PART_STEPSYS)
PF_STEP_DEF(step_sys, 1)
#endif
#if defined(PF_PART_STEPVOSE)
PF_STEP_DEF(step_vose, 2)
#endif
#endif

}  // namespace pfdev
