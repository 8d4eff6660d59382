// Model-independent launchers: RNG in the reference layout, Box-Muller,
// all-to-all merge, and the kernel-level test entry points.
#include "pf_launch.cuh"

namespace pfdev {

cudaError_t launch_test_sort(int M, int E, int nsub, float* keys, int32_t* idx, cudaStream_t st)
{
#define PF_TS(m, e)                                                  \
    if (M == m && E == e) {                                          \
        k_test_sort<m, e><<<nsub, m / e, 0, st>>>(keys, idx);        \
        return cudaGetLastError();                                   \
    }
    PF_ME_LIST(PF_TS)
#undef PF_TS
    return cudaErrorInvalidValue;
}

template <int RES>
static cudaError_t test_resample_res(int M, int E, int nsub, const float* w, const float* u, int32_t* sel,
                                     float* prob, uint32_t* alias, cudaStream_t st)
{
#define PF_TR(m, e)                                                                          \
    if (M == m && E == e) {                                                                  \
        constexpr size_t sm = RES == PF_RESAMPLE_SYSTEMATIC ? (size_t)m * 8                  \
                            : (RES == PF_RESAMPLE_REFERENCE ? (size_t)m * 4 : (size_t)m * 16); \
        k_test_resample<m, e, RES><<<nsub, m / e, sm, st>>>(w, u, sel, prob, alias);         \
        return cudaGetLastError();                                                           \
    }
    PF_ME_LIST(PF_TR)
#undef PF_TR
    return cudaErrorInvalidValue;
}

cudaError_t launch_test_resample(int res, int M, int E, int nsub, const float* w, const float* u, int32_t* sel,
                                 float* prob, uint32_t* alias, cudaStream_t st)
{
    if (res == PF_RESAMPLE_SYSTEMATIC)
        return test_resample_res<PF_RESAMPLE_SYSTEMATIC>(M, E, nsub, w, u, sel, prob, alias, st);
    if (res == PF_RESAMPLE_REFERENCE)
        return test_resample_res<PF_RESAMPLE_REFERENCE>(M, E, nsub, w, u, sel, prob, alias, st);
    return test_resample_res<PF_RESAMPLE_VOSE>(M, E, nsub, w, u, sel, prob, alias, st);
}

cudaError_t launch_mtgp_blocks(int G, uint32_t* states, uint32_t* out, int64_t size, uint32_t mask, int float_out,
                               int set_base, cudaStream_t st)
{
    k_mtgp_blocks<<<G, 256, 0, st>>>(states, out, size, mask, float_out, set_base);
    return cudaGetLastError();
}

cudaError_t launch_boxmuller(float* data, int64_t n, cudaStream_t st)
{
    const int64_t pairs = (n + 1) / 2;
    if (pairs == 0) return cudaSuccess;
    k_boxmuller<<<(unsigned)((pairs + 255) / 256), 256, 0, st>>>(data, n);
    return cudaGetLastError();
}

cudaError_t launch_a2a_merge(int nfilters, const FilterDesc* d, cudaStream_t st)
{
    k_a2a_merge<<<nfilters, 1024, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_exchange_sources(const FilterDesc* d, int32_t* src, cudaStream_t st)
{
    FilterDesc h;
    cudaError_t e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    k_exchange_sources<<<h.N, 256, 0, st>>>(d, src);
    return cudaGetLastError();
}

}  // namespace pfdev
