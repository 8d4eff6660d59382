// pf_step.cuh -- state shared by the single-kernel step (pf_step_cta.cuh):
// the second half of the double-buffered sorted copy, the persistent step
// count whose parity selects the halves, the first-step flag and the group
// tickets of the estimate, and the estimate combination run by the last CTAs
// to finish a step.
#pragma once

#include "pf_kernels.cuh"

namespace pfdev {

// Extra per-filter state of the single-kernel pipeline.
struct StepState {
    float* tmp2;        // second half of the sorted-state double buffer (S*T)
    float* tkey2;       // second half of the sorted-key double buffer (T)
    int32_t* steps;     // persistent step count (buffer parity), never reset by runs
    int32_t* need_init; // 1: `state` holds the particles (first step / after set / restore)
    int32_t* grp_ctr;   // ceil(N/32) group tickets
};

// Group + final estimate by the last CTAs to finish (two-level ticket), run by
// one warp of each: the last CTA of a group of 32 sub-filters combines the
// group's partials, the last group the global estimate.
template <int S>
__device__ __forceinline__ void estimate_last_done(const FilterDesc& D, const StepState& X, int b,
                                                   const InputRef& in, int32_t* step_ctr, int lane)
{
    __syncwarp();
    __threadfence();
    const int g = b >> 5, ng = (D.N + 31) >> 5;
    const int gsize = (g == ng - 1) ? D.N - 32 * g : 32;
    int last = 0;
    if (lane == 0) last = atomicAdd(&X.grp_ctr[g], 1) == gsize - 1;
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    const int NV = 2 + S + D.na;
    group_row<S>(D, D.part + (int64_t)(32 * g) * kPartStride, D.winner + 32 * g, gsize, NV, 32 * g, lane,
              D.gpart + (int64_t)g * kPartStride);
    if (lane == 0) X.grp_ctr[g] = 0;
    // second level: the same combination as estimate_group
    __syncwarp();
    __threadfence();
    last = 0;
    if (lane == 0) last = atomicAdd(D.est_ctr, 1) == ng - 1;
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    double gm = -INFINITY;
    float bk = -INFINITY;
    int bi = 0x7fffffff;
    for (int q = lane; q < ng; q += 32) {
        const double* gq = D.gpart + (int64_t)q * kPartStride;
        gm = fmax(gm, __ldcg(gq));
        const float k = (float)__ldcg(gq + NV);
        const int i = (int)__ldcg(gq + NV + 1);
        if (k > bk || (k == bk && i < bi)) {
            bk = k;
            bi = i;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gm = fmax(gm, __shfl_xor_sync(kFull, gm, o));
        const float ok = __shfl_xor_sync(kFull, bk, o);
        const int oi = __shfl_xor_sync(kFull, bi, o);
        if (ok > bk || (ok == bk && oi < bi)) {
            bk = ok;
            bi = oi;
        }
    }
    const int par = (*X.steps) & 1;
    const float* cur_tmp = par ? X.tmp2 : D.tmp;
    estimate_write<S>(D, lane, ng, NV, gm, bk, bi, cur_tmp, D.est[step_index(in)], in.ctr ? *in.ctr + 1 : 0);
    if (lane == 0) {
        *D.est_ctr = 0;
        *X.need_init = 0;
        __threadfence();
        *X.steps += 1;
        if (step_ctr) *step_ctr += 1;
    }
}

}  // namespace pfdev
