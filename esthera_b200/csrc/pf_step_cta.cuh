// pf_step_cta.cuh -- the single-kernel step, one CTA per sub-filter.
//
// One launch per filter step.  The exchange needs every neighbour's sorted
// top-t, so the resampling of step k-1 runs at the start of step k, from the
// sorted copy step k-1 left in one half of a double buffer (tmp/tkey or
// tmp2/tkey2, by the parity of the persistent step count); step k writes its
// sorted copy to the other half.  Phases per CTA:
//   R  resample_from() the previous sorted copy (exchange applied virtually)
//      into registers -- or load `state` on the first step after it was set,
//      and for a sub-filter that skipped resampling (it keeps its propagated
//      particles, written in place)
//   G  this step's MTGP32 draws (normals -> shared memory, uniforms -> ru),
//      Box-Muller
//   P  propagate + log-likelihood of the thread's E particles
//   S  bitonic sort; sorted keys and particles -> this step's half; winner;
//      FP64 estimate partials
//   E  group / final estimate by the last CTAs to finish (two-level tickets)
// The arithmetic of every phase is the split pipeline's (k_exchange_resample
// + k_sample_sort), so both give bit-identical particles and estimates; the
// resampled particles stay in registers instead of a round trip through HBM.
#pragma once

#include "pf_step.cuh"

namespace pfdev {

template <class Mdl, int M, int E, int RES>
constexpr size_t step_cta_smem()
{
    const size_t a = k1_smem<Mdl, M, true>(), b = k2_smem<Mdl::S, M, E, RES>();
    return a > b ? a : b;
}

template <class Mdl, int M, int E, int RES>
__global__ void __launch_bounds__(M / E, pf_min_blocks(M / E, pf_k1_warps(Mdl::S)))
    k_step_cta(const FilterDesc* __restrict__ descs, StepState X, InputRef in, int32_t* step_ctr)
{
    constexpr int NT = M / E, S = Mdl::S, K = Mdl::K, NA = Mdl::NA;
    constexpr int NANG = NA > 0 ? NA : 1;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ typename Mdl::Consts cst;
    __shared__ double dred[64];
    __shared__ int ired[34];
    __shared__ float s_lmax;
    __shared__ uint64_t mbar;
    __shared__ FilterDesc sdesc;
    const FilterDesc& D = load_desc(sdesc, descs);
    const int b = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t T = D.T;
    const int64_t base = (int64_t)b * M + E * tid;
    const int par = (*X.steps) & 1;
    const int init = *X.need_init;
    float* cur_tmp = par ? X.tmp2 : D.tmp;
    float* cur_key = par ? X.tkey2 : D.tkey;
    const float* prev_tmp = par ? D.tmp : X.tmp2;
    const float* prev_key = par ? D.tkey : X.tkey2;
    float* ru = D.ru + (int64_t)b * D.ru_stride;
    if (tid < 32) Mdl::prepare(cst, *input_of(in, 0), D.mp, tid);

    // ---- R
    float st[E][S];
    int rs = PF_RS_KEPT;
    if (!init) {
        int sel[E];
        rs = resample_from<S, M, E, RES>(D, b, prev_tmp, prev_key, ru, exchange_count(D), smem, dred, ired, &mbar,
                                         st, sel);
        if (D.sel) {
#pragma unroll
            for (int e = 0; e < E; ++e) D.sel[base + e] = rs == PF_RS_RESAMPLED ? sel[e] : -1;
        }
    }
    if (rs == PF_RS_LOST) {
        // bulk copies may still be landing in dynamic shared memory, which G..S
        // reuse: skip them (the status word already reports the timeout); the
        // estimate tickets still count this CTA so the next step starts clean
        if (tid < 32) estimate_last_done<S>(D, X, b, in, step_ctr, tid);
        return;
    }
    if (rs != PF_RS_RESAMPLED) {
#pragma unroll
        for (int v = 0; v < S; ++v) {
            float o[E];
            ldv<E>(D.state + v * T + base, o);
#pragma unroll
            for (int e = 0; e < E; ++e) st[e][v] = o[e];
        }
    }
    __syncthreads();  // R's shared memory and its reads of ru are done: G reuses both

    // ---- G (the sampling kernel's layout of shared memory)
    unsigned char* p = smem;
    MtgpSmem* ms = reinterpret_cast<MtgpSmem*>(p);
    p += sizeof(MtgpSmem);
    float* nz = reinterpret_cast<float*>(p);
    float* stage = nz;
    p += k1_stage_bytes<Mdl, M, true>();
    float* sk = reinterpret_cast<float*>(p);
    int* si = reinterpret_cast<int*>(p + (size_t)M * 4);
    {
        uint32_t* gst = D.mtgp + (int64_t)b * kMtgpN;
        mtgp_load(*ms, gst, (D.stream_base + b) % kMtgpSets, D.mask, true);
        const int nbm = D.nbm;
        mtgp_generate_bm<raw_normals<Mdl, E>()>(*ms, D.draws, nbm, nz,
                                                [&](int k, uint32_t o) { ru[k - nbm] = __uint_as_float(o); });
        mtgp_store(*ms, gst, D.draws);
    }
    __syncthreads();

    // ---- P
    float okey[E], sn[E][NANG], cs[E][NANG];
    {
        float ll[E];
        if constexpr (raw_normals<Mdl, E>()) {
            float z[E][K];
            normals_from_raw<Mdl, M, E>(nz, tid, z);
            model_step_batch<Mdl, E>(cst, st, [&](int e, int v) { return z[e][v]; }, sn, cs, ll);
        } else {
            model_step_batch<Mdl, E>(
                cst, st, [&](int e, int v) { return nz[v * M + E * tid + e]; }, sn, cs, ll);
        }
#pragma unroll
        for (int e = 0; e < E; ++e) okey[e] = D.log_weights ? ll[e] : __expf(ll[e]);
    }
    if (D.inplace) {
#pragma unroll
        for (int v = 0; v < S; ++v) {
            float o[E];
#pragma unroll
            for (int e = 0; e < E; ++e) o[e] = st[e][v];
            stv<E>(D.state + v * T + base, o);
        }
    }

    // ---- S
    float k[E];
    int ix[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        k[e] = okey[e];
        ix[e] = E * tid + e;
    }
    sort_subfilter<Mdl, M, E>(k, ix, sk, si);
    stv<E>(cur_key + base, k);
    __syncthreads();  // normals consumed, sort buffers free: stage the state
#pragma unroll
    for (int v = 0; v < S; ++v)
#pragma unroll
        for (int e = 0; e < E; ++e) stage[v * M + E * tid + e] = st[e][v];
    if (tid == 0) {
        D.winner[b] = k[0];
        s_lmax = k[0];
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
#pragma unroll
        for (int e = 0; e < E; ++e) o[e] = stage[v * M + ix[e]];
        stv<E>(cur_tmp + v * T + base, o);
    }
    write_partials<Mdl, E, NT, k1_stage_bytes<Mdl, M, true>()>(D, b, D.log_weights ? s_lmax : 0.0f, okey, st, sn,
                                                                cs, reinterpret_cast<double*>(stage));

    // ---- E (warp 0 wrote the partials)
    if (tid < 32) estimate_last_done<S>(D, X, b, in, step_ctr, tid);
}

// Phase R alone: the particles after the last step's resampling into `state`
// (the selection optionally recorded).  Reads the half written last.
template <class Mdl, int M, int E, int RES>
__global__ void __launch_bounds__(M / E) k_resample_only_cta(const FilterDesc* __restrict__ descs, StepState X)
{
    constexpr int S = Mdl::S;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double dred[64];
    __shared__ int ired[34];
    __shared__ uint64_t mbar;
    __shared__ FilterDesc sdesc;
    const FilterDesc& D = load_desc(sdesc, descs);
    if (*X.need_init) return;  // `state` already holds the particles
    const int b = blockIdx.x;
    const int64_t base = (int64_t)b * M + E * threadIdx.x;
    const int par = ((*X.steps) & 1) ^ 1;
    const float* t_tmp = par ? X.tmp2 : D.tmp;
    const float* t_key = par ? X.tkey2 : D.tkey;
    const float* ru = D.ru + (int64_t)b * D.ru_stride;
    float st[E][S];
    int sel[E];
    const bool resampled = resample_from<S, M, E, RES>(D, b, t_tmp, t_key, ru, exchange_count(D), smem, dred, ired,
                                                       &mbar, st, sel) == PF_RS_RESAMPLED;
    if (D.sel) {
#pragma unroll
        for (int e = 0; e < E; ++e) D.sel[base + e] = resampled ? sel[e] : -1;
    }
    if (!resampled) return;  // skipped: `state` holds the propagated particles (written in place)
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
#pragma unroll
        for (int e = 0; e < E; ++e) o[e] = st[e][v];
        stv<E>(D.state + v * D.T + base, o);
    }
}

}  // namespace pfdev
