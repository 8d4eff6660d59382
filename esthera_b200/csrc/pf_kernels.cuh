// pf_kernels.cuh -- kernels of the particle-filter step (sm_100a).
//
// Split pipeline (two launches per step; batches and the server use it too):
//   k_sample_sort       one CTA per sub-filter: MTGP32 stream -> Box-Muller in
//                       shared memory -> propagate + log-weight (float4 SoA
//                       loads) -> bitonic sort -> sorted state/keys, winner,
//                       FP64 estimate partials
//   k_a2a_merge         (all-to-all exchange only) global top-t of the sorted lists
//   k_exchange_resample one CTA per sub-filter, estimate-combining group
//                       leaders first: neighbours' top-t into the weakest
//                       slots, weights, resampling, gather, store
// Single-kernel pipeline: k_step_cta (pf_step_cta.cuh), the same phases in one
// launch with the resampling deferred to the next step.
// Phased pipeline (the reference's kernel sequence, pf_generic_soa.cu:842-1234):
//   k_mtgp_blocks -> k_boxmuller -> k_sample_weight -> k_block_sort ->
//   k_exchange_inplace -> k_exchange_resample (estimate combined at its start)
#pragma once

#include "pf_device.cuh"

namespace pfdev {

constexpr int kPartStride = 32;  // doubles of estimate partials per sub-filter

struct FilterDesc {
    float* state;      // S*T SoA (var-major), propagated / resampled particles
    float* tmp;        // S*T sorted (pre-exchange) particles
    float* tkey;       // T sorted keys
    float* key;        // T unsorted keys (phased pipeline)
    float* winner;     // N best keys
    double* part;      // N * kPartStride estimate partials
    uint32_t* mtgp;    // MTGP32 stream words (351 per stream)
    float* ru;         // per sub-filter resampling uniforms (fused RNG): decision, then resampler draws
    const float* rbuf; // reference-layout random buffer: normals then uniforms
    int32_t* a2a;      // all-to-all: t global slots of the global best
    int32_t* sel;      // optional T selected slots
    pf_estimate* est;  // estimate output (indexed by the step counter when one is used)
    int64_t T;
    int32_t N, M, t, exchange, resampler, dx, dy;
    int32_t log_weights, inplace, rng_fused, draws, nbm, ru_stride;
    uint32_t mask;
    int32_t stream_base;
    float freq;
    float ess_frac;    // > 0: a sub-filter resamples only while its ESS < ess_frac * m
    int64_t nnorm;     // normals in rbuf before the uniforms (K*T)
    int32_t* est_ctr;  // ticket counter of the two-level estimate (0 between steps)
    double* gpart;     // ceil(N/32) * kPartStride group partials
    uint32_t angle_mask;
    int32_t na;        // angular state variables (circular means)
    int32_t exch_period;  // exchange on steps with step % period == 0 (<= 1: every step)
    int32_t* status;      // PF_STATUS_* bits set by the kernels (0: all well)
    // a shard of a larger filter (pf_shard_*): this filter's sub-filters are
    // the global ones b0 .. b0+N-1, whole rows r0 .. r0 + N/dx - 1 of the
    // global dx x gdy torus; the rows just outside come from the neighbouring
    // shards through `halo`
    int32_t shard;        // 0: a whole filter
    int32_t b0, r0, gdy;
    const float* halo;    // [2][1+S][dx*t]: block 0 row r0-1 (top), block 1 the row after the last (bottom); key row then state rows
    ModelParams mp;
};

// status bits: a bounded wait on a bulk copy ran out (the sub-filter kept its
// propagated particles); a sorted copy handed to the resampling was not
// 16-byte aligned (not this library's allocation; the sub-filter kept its
// propagated particles)
constexpr int PF_STATUS_WAIT_TIMEOUT = 1;
constexpr int PF_STATUS_MISALIGNED = 2;

// Outcome of resample_from: the CTA resampled; it kept its propagated
// particles (decision uniform, ESS gate, misaligned rows, or a wait that ran
// out after which the copies still landed); or its bulk copies may still be
// landing in shared memory, so the CTA must not touch its dynamic shared
// memory again.
constexpr int PF_RS_RESAMPLED = 1;
constexpr int PF_RS_KEPT = 0;
constexpr int PF_RS_LOST = -1;

// A CTA's filter descriptor, copied once into shared memory (all threads of
// the CTA call this at their start).  The kernels read descriptor fields all
// through their phases; read from global memory, a field whose line the
// streamed particle tiles have evicted from L1 costs a round trip to L2 in
// the middle of a dependent chain.
__device__ __forceinline__ const FilterDesc& load_desc(FilterDesc& sd, const FilterDesc* g)
{
    static_assert(sizeof(FilterDesc) % 8 == 0, "descriptor copied in 8-byte words");
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(g);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
    for (int i = threadIdx.x; i < (int)(sizeof(FilterDesc) / 8); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    return sd;
}

// Programmatic dependent launch (split pipeline): the sampling kernel lets the
// resampling kernel's CTAs launch once all of its own CTAs are running, and
// those wait in wait_prerequisites() -- after their prologue -- until the
// sampling kernel has completed and its writes are visible.  Both are no-ops
// for kernels launched without the programmatic attribute.
__device__ __forceinline__ void allow_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void wait_prerequisites() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Register budgets of the split pipeline's kernels, as resident warps per SM
// asked of the compiler: __launch_bounds__(threads, ceil(warps * 32 / threads))
// caps the registers at 65536 / (that many threads).  Small states (the
// unicycle's 3 variables) take 36 / 32 warps: the sampling kernel at m = 512,
// 4 particles per thread runs 53 us capped at 56 registers against 59 us at
// the compiler's own 83.  The arms' states (9-12 variables, forward
// kinematics) need ~128 registers per thread; capping them lower spills.
// The sampling kernel with two threads per particle asks for 4 warps fewer
// (its CTAs are twice as large, so the rounding up of whole CTAs would
// otherwise cut its registers below the one-thread kernel's).
#ifndef PF_K1_WARPS_SMALL
#define PF_K1_WARPS_SMALL 36
#endif
#ifndef PF_K1_WARPS_LARGE
#define PF_K1_WARPS_LARGE 16
#endif
#ifndef PF_K2_WARPS_SMALL
#define PF_K2_WARPS_SMALL 32
#endif
#ifndef PF_K2_WARPS_LARGE
#define PF_K2_WARPS_LARGE 16
#endif
__host__ __device__ constexpr int pf_min_blocks(int threads, int warps)
{
    return (warps * 32 + threads - 1) / threads > 32 ? 32 : (warps * 32 + threads - 1) / threads;
}
// Large states with 2 or fewer particles per thread hold half the registers a
// thread of 4 needs: their budget is 32 warps (64 registers; the DH arm's
// sampling kernel at m = 256 runs 26.4 us against 29.6 us at 128 registers
// and 28.8 us with 4 particles per thread).
#ifndef PF_K1_WARPS_LARGE_E2
#define PF_K1_WARPS_LARGE_E2 32
#endif
__host__ __device__ constexpr int pf_k1_warps(int S, int E = 4)
{
    return S <= 3 ? PF_K1_WARPS_SMALL : (E <= 2 ? PF_K1_WARPS_LARGE_E2 : PF_K1_WARPS_LARGE);
}
__host__ __device__ constexpr int pf_k2_warps(int S) { return S <= 3 ? PF_K2_WARPS_SMALL : PF_K2_WARPS_LARGE; }

struct InputRef {
    const pf_step_input* base;
    int64_t filter_stride;   // inputs per filter (batched: [filter][step])
    const int32_t* ctr;      // device step counter (graph replays) or null
    int32_t cap;             // inputs / estimates per filter: the counter indexes them modulo cap
    int32_t step;            // step number of this step when there is no device counter
};

// Step number within the run: the device counter, else the host-given number.
__device__ __forceinline__ int32_t run_step(const InputRef& in) { return in.ctr ? *in.ctr : in.step; }

__device__ __forceinline__ int64_t step_index(const InputRef& in)
{
    // unsigned: a counter that wrapped past 2^31 steps still maps into [0, cap)
    return in.ctr ? (int64_t)((uint32_t)*in.ctr % (uint32_t)(in.cap > 0 ? in.cap : 1)) : 0;
}


// E consecutive floats per thread: float4 chunks when E is a multiple of 4.
template <int E>
__device__ __forceinline__ void ldv(const float* __restrict__ p, float (&o)[E])
{
    if constexpr (E % 4 == 0) {
#pragma unroll
        for (int q = 0; q < E; q += 4) {
            const float4 v = *reinterpret_cast<const float4*>(p + q);
            o[q] = v.x; o[q + 1] = v.y; o[q + 2] = v.z; o[q + 3] = v.w;
        }
    } else if constexpr (E == 2) {
        const float2 v = *reinterpret_cast<const float2*>(p);
        o[0] = v.x; o[1] = v.y;
    } else {
#pragma unroll
        for (int q = 0; q < E; ++q) o[q] = p[q];
    }
}
template <int E>
__device__ __forceinline__ void stv(float* __restrict__ p, const float (&o)[E])
{
    if constexpr (E % 4 == 0) {
#pragma unroll
        for (int q = 0; q < E; q += 4)
            *reinterpret_cast<float4*>(p + q) = make_float4(o[q], o[q + 1], o[q + 2], o[q + 3]);
    } else if constexpr (E == 2) {
        *reinterpret_cast<float2*>(p) = make_float2(o[0], o[1]);
    } else {
#pragma unroll
        for (int q = 0; q < E; ++q) p[q] = o[q];
    }
}

__device__ __forceinline__ void cta_target(const int2* __restrict__ cta_map, int& f, int& b)
{
    if (cta_map) {
        const int2 c = cta_map[blockIdx.x];
        f = c.x;
        b = c.y;
    } else {
        f = 0;
        b = blockIdx.x;
    }
}

// The resampling kernel's grid: one estimate CTA per group of 32 sub-filters
// first (it combines the group's partial rows; the last of them, by ticket,
// the global estimate), then one CTA per sub-filter, so the estimate runs in
// short CTAs of the first wave instead of lengthening resampling CTAs.
// Without a CTA map CTA i < ng is group i's estimate CTA and CTA ng + j
// resamples sub-filter j; maps built by the batch and the server list
// (filter, -1 - g) entries first in the same way (the sampling kernel is
// given the map past them).  Returns the sub-filter, or -1 - g.
__host__ __device__ constexpr int estimate_ctas(int N) { return (N + 31) >> 5; }
__device__ __forceinline__ int resample_cta(int i, int N)
{
    const int ng = estimate_ctas(N);
    return i < ng ? -1 - i : i - ng;
}

__device__ __forceinline__ const pf_step_input* input_of(const InputRef& in, int f)
{
    return in.base + (int64_t)f * in.filter_stride + step_index(in);
}

// Whether the sampling kernels leave Box-Muller out of the MTGP32 rounds: for
// small states with an even number of particles per thread, each thread turns
// the raw pairs of its own particles (e, e+1) into normals in registers right
// before the model (independent chains, no barrier between them).
template <class Mdl, int E>
constexpr bool raw_normals() { return E % 2 == 0 && Mdl::K * E <= 16; }

// This thread's E x K normals from the raw MTGP32 words in shared memory
// (raw_normals): pair (v M + E tid + e, +1) -> particles e, e+1 of variable v.
template <class Mdl, int M, int E>
__device__ __forceinline__ void normals_from_raw(const float* nz, int tid, float (&z)[E][Mdl::K])
{
#pragma unroll
    for (int v = 0; v < Mdl::K; ++v)
#pragma unroll
        for (int e = 0; e < E; e += 2) {
            const float2 u = *reinterpret_cast<const float2*>(nz + v * M + E * tid + e);
            box_muller(u.x, u.y, z[e][v], z[e + 1][v]);
        }
}

// k_sample_sort's dynamic shared memory: the MTGP32 ring (FR), one region
// holding in turn the normals, the state stage of the sorted gather and the
// estimate partials' per-thread sums, then the sort keys + indices.
template <class Mdl, int M, bool FR, int TP = 1>
constexpr size_t k1_stage_bytes()
{
    const size_t nz = FR ? (size_t)(2 * ((Mdl::K * M + 1) / 2)) * 4 : 0;
    size_t stage = (size_t)Mdl::S * M * 4;
    if (TP > 1 && stage < (size_t)TP * M * 8) stage = (size_t)TP * M * 8;  // a row of partials per thread
    return nz > stage ? nz : stage;
}
template <class Mdl, int M, bool FR, int TP = 1>
constexpr size_t k1_smem()
{
    return (FR ? sizeof(MtgpSmem) : 0) + k1_stage_bytes<Mdl, M, FR, TP>() + (size_t)M * 8;
}

// Estimate partials of one sub-filter from particles in any order:
// [0] key max, [1] sum w, [2+v] sum w x_v (angles: sum w sin), [2+S+a] sum w cos.
// Each thread sums its E particles in FP64, in order; sn / cs are the sines
// and cosines of the angular state variables, as the model returned them.
// The NV x NT per-thread sums then go through shared memory (acc, ACC_BYTES
// bytes, free for this call; chunks of values when they do not all fit): P
// consecutive lanes per value (P the largest power of two with NV * P <= NT,
// at most 32) each add NT / P rows in order, then an xor-shuffle tree over
// the P lanes.  A fixed order: deterministic for a given (M, E).  A thread
// with counts = false (the second lane of a particle pair) adds zeros.
template <class Mdl, int E, int NT, size_t ACC_BYTES>
__device__ __forceinline__ void write_partials(const FilterDesc& D, int b, float lmax, const float (&okey)[E],
                                               const float (&st)[E][Mdl::S],
                                               const float (&sn)[E][Mdl::NA > 0 ? Mdl::NA : 1],
                                               const float (&cs)[E][Mdl::NA > 0 ? Mdl::NA : 1], double* acc,
                                               bool counts = true)
{
    constexpr int S = Mdl::S, NA = Mdl::NA, NV = 1 + S + NA;
    constexpr int CH = (int)(ACC_BYTES / (8 * NT)) < NV ? (int)(ACC_BYTES / (8 * NT)) : NV;  // values per chunk
    static_assert(CH >= 1, "the partials buffer holds at least one row of per-thread sums");
    constexpr int PR = NT / CH;
    constexpr int P = PR >= 32 ? 32 : (PR >= 16 ? 16 : (PR >= 8 ? 8 : (PR >= 4 ? 4 : (PR >= 2 ? 2 : 1))));
    const int tid = threadIdx.x;
    double w[E];
#pragma unroll
    for (int e = 0; e < E; ++e) w[e] = D.log_weights ? (double)__expf(okey[e] - lmax) : (double)okey[e];
    double* out = D.part + (int64_t)b * kPartStride;
#pragma unroll
    for (int c0 = 0; c0 < NV; c0 += CH) {
        __syncthreads();  // the buffer (or the previous chunk) is free
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int i = c0 + c;
            if (i < NV) {
                double a = 0.0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    if (i == 0) {
                        a += w[e];
                    } else if (i <= S) {
                        const int v = i - 1;
                        float x = st[e][v];
                        if constexpr (NA > 0) {
                            if (is_angle_var<Mdl>(v)) {
                                int ai = 0;
#pragma unroll
                                for (int q = 0; q < NA; ++q)
                                    if (Mdl::angle_var(q) == v) ai = q;
                                x = sn[e][ai];
                            }
                        }
                        a += w[e] * (double)x;
                    } else {
                        a += w[e] * (double)cs[e][i - 1 - S];
                    }
                }
                acc[c * NT + tid] = counts ? a : 0.0;
            }
        }
        __syncthreads();
        const int c = tid / P, j = tid % P;
        double a = 0.0;
        if (c < CH && c0 + c < NV) {
#pragma unroll 4
            for (int t = j; t < NT; t += P) a += acc[c * NT + t];
        }
#pragma unroll
        for (int o = P / 2; o > 0; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
        if (j == 0 && c < CH && c0 + c < NV) out[1 + c0 + c] = a;
    }
    if (tid == 0) out[0] = (double)lmax;
}

// ---------------------------------------------------------------------------
// Fused propagate + weight + sort.  FR: generate this sub-filter's MTGP32
// stream in the kernel; otherwise read reference-layout normals from rbuf.
// TP = 2: two threads per particle -- lanes 2g and 2g+1 both hold particles
// E g .. E g + E - 1, split each particle's model work (model_step_tp), run the
// sort together, and lane 2g alone writes (its partials carry the particles).
// ---------------------------------------------------------------------------
template <class Mdl, int M, int E, bool FR, int TP = 1>
__global__ void __launch_bounds__(TP * M / E, pf_min_blocks(TP * M / E, pf_k1_warps(Mdl::S, E) - (TP - 1) * 4)) k_sample_sort(const FilterDesc* __restrict__ descs,
                                                       const int2* __restrict__ cta_map, InputRef in)
{
    constexpr int NT = TP * M / E, S = Mdl::S, K = Mdl::K, NA = Mdl::NA;
    constexpr int NANG = NA > 0 ? NA : 1;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ typename Mdl::Consts cst;
    __shared__ float s_lmax;
    __shared__ FilterDesc sdesc;
    int f, b;
    cta_target(cta_map, f, b);
    allow_dependents();
    const FilterDesc& D = load_desc(sdesc, descs + f);
    const int tid = threadIdx.x;
    const int vt = tid / TP, h = tid % TP;  // the thread's E particles, its half of them
    const bool writer = h == 0;
    const int64_t T = D.T;
    const int64_t base = (int64_t)b * M + E * vt;

    unsigned char* p = smem;
    MtgpSmem* ms = nullptr;
    if constexpr (FR) {
        ms = reinterpret_cast<MtgpSmem*>(p);
        p += sizeof(MtgpSmem);
    }
    float* nz = reinterpret_cast<float*>(p);     // normals (FR), later the state stage, then the partials
    float* stage = nz;
    p += k1_stage_bytes<Mdl, M, FR, TP>();
    float* sk = reinterpret_cast<float*>(p);
    int* si = reinterpret_cast<int*>(p + (size_t)M * 4);

    if constexpr (FR) {
        uint32_t* gst = D.mtgp + (int64_t)b * kMtgpN;
        // the step's model constants (one warp) while the stream words are in flight
        mtgp_load_overlap<NT>(*ms, gst, (D.stream_base + b) % kMtgpSets, D.mask, [&] {
            if (tid < 32) Mdl::prepare(cst, *input_of(in, f), D.mp, tid);
        });
        const int nbm = D.nbm;
        float* ru = D.ru + (int64_t)b * D.ru_stride;
        mtgp_generate_bm<raw_normals<Mdl, E>()>(*ms, D.draws, nbm, nz,
                                                [&](int k, uint32_t o) { ru[k - nbm] = __uint_as_float(o); });
        mtgp_store(*ms, gst, D.draws);
    } else {
        if (tid < 32) Mdl::prepare(cst, *input_of(in, f), D.mp, tid);
    }
    __syncthreads();

    float st[E][S];
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
        ldv<E>(D.state + v * T + base, o);
#pragma unroll
        for (int e = 0; e < E; ++e) st[e][v] = o[e];
    }
    float okey[E], sn[E][NANG], cs[E][NANG];
    {
        float ll[E];
        if constexpr (FR && raw_normals<Mdl, E>()) {
            float z[E][K];
            normals_from_raw<Mdl, M, E>(nz, vt, z);
            model_step_tp<Mdl, E, TP>(cst, st, [&](int e, int v) { return z[e][v]; }, h, sn, cs, ll);
        } else {
            model_step_tp<Mdl, E, TP>(
                cst, st,
                [&](int e, int v) { return FR ? nz[v * M + E * vt + e] : D.rbuf[v * T + base + e]; }, h, sn, cs,
                ll);
        }
#pragma unroll
        for (int e = 0; e < E; ++e) okey[e] = D.log_weights ? ll[e] : __expf(ll[e]);
    }
    if (D.inplace && writer) {
#pragma unroll
        for (int v = 0; v < S; ++v) {
            float o[E];
#pragma unroll
            for (int e = 0; e < E; ++e) o[e] = st[e][v];
            stv<E>(D.state + v * T + base, o);
        }
    }
    float k[E];
    int ix[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        k[e] = okey[e];
        ix[e] = E * vt + e;
    }
    sort_subfilter<Mdl, M, E, TP>(k, ix, sk, si);
    if (writer) stv<E>(D.tkey + base, k);
    __syncthreads();  // normals consumed, sort buffers free: stage the state
    if (writer) {
#pragma unroll
        for (int v = 0; v < S; ++v)
#pragma unroll
            for (int e = 0; e < E; ++e) stage[v * M + E * vt + e] = st[e][v];
    }
    if (tid == 0) {
        D.winner[b] = k[0];
        s_lmax = k[0];
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < S; ++v) {
        if (v % TP != h) continue;  // a pair's lanes gather alternate variables
        float o[E];
#pragma unroll
        for (int e = 0; e < E; ++e) o[e] = stage[v * M + ix[e]];
        stv<E>(D.tmp + v * T + base, o);
    }
    write_partials<Mdl, E, NT, k1_stage_bytes<Mdl, M, FR, TP>()>(D, b, D.log_weights ? s_lmax : 0.0f, okey, st, sn,
                                                                  cs, reinterpret_cast<double*>(stage), writer);
}

// ---------------------------------------------------------------------------
// Phased pipeline: propagate + weight only (sampling_importance,
// pf_generic_soa.cu:245-287): state in place, unsorted keys.
// ---------------------------------------------------------------------------
template <class Mdl, int M, int E>
__global__ void __launch_bounds__(M / E) k_sample_weight(const FilterDesc* __restrict__ descs,
                                                         const int2* __restrict__ cta_map, InputRef in)
{
    constexpr int S = Mdl::S, K = Mdl::K, NA = Mdl::NA;
    constexpr int NANG = NA > 0 ? NA : 1;
    __shared__ typename Mdl::Consts cst;
    __shared__ FilterDesc sdesc;
    int f, b;
    cta_target(cta_map, f, b);
    const FilterDesc& D = load_desc(sdesc, descs + f);
    const int tid = threadIdx.x;
    const int64_t T = D.T;
    const int64_t base = (int64_t)b * M + E * tid;
    if (tid < 32) Mdl::prepare(cst, *input_of(in, f), D.mp, tid);
    __syncthreads();
    float st[E][S];
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
        ldv<E>(D.state + v * T + base, o);
#pragma unroll
        for (int e = 0; e < E; ++e) st[e][v] = o[e];
    }
    float key[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        float n[K], sn[NANG], cs[NANG];
#pragma unroll
        for (int v = 0; v < K; ++v) n[v] = D.rbuf[v * T + base + e];
        const float ll = Mdl::step(cst, st[e], n, sn, cs);
        key[e] = D.log_weights ? ll : __expf(ll);
    }
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
#pragma unroll
        for (int e = 0; e < E; ++e) o[e] = st[e][v];
        stv<E>(D.state + v * T + base, o);
    }
    stv<E>(D.key + base, key);
}

// Phased pipeline: block_sort (pf_generic_soa.cu:289-323) + estimate partials.
template <class Mdl, int M, int E>
__global__ void __launch_bounds__(M / E) k_block_sort(const FilterDesc* __restrict__ descs,
                                                      const int2* __restrict__ cta_map)
{
    constexpr int NT = M / E, S = Mdl::S, NA = Mdl::NA;
    constexpr int NANG = NA > 0 ? NA : 1;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float s_lmax;
    __shared__ FilterDesc sdesc;
    int f, b;
    cta_target(cta_map, f, b);
    const FilterDesc& D = load_desc(sdesc, descs + f);
    const int tid = threadIdx.x;
    const int64_t T = D.T;
    const int64_t base = (int64_t)b * M + E * tid;
    float* stage = reinterpret_cast<float*>(smem);
    float* sk = stage + (size_t)S * M;
    int* si = reinterpret_cast<int*>(sk + M);
    float st[E][S], okey[E], sn[E][NANG], cs[E][NANG];
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
        ldv<E>(D.state + v * T + base, o);
#pragma unroll
        for (int e = 0; e < E; ++e) st[e][v] = o[e];
    }
    ldv<E>(D.key + base, okey);
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
        for (int a = 0; a < NA; ++a) __sincosf(st[e][Mdl::angle_var(a)], &sn[e][a], &cs[e][a]);
    float k[E];
    int ix[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        k[e] = okey[e];
        ix[e] = E * tid + e;
    }
    bitonic_sort_desc<M, E>(k, ix, sk, si);
    stv<E>(D.tkey + base, k);
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
        stv<E>(D.tmp + v * T + base, o);
    }
    write_partials<Mdl, E, NT, (size_t)S * M * 4>(D, b, D.log_weights ? s_lmax : 0.0f, okey, st, sn, cs,
                                                   reinterpret_cast<double*>(stage));
}

// ---------------------------------------------------------------------------
// Exchange routing: the global slot (within the filter) that receiving slot
// M-1-x of sub-filter b takes, x < t (ring, all-to-all) or x < 4t (torus).
// ring: exchange_ring (pf_generic_soa.cu:400-413); torus: exchange_2dtorus
// (pf_generic.cu:352-393) with receiver slots m-1-j-k*t, k = sender's
// direction L,R,T,B; all-to-all: pf_generic2_all2all.cu:404-419.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t exchange_source(const FilterDesc& D, int b, int x)
{
    const int M = D.M, N = D.N, t = D.t;
    if (D.exchange == PF_EXCHANGE_RING) return (int64_t)(b == 0 ? N - 1 : b - 1) * M + x;
    if (D.exchange == PF_EXCHANGE_ALL2ALL) return D.a2a[x];
    // the torus width dx is a power of two: shifts and masks, no divisions
    const int k = x >= 2 * t ? (x >= 3 * t ? 3 : 2) : (x >= t ? 1 : 0);
    const int j = x - k * t;
    const int dx = D.dx, dy = D.shard ? D.gdy : D.dy;
    const int sh = __ffs(dx) - 1, mk = dx - 1;
    const int bg = b + D.b0;
    const int cx = bg & mk, cy = bg >> sh;
    int from;
    if (k == 0) from = (cy << sh) + ((cx + 1) & mk);            // right neighbour sent "left"
    else if (k == 1) from = (cy << sh) + ((cx - 1) & mk);       // left neighbour sent "right"
    else if (k == 2) from = ((cy + 1 == dy ? 0 : cy + 1) << sh) + cx;  // bottom neighbour sent "top"
    else from = ((cy == 0 ? dy - 1 : cy - 1) << sh) + cx;       // top neighbour sent "bottom"
    if (D.shard) {
        // a row of this shard, or the halo row above (block 0) / below (block 1):
        // halo slots are returned as -(1 + index into a block's rows)
        const int fy = from >> sh, fx = from & mk, rows = N >> sh;
        int ry = fy - D.r0;
        if (ry < 0) ry += dy;
        if (ry < rows) return (int64_t)(from - D.b0) * M + j;
        const int h = ry == dy - 1 ? 0 : 1;
        return -(1 + ((int64_t)(h * dx + fx) * t + j));
    }
    return (int64_t)from * M + j;
}

// The sorted key and state of exchange source g (exchange_source): this
// filter's sorted copy, or a shard's halo block.
template <int S>
__device__ __forceinline__ void exchange_fetch(const FilterDesc& D, const float* __restrict__ src_key,
                                               const float* __restrict__ src_tmp, int64_t T, int64_t g, float& key,
                                               float (&v)[S])
{
    if (g >= 0) {
        key = src_key[g];
#pragma unroll
        for (int s = 0; s < S; ++s) v[s] = src_tmp[s * T + g];
    } else {
        const int64_t i = -(g + 1);  // (h dx + x) t + j
        const int P = D.dx * D.t;
        const int h = (int)(i / P);
        const float* blk = D.halo + (int64_t)h * (1 + S) * P;
        const int64_t o = i - (int64_t)h * P;
        key = blk[o];
#pragma unroll
        for (int s = 0; s < S; ++s) v[s] = blk[(int64_t)(1 + s) * P + o];
    }
}

__device__ __forceinline__ int exchange_count(const FilterDesc& D)
{
    if (D.exchange == PF_EXCHANGE_NONE || D.t <= 0) return 0;
    return D.exchange == PF_EXCHANGE_TORUS ? 4 * D.t : D.t;
}

// Phased pipeline: copy the exchanged particles into the receivers' weakest
// slots of tmp/tkey (reads slots [0,t), writes [M-4t, M): disjoint by the
// create-time constraint, so the in-place copy equals the out-of-place one).
template <int S>
__global__ void k_exchange_inplace(const FilterDesc* __restrict__ descs, const int2* __restrict__ cta_map)
{
    int f, b;
    cta_target(cta_map, f, b);
    const FilterDesc& D = descs[f];
    const int nx = exchange_count(D);
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        const int64_t d = (int64_t)b * D.M + D.M - 1 - x;
        float kk, v[S];
        exchange_fetch<S>(D, D.tkey, D.tmp, D.T, exchange_source(D, b, x), kk, v);
        D.tkey[d] = kk;
#pragma unroll
        for (int s = 0; s < S; ++s) D.tmp[s * D.T + d] = v[s];
    }
}

// ---------------------------------------------------------------------------
// One warp: the sum over rows r < nr (<= 32) of sc_r * rows[r * kPartStride
// + j] for every value j < NV (sc_r held by lane r), returned in lane j.  P =
// 4, 2 or 1 lanes per value (as many as fit 32 / NV): lane (q, j) adds rows
// q, q + P, q + 2P, ... in that order, loading them eight at a time (all of
// them independent loads of contiguous rows), then an xor tree over the P
// lanes.  A fixed order for a given NV.
__device__ __forceinline__ double weighted_rows(const double* __restrict__ rows, int nr, double sc, int NV, int lane)
{
    const int P = NV <= 8 ? 4 : (NV <= 16 ? 2 : 1);
    const int W = 32 / P, j = lane & (W - 1), q = lane / W;
    const bool on = j < NV;
    double a = 0.0;
    for (int k0 = 0; k0 < W; k0 += 8) {
        double v[8], w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int r = q + P * (k0 + i);
            w[i] = __shfl_sync(kFull, sc, r & 31);
            v[i] = (on && r < nr) ? __ldcg(rows + (int64_t)r * kPartStride + j) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) a += w[i] * v[i];
    }
    for (int o = W; o < 32; o <<= 1) a += __shfl_xor_sync(kFull, a, o);
    return a;
}

// The same sums in the same order for rows of more than 8 values, loaded
// sixteen at a time, the first batch issued before scale() -- which computes
// lane r's factor sc_r and whose own loads and reductions then overlap the
// rows in flight (rows of up to 8 values keep weighted_rows: their kernels'
// registers hold no more).
template <class Scale>
__device__ __forceinline__ double weighted_rows_late(const double* __restrict__ rows, int nr, int NV, int lane,
                                                     Scale scale)
{
    constexpr int B = 16;
    const int P = NV <= 8 ? 4 : (NV <= 16 ? 2 : 1);
    const int W = 32 / P, j = lane & (W - 1), q = lane / W;
    const bool on = j < NV;
    double a = 0.0, sc = 0.0;
    for (int k0 = 0; k0 < W; k0 += B) {
        double v[B];
#pragma unroll
        for (int i = 0; i < B; ++i) {
            const int r = q + P * (k0 + i);
            v[i] = (k0 + i < W && on && r < nr) ? __ldcg(rows + (int64_t)r * kPartStride + j) : 0.0;
        }
        if (k0 == 0) sc = scale();
#pragma unroll
        for (int i = 0; i < B; ++i) {
            if (k0 + i < W) {  // warp-uniform
                const double w = __shfl_sync(kFull, sc, (q + P * (k0 + i)) & 31);
                a += w * v[i];
            }
        }
    }
    for (int o = W; o < 32; o <<= 1) a += __shfl_xor_sync(kFull, a, o);
    return a;
}

// E consecutive floats global -> shared without passing through registers
// (cp.async; both addresses aligned to 4E bytes).  cp_async_wait() waits for
// this thread's copies.
template <int E>
__device__ __forceinline__ void cp_async_floats(float* dst, const float* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (E % 4 == 0) {
#pragma unroll
        for (int q = 0; q < E; q += 4)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d + 4 * q), "l"(src + q) : "memory");
    } else if constexpr (E == 2) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    } else {
#pragma unroll
        for (int q = 0; q < E; ++q)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d + 4 * q), "l"(src + q) : "memory");
    }
}

__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Rows r < nr of `src` (kPartStride doubles apart, 16-byte aligned), their
// first nv (<= 32) values, into stage[r * rs + j], rs = nv rounded up to even:
// one warp's cp.async copies of value pairs (16 bytes, through L2 only), lane
// (q, p) copying pair p of rows q, q + 32 / W, ... (W the power of two >= the
// pairs per row).  The caller waits (cp_async_wait + __syncwarp).
__device__ __forceinline__ int staged_stride(int nv) { return (nv + 1) & ~1; }
__device__ __forceinline__ void stage_rows(double* stage, const double* __restrict__ src, int nr, int nv, int lane)
{
    const int np = (nv + 1) >> 1, rs = 2 * np;
    const int sh = np <= 4 ? 2 : (np <= 8 ? 3 : 4);
    const int pr = lane & ((1 << sh) - 1);
    if (pr >= np) return;
    for (int r = lane >> sh; r < nr; r += 32 >> sh) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(stage + r * rs + 2 * pr);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d),
                     "l"(src + (int64_t)r * kPartStride + 2 * pr)
                     : "memory");
    }
}

// weighted_rows over rows staged in shared memory (row r's value j at
// rows[r * rs + j]): the same products added in the same order.
__device__ __forceinline__ double weighted_rows_staged(const double* rows, int rs, int nr, double sc, int NV, int lane)
{
    const int P = NV <= 8 ? 4 : (NV <= 16 ? 2 : 1);
    const int W = 32 / P, j = lane & (W - 1), q = lane / W;
    const bool on = j < NV;
    double a = 0.0;
    for (int k = 0; k < W; ++k) {
        const int r = q + P * k;
        const double w = __shfl_sync(kFull, sc, r & 31);
        const double v = (on && r < nr) ? rows[r * rs + j] : 0.0;
        a += w * v;
    }
    for (int o = W; o < 32; o <<= 1) a += __shfl_xor_sync(kFull, a, o);
    return a;
}

// A group's row from its nr (<= 32) sub-filters' partial rows, one warp:
// [0] the group's key maximum, [1 .. NV) the sums scaled to it, [NV] the
// first-maximum winner's key, [NV + 1] its index (idx0 + the sub-filter).
// STAGED (`stage`: 32 rows of NV values in shared memory, `part` 16-byte
// aligned): every row arrives in one round of copies before the maximum and
// the sums; otherwise the maximum's values load first and the rows after.
// The same result either way.
template <int S, bool STAGED = false>
__device__ __forceinline__ void group_row(const FilterDesc& D, const double* __restrict__ part,
                                          const float* __restrict__ winner, int nr, int NV, int idx0, int lane,
                                          double* __restrict__ go, double* stage = nullptr)
{
    const bool valid = lane < nr;
    if constexpr (STAGED) stage_rows(stage, part, nr, NV, lane);
    const float lw = valid ? __ldcg(winner + lane) : -INFINITY;
    double l;
    if constexpr (STAGED) {
        cp_async_wait();
        __syncwarp();
        l = valid ? stage[lane * staged_stride(NV)] : -INFINITY;
    } else {
        l = valid ? __ldcg(part + (int64_t)lane * kPartStride) : -INFINITY;
    }
    double gl = l;
    float wk = lw;
    int wi = valid ? lane : 0x7fffffff;
    auto reduce = [&] {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            gl = fmax(gl, __shfl_xor_sync(kFull, gl, o));
            const float ok = __shfl_xor_sync(kFull, wk, o);
            const int oi = __shfl_xor_sync(kFull, wi, o);
            if (ok > wk || (ok == wk && oi < wi)) {
                wk = ok;
                wi = oi;
            }
        }
        return valid ? (D.log_weights ? exp(l - gl) : 1.0) : 0.0;
    };
    double a;
    if constexpr (STAGED) {
        a = weighted_rows_staged(stage, staged_stride(NV), nr, reduce(), NV, lane);
    } else if constexpr (2 + 2 * S <= 8) {
        a = weighted_rows(part, nr, reduce(), NV, lane);
    } else {
        a = weighted_rows_late(part, nr, NV, lane, reduce);
    }
    if (lane >= 1 && lane < NV) go[lane] = a;
    if (lane == 0) {
        go[0] = D.log_weights ? gl : 0.0;
        go[NV] = (double)wk;
        go[NV + 1] = (double)(wi + idx0);
    }
}

// Global winner (first maximum, thrust::max_element semantics,
// pf_generic_soa.cu:1014-1017) + FP64 posterior mean, reduced in two fixed-order
// levels inside the resampling kernel: warp 0 of the CTA of sub-filter 32g
// combines sub-filters 32g..32g+31 (all partials are final when that kernel
// starts); the last group to finish (atomic ticket) combines the groups in
// index order and writes the estimate.  Deterministic for a given N.
// ---------------------------------------------------------------------------
// The estimate's fields from the sums `acc` (lane j < NV holds sum j), one
// warp at once -- lane v the mean (or circular mean) of variable v, lane 16 +
// v the winner's variable v (best_v), lane 0 the rest.
template <int S>
__device__ __forceinline__ void estimate_store(const FilterDesc& D, int lane, int NV, double gm, float bk, int best,
                                               float best_v, double acc, pf_estimate& E, int32_t step_no)
{
    __shared__ double s_acc[2 + 2 * PF_MAX_STATE];
    if (lane >= 1 && lane < NV) s_acc[lane] = acc;
    __syncwarp();
    const double W = s_acc[1];
    if (lane < PF_MAX_STATE) {
        const int v = lane;
        double m = 0.0;
        if (v < S) {
            if ((D.angle_mask >> v) & 1u) {
                const int a = __popc(D.angle_mask & ((1u << v) - 1u));
                m = atan2(s_acc[2 + v], s_acc[2 + S + a]);
            } else {
                m = s_acc[2 + v] / W;
            }
        }
        E.mean[v] = m;
    } else {
        E.best[lane - PF_MAX_STATE] = best_v;
    }
    if (lane == 0) {
        const double lg = D.log_weights ? gm : 0.0;
        E.log_norm = lg + log(W);
        E.best_key = bk;
        E.best_subfilter = best;
        E.step = step_no;
        E.flags = (isfinite(lg) && isfinite(W) && W > 0.0) ? 0 : 1;
    }
    __syncwarp();
}

// The global estimate from the group partials gpart[0..ng) (one warp, after
// the global maximum gm and the winner (bk, bi) are known): the FP64 sums of
// the NV values, then estimate_store with the winner's state from best_src.
// Each sum keeps one order: the groups ascending in chunks of 32, the
// chunks' sums in order.
template <int S>
__device__ __forceinline__ void estimate_write(const FilterDesc& D, int lane, int ng, int NV, double gm, float bk,
                                               int bi, const float* __restrict__ best_src, pf_estimate& E,
                                               int32_t step_no)
{
    const int best = (bi >= 0 && bi < D.N) ? bi : 0;  // NaN keys everywhere: report sub-filter 0
    // the winner's state first: its load overlaps the sums
    const int bv = lane - PF_MAX_STATE;
    const float best_v = (bv >= 0 && bv < S) ? __ldcg(best_src + bv * D.T + (int64_t)best * D.M) : 0.0f;
    // lane j sums value j over the groups, 32 rows at a time (weighted_rows)
    double acc = 0.0;
    for (int c = 0; c < ng; c += 32) {
        const int nr = min(32, ng - c);
        const double* rows = D.gpart + (int64_t)c * kPartStride;
        const double l = lane < nr ? __ldcg(rows + (int64_t)lane * kPartStride) : 0.0;
        auto scale = [&] { return lane < nr ? (D.log_weights ? exp(l - gm) : 1.0) : 0.0; };
        if constexpr (2 + 2 * S <= 8) {
            acc += weighted_rows(rows, nr, scale(), NV, lane);
        } else {
            acc += weighted_rows_late(rows, nr, NV, lane, scale);
        }
    }
    estimate_store<S>(D, lane, NV, gm, bk, best, best_v, acc, E, step_no);
}

// The winner and the maximum: lane q's own rows in ascending order, then an
// xor tree (first maximum, lowest index on ties).
__device__ __forceinline__ void winner_merge(double& gm, float& bk, int& bi, double g0, double gk, double gi)
{
    gm = fmax(gm, g0);
    const float k = (float)gk;
    const int i = (int)gi;
    if (k > bk || (k == bk && i < bi)) {
        bk = k;
        bi = i;
    }
}
__device__ __forceinline__ void winner_tree(double& gm, float& bk, int& bi)
{
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
}

// The global estimate from the group partial rows gpart[0..ng) (one warp): the
// global maximum, the first-maximum winner, then estimate_write (whose winner
// state is read at best_src + v T + winner M).
template <int S>
__device__ __forceinline__ void estimate_final(const FilterDesc& D, int lane, int ng, int NV,
                                               const float* __restrict__ best_src, pf_estimate& E, int32_t step_no)
{
    double gm = -INFINITY;
    float bk = -INFINITY;
    int bi = 0x7fffffff;
#pragma unroll 2
    for (int q = lane; q < ng; q += 32) {
        const double* gq = D.gpart + (int64_t)q * kPartStride;
        winner_merge(gm, bk, bi, __ldcg(gq), __ldcg(gq + NV), __ldcg(gq + NV + 1));
    }
    winner_tree(gm, bk, bi);
    estimate_write<S>(D, lane, ng, NV, gm, bk, bi, best_src, E, step_no);
}

// estimate_final with the group rows staged in shared memory (`stage`: wr
// rows of NV + 2 values, wr a multiple of 32; gpart 16-byte aligned): the
// rows arrive in windows of wr, one round of copies each -- a single window,
// copied once, for ng <= wr -- and give the same maximum, winner and sums in
// the same order.
template <int S>
__device__ __forceinline__ void estimate_final_staged(const FilterDesc& D, int lane, int ng, int NV,
                                                      const float* __restrict__ best_src, pf_estimate& E,
                                                      int32_t step_no, double* stage, int wr)
{
    const int rs = staged_stride(NV + 2);
    auto load_window = [&](int w0) {
        __syncwarp();  // the previous window's reads are done
        stage_rows(stage, D.gpart + (int64_t)w0 * kPartStride, min(wr, ng - w0), NV + 2, lane);
        cp_async_wait();
        __syncwarp();
    };
    double gm = -INFINITY;
    float bk = -INFINITY;
    int bi = 0x7fffffff;
    for (int w0 = 0; w0 < ng; w0 += wr) {
        load_window(w0);
        const int nr = min(wr, ng - w0);
        for (int q = lane; q < nr; q += 32) {
            const double* sq = stage + q * rs;
            winner_merge(gm, bk, bi, sq[0], sq[NV], sq[NV + 1]);
        }
    }
    winner_tree(gm, bk, bi);
    const int best = (bi >= 0 && bi < D.N) ? bi : 0;  // NaN keys everywhere: report sub-filter 0
    const int bv = lane - PF_MAX_STATE;
    const float best_v = (bv >= 0 && bv < S) ? __ldcg(best_src + bv * D.T + (int64_t)best * D.M) : 0.0f;
    double acc = 0.0;
    for (int w0 = 0; w0 < ng; w0 += wr) {
        if (ng > wr) load_window(w0);
        const int nw = min(wr, ng - w0);
        for (int c = 0; c < nw; c += 32) {
            const int nr = min(32, nw - c);
            const double* sr = stage + c * rs;
            const double l = lane < nr ? sr[lane * rs] : 0.0;
            acc += weighted_rows_staged(sr, rs, nr, lane < nr ? (D.log_weights ? exp(l - gm) : 1.0) : 0.0, NV, lane);
        }
    }
    estimate_store<S>(D, lane, NV, gm, bk, best, best_v, acc, E, step_no);
}

// Group g's estimate row from its 32 sub-filters' partial rows (one warp);
// the last group to finish (ticket) combines every group row into the
// filter's estimate.  With CAP >= 32 kPartStride doubles of the kernel's
// shared memory at `smem` (the partial rows are 256-byte aligned in every
// allocation of this library) both levels read their rows staged there.
template <int S, int CAP>
__device__ __forceinline__ void estimate_group(const FilterDesc& D, int g, const InputRef& in, int32_t* step_ctr,
                                               double* smem)
{
    constexpr bool STAGED = CAP >= 32 * kPartStride;
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const int b = g << 5, ng = (D.N + 31) >> 5;
    const int NV = 2 + S + D.na;
    // winners as filter-wide indices (a shard's sub-filters start at b0)
    group_row<S, STAGED>(D, D.part + (int64_t)b * kPartStride, D.winner + b, min(32, D.N - b), NV, b + D.b0, lane,
                         D.gpart + (int64_t)g * kPartStride, smem);
    if (D.shard) return;  // the shards' group rows are combined across shards (pf_shard_estimate)
    __syncwarp();
    __threadfence();
    int last = 0;
    if (lane == 0) last = atomicAdd(D.est_ctr, 1) == ng - 1;
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    const int32_t step_no = in.ctr ? *in.ctr + 1 : 0;
    if constexpr (STAGED) {
        const int wr = (CAP / staged_stride(NV + 2)) & ~31;
        estimate_final_staged<S>(D, lane, ng, NV, D.tmp, D.est[step_index(in)], step_no, smem, wr);
    } else {
        estimate_final<S>(D, lane, ng, NV, D.tmp, D.est[step_index(in)], step_no);
    }
    if (lane == 0) {
        *D.est_ctr = 0;
        __threadfence();
        if (step_ctr) *step_ctr += 1;
    }
}

// ---------------------------------------------------------------------------
// Exchange + resample + gather, one CTA per sub-filter.  `virt`: apply the
// exchange virtually (read the neighbours' slots straight from tmp).
// Resampling restates resampling (pf_generic_soa.cu:415-453) for
// PF_RESAMPLE_REFERENCE, resampling_valias (resampling-valias.cl:214-300)
// for PF_RESAMPLE_VOSE; PF_RESAMPLE_SYSTEMATIC uses the FP64 scan.
// ---------------------------------------------------------------------------
template <int S, int M, int E, int RES>
constexpr size_t k2_smem()
{
    size_t s = (size_t)M * 4 + (size_t)S * M * 4;  // keys + state tile
    if (RES == PF_RESAMPLE_SYSTEMATIC) s += 0;       // the scan stays in registers, the runs reuse the keys
    else if (RES == PF_RESAMPLE_REFERENCE) s += (size_t)M * 4;
    else s += (size_t)M * 16;  // prob, alias, work list, scratch
    return s;
}

// Bulk copies global -> shared through the TMA engine (cp.async.bulk, no
// multicast), completion counted in bytes on a shared-memory mbarrier.  Both
// addresses 16-byte aligned, sizes multiples of 16.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init_expect(uint64_t* mbar, unsigned bytes)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n"
                 "fence.mbarrier_init.release.cluster;\n"
                 "fence.proxy.async.shared::cta;\n"
                 "fence.proxy.async.global;\n"
                 "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mbar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(mbar))
                 : "memory");
}

// Waits for phase `parity` of the mbarrier, at most `limit` polls (each
// try_wait may suspend the thread for a while); false when they ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, unsigned parity, int limit = 1 << 18)
{
    const unsigned a = smem_u32(mbar);
    for (int i = 0; i < limit; ++i) {
        unsigned done;
        asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// CTA-wide bounded wait for the bulk copies counted on `mbar`.  Each thread
// polls at most limits[0] times, then the CTA agrees (__syncthreads_and), so
// every thread takes the same branch even when only some of them ran out.  If
// any gave up, every thread waits again, at most limits[1] polls, for the
// copies still in flight, so that none is writing this CTA's shared memory
// when the CTA moves on to reuse it or exits.  Returns 1 when the copies landed
// within the first wait, 0 when they landed only in the second (the caller
// reports the timeout; shared memory is quiet), -1 when they may still be in
// flight (the caller must not touch the destination again).  Every thread of
// the CTA must call it.
__device__ __forceinline__ int mbar_wait_cta(uint64_t* mbar, unsigned parity, int limit, int drain_limit)
{
    if (__syncthreads_and(mbar_wait(mbar, parity, limit))) return 1;
    return __syncthreads_and(mbar_wait(mbar, parity, drain_limit)) ? 0 : -1;
}
constexpr int kBulkWaitPolls = 1 << 18;
constexpr int kBulkDrainPolls = 1 << 18;

// Resampling of sub-filter b from a sorted copy (src_tmp, src_key: this
// filter's arrays, sorted per sub-filter) with the exchange applied virtually
// (nx weakest slots take the neighbours' top-t, read from the same sorted
// copy).  U: the sub-filter's uniforms (decision first).  Returns PF_RS_KEPT
// when the decision uniform exceeds resampling_freq or the ESS gate holds (the
// sub-filter keeps its propagated particles), PF_RS_RESAMPLED with st holding
// this thread's E resampled particles (positions E*tid+e) and sel their source
// slots, or -- with a status bit set -- PF_RS_KEPT (rows not 16-byte aligned,
// or a wait that ran out before the copies landed) or PF_RS_LOST (the copies
// may still be landing in smem).  The result is the same in every thread.
// Every thread of the CTA must call it (it synchronises the CTA).  Restates resampling
// (pf_generic_soa.cu:415-453) for PF_RESAMPLE_REFERENCE and resampling_valias
// (resampling-valias.cl:214-300) for PF_RESAMPLE_VOSE; PF_RESAMPLE_SYSTEMATIC
// uses the FP64 scan.
template <int S, int M, int E, int RES>
__device__ __forceinline__ int resample_from(const FilterDesc& D, int b, const float* __restrict__ src_tmp,
                                              const float* __restrict__ src_key, const float* __restrict__ U,
                                              int nx, unsigned char* smem, double* dred, int* ired,
                                              uint64_t* mbar, float (&st)[E][S], int (&sel)[E])
{
    const int tid = threadIdx.x;
    const int64_t T = D.T;
    const int64_t base = (int64_t)b * M + E * tid;
    // Every global read is issued before the first barrier: the decision and
    // resampling uniforms, the sorted keys and state of this sub-filter, and --
    // for the slots in the exchange range -- the neighbours' top-t (the slot's
    // owner loads them, so each shared-memory slot has one writer).
    const float dec_u = D.rng_fused ? U[0] : U[T + b];
    float ur[RES == PF_RESAMPLE_VOSE ? 2 * E : E];
    if constexpr (RES == PF_RESAMPLE_SYSTEMATIC) {
        ur[0] = D.rng_fused ? U[1] : U[(int64_t)b * M];
    } else if constexpr (RES == PF_RESAMPLE_REFERENCE) {
#pragma unroll
        for (int e = 0; e < E; ++e) ur[e] = D.rng_fused ? U[1 + E * tid + e] : U[(int64_t)b * M + E * tid + e];
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int64_t i = E * tid + e;
            ur[2 * e] = D.rng_fused ? U[1 + 2 * i] : U[2 * ((int64_t)b * M + i)];
            ur[2 * e + 1] = D.rng_fused ? U[2 + 2 * i] : U[2 * ((int64_t)b * M + i) + 1];
        }
    }
    float* kb = reinterpret_cast<float*>(smem);
    float* tile = kb + M;
    unsigned char* scratch = reinterpret_cast<unsigned char*>(tile + (size_t)S * M);
    const bool xch = E * tid + E - 1 >= M - nx;  // this thread owns slots in the exchange range
    if constexpr (S <= 3) {
        // Small states: the sub-filter's sorted keys and state rows by bulk
        // copies (one thread issues them), the exchanged slots patched by
        // their owners once the rows landed.  (The arm's 13 rows ran slower as
        // bulk copies issued by one thread than as per-thread cp.async:
        // resampling kernel 34.4 vs 26.0 us at 2^18 particles.)
        const bool bulk = ((reinterpret_cast<uintptr_t>(src_key) | reinterpret_cast<uintptr_t>(src_tmp) |
                            (uintptr_t)(T * 4)) & 15) == 0;
        if (!bulk) {  // rows not 16-byte aligned: not this library's allocations (no copy issued)
            if (tid == 0 && D.status) atomicOr(D.status, PF_STATUS_MISALIGNED);
            return PF_RS_KEPT;
        }
        if (tid == 0) {
            mbar_init_expect(mbar, (unsigned)((1 + S) * M * 4));
            bulk_g2s(kb, src_key + (int64_t)b * M, M * 4, mbar);
#pragma unroll
            for (int v = 0; v < S; ++v) bulk_g2s(tile + v * M, src_tmp + v * T + (int64_t)b * M, M * 4, mbar);
        }
        // the neighbours' values into registers while the rows are in flight
        float xk[E], xs[E][S];
        if (xch) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int x = M - 1 - (E * tid + e);
                if (x < nx) exchange_fetch<S>(D, src_key, src_tmp, T, exchange_source(D, b, x), xk[e], xs[e]);
            }
        }
        __syncthreads();  // the mbarrier is initialised
        const int landed = mbar_wait_cta(mbar, 0, kBulkWaitPolls, kBulkDrainPolls);
        if (landed <= 0) {
            if (tid == 0 && D.status) atomicOr(D.status, PF_STATUS_WAIT_TIMEOUT);
            return landed < 0 ? PF_RS_LOST : PF_RS_KEPT;
        }
        if (dec_u - 1.0f > D.freq) return PF_RS_KEPT;
        if (xch) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int x = M - 1 - (E * tid + e);
                if (x < nx) {
                    kb[E * tid + e] = xk[e];
#pragma unroll
                    for (int v = 0; v < S; ++v) tile[v * M + E * tid + e] = xs[e][v];
                }
            }
        }
    } else {
        // large states: straight into shared memory (cp.async).  A thread
        // owning exchanged slots copies slot by slot, each from its source --
        // its own row, a neighbour's sorted copy or a shard's halo block -- so
        // the neighbours' values arrive with the rows, in one round trip
        if (!xch) {
            cp_async_floats<E>(kb + E * tid, src_key + base);
#pragma unroll
            for (int v = 0; v < S; ++v) cp_async_floats<E>(tile + v * M + E * tid, src_tmp + v * T + base);
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int x = M - 1 - (E * tid + e);
                const float* ks = src_key + base + e;
                const float* vs = src_tmp + base + e;
                int64_t vstride = T;
                if (x < nx) {
                    const int64_t g = exchange_source(D, b, x);
                    if (g >= 0) {
                        ks = src_key + g;
                        vs = src_tmp + g;
                    } else {  // a shard's halo block: key row, then the state rows
                        const int64_t i = -(g + 1);
                        const int P = D.dx * D.t;
                        const int h = (int)(i / P);
                        const float* blk = D.halo + (int64_t)h * (1 + S) * P + (i - (int64_t)h * P);
                        ks = blk;
                        vs = blk + P;
                        vstride = P;
                    }
                }
                cp_async_floats<1>(kb + E * tid + e, ks);
#pragma unroll
                for (int v = 0; v < S; ++v) cp_async_floats<1>(tile + v * M + E * tid + e, vs + v * vstride);
            }
        }
        cp_async_wait();
        if (dec_u - 1.0f > D.freq) return PF_RS_KEPT;
    }
    // this thread's own slots (copied, or patched by this thread) are readable
    // already; the barrier orders every slot's patch before the reads below
    float w[E];
    bool nan = false;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        w[e] = kb[E * tid + e];
        nan |= w[e] != w[e];
    }
    const bool any_nan = __syncthreads_or(nan);
    if (D.log_weights) {
        // the keys are sorted per sub-filter, so their maximum is the head or one
        // of the weakest slots an exchange may have replaced (the same value as
        // the CTA-wide maximum); a NaN key breaks the order: then the CTA-wide one
        const int nxc = exchange_count(D);
        float mx;
        if (!any_nan && nxc <= 32 && nxc < M) {
            mx = kb[0];
            for (int x = 0; x < nxc; ++x) mx = fmaxf(mx, kb[M - 1 - x]);
        } else {
            mx = w[0];
#pragma unroll
            for (int e = 1; e < E; ++e) mx = fmaxf(mx, w[e]);
            mx = block_max(mx, reinterpret_cast<float*>(ired));
        }
#pragma unroll
        for (int e = 0; e < E; ++e) w[e] = pf_expneg(w[e] - mx);
    }
    if (D.ess_frac > 0.0f) {
        // effective sample size (sum w)^2 / sum w^2 in FP64; a sub-filter whose
        // weights are still spread out keeps its propagated particles
        static_assert(M / E <= 16 * 32, "two 16-warp partial arrays in dred");
        const int lane = tid & 31, wp = tid >> 5, nw = (M / E + 31) >> 5;
        double s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            s1 += (double)w[e];
            s2 += (double)w[e] * (double)w[e];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_xor_sync(kFull, s1, o);
            s2 += __shfl_xor_sync(kFull, s2, o);
        }
        if (lane == 0) {
            dred[wp] = s1;
            dred[16 + wp] = s2;
        }
        __syncthreads();
        double t1 = 0.0, t2 = 0.0;
        for (int q = 0; q < nw; ++q) {
            t1 += dred[q];
            t2 += dred[16 + q];
        }
        __syncthreads();
        // all-zero weights count as uniform (ESS = m): no resampling
        if (!(t2 > 0.0) || t1 * t1 >= (double)D.ess_frac * (double)M * t2) return PF_RS_KEPT;
    }
    if constexpr (RES == PF_RESAMPLE_SYSTEMATIC) {
        double cum[E], prev;
        const double tot = scan_f64<M, E>(w, cum, dred, &prev);
        // the keys were read into w before the scan's barriers: kb holds the output runs
        systematic_select<M, E>(cum, prev, ur[0] - 1.0f, tot / (double)M, reinterpret_cast<int*>(kb), sel);
    } else if constexpr (RES == PF_RESAMPLE_REFERENCE) {
        float* ex = reinterpret_cast<float*>(scratch);
#pragma unroll
        for (int e = 0; e < E; ++e) ex[E * tid + e] = w[e];
        const float tot = blelloch_scan<M>(ex);
#pragma unroll
        for (int e = 0; e < E; ++e) sel[e] = ref_binary_search(ex, (ur[e] - 1.0f) * tot, M);
    } else {
        float* prob = reinterpret_cast<float*>(scratch);
        unsigned* alias = reinterpret_cast<unsigned*>(prob + M);
        unsigned* sl = alias + M;
        float* scr = reinterpret_cast<float*>(sl + M);
        vose_build<M, E>(w, prob, alias, sl, scr, ired);
#pragma unroll
        for (int e = 0; e < E; ++e)
            sel[e] = (int)vose_draw<M>(prob, alias, ur[2 * e] - 1.0f, ur[2 * e + 1] - 1.0f);
    }
#pragma unroll
    for (int v = 0; v < S; ++v)
#pragma unroll
        for (int e = 0; e < E; ++e) st[e][v] = tile[v * M + sel[e]];
    return PF_RS_RESAMPLED;
}

template <int S, int M, int E, int RES>
__global__ void __launch_bounds__(M / E, pf_min_blocks(M / E, pf_k2_warps(S))) k_exchange_resample(const FilterDesc* __restrict__ descs,
                                                             const int2* __restrict__ cta_map, InputRef in,
                                                             int32_t* step_ctr, int virt)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double dred[64];
    __shared__ int ired[34];
    int f, b;
    if (cta_map) {
        const int2 c = cta_map[blockIdx.x];
        f = c.x;
        b = c.y;
    } else {
        f = 0;
        b = resample_cta(blockIdx.x, descs[0].N);
    }
    __shared__ FilterDesc sdesc;
    __shared__ uint64_t mbar;
    const FilterDesc& D = load_desc(sdesc, descs + f);
    const int tid = threadIdx.x;
    wait_prerequisites();
    if (b < 0) {
        constexpr int cap = (int)(k2_smem<S, M, E, RES>() / 8);  // doubles of dynamic shared memory
        estimate_group<S, cap>(D, -1 - b, in, step_ctr, reinterpret_cast<double*>(smem));
        return;
    }
    const int64_t T = D.T;
    const int64_t base = (int64_t)b * M + E * tid;
    const float* U = D.rng_fused ? D.ru + (int64_t)b * D.ru_stride : D.rbuf + D.nnorm;
    int nx = 0;
    if (virt) {
        nx = exchange_count(D);
        if (D.exch_period > 1 && (run_step(in) % D.exch_period) != 0) nx = 0;
    }
    float st[E][S];
    int sel[E];
    if (resample_from<S, M, E, RES>(D, b, D.tmp, D.tkey, U, nx, smem, dred, ired, &mbar, st, sel) != PF_RS_RESAMPLED) {
        if (D.sel) {
#pragma unroll
            for (int e = 0; e < E; ++e) D.sel[base + e] = -1;
        }
        return;  // the propagated state was written in place by the sampling kernel
    }
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
#pragma unroll
        for (int e = 0; e < E; ++e) o[e] = st[e][v];
        stv<E>(D.state + v * T + base, o);
    }
    if (D.sel) {
#pragma unroll
        for (int e = 0; e < E; ++e) D.sel[base + e] = sel[e];
    }
}

// ---------------------------------------------------------------------------
// Kernel-level test entry points (one CTA per sub-filter).
// ---------------------------------------------------------------------------
template <int M, int E, bool RANK>
__global__ void __launch_bounds__(M / E) k_test_sort(float* keys, int32_t* idx, int32_t* fallbacks)
{
    __shared__ float sk[M];
    __shared__ int si[M];
    const int64_t base = (int64_t)blockIdx.x * M + E * threadIdx.x;
    float k[E];
    int ix[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        k[e] = keys[base + e];
        ix[e] = E * threadIdx.x + e;
    }
    if constexpr (RANK) {
        const bool fell_back = rank_sort_desc<M, E>(k, ix, sk, si);
        if (fell_back && threadIdx.x == 0 && fallbacks) atomicAdd(fallbacks, 1);
    } else {
        bitonic_sort_desc<M, E>(k, ix, sk, si);
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
        keys[base + e] = k[e];
        idx[base + e] = ix[e];
    }
}

template <int M, int E, int RES>
__global__ void __launch_bounds__(M / E) k_test_resample(const float* w_in, const float* u, int32_t* sel_out,
                                                         float* prob_out, uint32_t* alias_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double dred[64];
    __shared__ int ired[34];
    const int b = blockIdx.x, tid = threadIdx.x;
    const int64_t base = (int64_t)b * M + E * tid;
    float w[E];
#pragma unroll
    for (int e = 0; e < E; ++e) w[e] = w_in[base + e];
    int sel[E];
    if constexpr (RES == PF_RESAMPLE_SYSTEMATIC) {
        double cum[E], prev;
        const double tot = scan_f64<M, E>(w, cum, dred, &prev);
        systematic_select<M, E>(cum, prev, u[b], tot / (double)M, reinterpret_cast<int*>(smem), sel);
    } else if constexpr (RES == PF_RESAMPLE_REFERENCE) {
        float* ex = reinterpret_cast<float*>(smem);
#pragma unroll
        for (int e = 0; e < E; ++e) ex[E * tid + e] = w[e];
        const float tot = blelloch_scan<M>(ex);
#pragma unroll
        for (int e = 0; e < E; ++e) sel[e] = ref_binary_search(ex, (u[base + e] - 1.0f) * tot, M);
    } else {
        float* prob = reinterpret_cast<float*>(smem);
        unsigned* alias = reinterpret_cast<unsigned*>(prob + M);
        unsigned* sl = alias + M;
        float* scr = reinterpret_cast<float*>(sl + M);
        vose_build<M, E>(w, prob, alias, sl, scr, ired);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int64_t i = base + e;
            sel[e] = (int)vose_draw<M>(prob, alias, u[2 * i], u[2 * i + 1]);
            if (prob_out) {
                prob_out[i] = prob[E * tid + e];
                alias_out[i] = alias[E * tid + e];
            }
        }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) sel_out[base + e] = sel[e];
}

template <class Mdl>
__global__ void k_test_model(ModelParams mp, const pf_step_input* in, int n, float* state, const float* noise,
                             float* ll)
{
    __shared__ typename Mdl::Consts cst;
    if (threadIdx.x < 32) Mdl::prepare(cst, *in, mp, threadIdx.x);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s[Mdl::S], z[Mdl::K], sn[Mdl::NA > 0 ? Mdl::NA : 1], cs[Mdl::NA > 0 ? Mdl::NA : 1];
    for (int v = 0; v < Mdl::S; ++v) s[v] = state[(int64_t)v * n + i];
    for (int v = 0; v < Mdl::K; ++v) z[v] = noise[(int64_t)v * n + i];
    ll[i] = Mdl::step(cst, s, z, sn, cs);
    for (int v = 0; v < Mdl::S; ++v) state[(int64_t)v * n + i] = s[v];
}

}  // namespace pfdev
