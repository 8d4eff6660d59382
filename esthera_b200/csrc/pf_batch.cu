// pf_batch.cu -- batched filters (include/esthera_b200.h, pf_batch_*): many
// independent filters of uneven particle counts stepped by one sequence of
// launches.  All filters share the model, the resampler and the exchange
// settings; each has its own particle count, model parameters, MTGP32
// streams, inputs and estimates.  The configured sub-filter size m is an upper
// bound: filter f runs sub-filters of m_f particles, the largest power of two
// <= m that divides its count (and, for the torus, gives a valid grid).
//
// One CTA per sub-filter of every filter: per sub-filter size, a CTA ->
// (filter, sub-filter) map drives the split pipeline's two kernels
// (k_sample_sort, k_exchange_resample) over that size's filters, the exchange
// stays inside each filter, and a run of many steps is captured once into a
// CUDA graph and replayed by one launch.
// Sub-filter b of filter f draws from stream stream_offset + first(f) + b,
// first(f) = the number of sub-filters of filters 0..f-1, so filter f alone
// (pf_create with that stream offset) reproduces its batched results exactly.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pf_host.cuh"

using namespace pfdev;
using namespace pfhost;

namespace {

// Fills every particle of filter f with init[f * S + v].
__global__ void k_batch_fill(const FilterDesc* __restrict__ descs, const int2* __restrict__ map,
                             const float* __restrict__ init, int S)
{
    int f, b;
    cta_target(map, f, b);
    if (b < 0) return;  // an estimate entry
    const FilterDesc& D = descs[f];
    for (int v = 0; v < S; ++v) {
        const float x = init[(int64_t)f * S + v];
        float* dst = D.state + v * D.T + (int64_t)b * D.M;
        for (int i = threadIdx.x; i < D.M; i += blockDim.x) dst[i] = x;
    }
}

constexpr int kMaxGraphSteps = 256;

}  // namespace

struct pf_batch {
    pf_config cfg;
    int model = 0;
    ModelInfo mi{};
    ModelOps ops{};
    int F = 0, M = 0, E = 0, S = 0, t = 0;  // M, E: the configured (largest) sub-filter size and its ppt
    int64_t P = 0;   // particles in all filters
    int NS = 0;      // sub-filters in all filters
    int map_len = 0;  // CTA-map entries: sub-filters and estimate CTAs
    std::vector<int32_t> nsub, sub_off, grp_off;  // grp_off: first estimate group (32 sub-filters) of a filter
    std::vector<int32_t> mf;                      // each filter's sub-filter size
    std::vector<int64_t> part_off, ru_off;
    struct Group {
        // one sub-filter size: ppt, threads per particle, sub-filters, estimate
        // CTAs (one per 32 sub-filters of each filter), first map entry
        int M, E, TP, NS, NE, map_off;
    };
    std::vector<Group> groups;
    std::vector<ModelParams> mp;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    int64_t dev_bytes = 0;
    float *state = nullptr, *tmp = nullptr, *tkey = nullptr, *winner = nullptr, *ru = nullptr;
    double *part = nullptr, *gpart = nullptr;
    uint32_t* mtgp = nullptr;
    int32_t *est_ctr = nullptr, *ctr = nullptr;
    int2* map = nullptr;
    FilterDesc* d_desc = nullptr;  // [0, F): pf_batch_step, [F, 2F): pf_batch_submit
    pf_step_input* d_in = nullptr;
    pf_estimate* d_est = nullptr;
    pf_step_input* h_in = nullptr;
    pf_estimate* h_est = nullptr;
    int32_t steps_done = 0;
    cudaGraphExec_t graph_n = nullptr, graph_1 = nullptr;
    int graph_steps = 0;
    const pf_step_input* graph_inputs = nullptr;
    pf_estimate* graph_est = nullptr;
    int32_t graph_cap = 0;
};

template <class T>
static pf_status balloc(pf_batch* B, T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) return PF_OK;
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PF_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", count * sizeof(T), cudaGetErrorString(e));
    }
    B->allocs.push_back(q);
    B->dev_bytes += (int64_t)(count * sizeof(T));
    *p = static_cast<T*>(q);
    return PF_OK;
}

static void drop_graphs(pf_batch* B)
{
    if (B->graph_n) cudaGraphExecDestroy(B->graph_n);
    if (B->graph_1) cudaGraphExecDestroy(B->graph_1);
    B->graph_n = B->graph_1 = nullptr;
    B->graph_steps = 0;
}

static void release(pf_batch* B)
{
    if (!B) return;
    drop_graphs(B);
    for (void* p : B->allocs) cudaFree(p);
    if (B->h_in) cudaFreeHost(B->h_in);
    if (B->h_est) cudaFreeHost(B->h_est);
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
}

static void fill_batch_desc(const pf_batch* B, int f, FilterDesc& D, pf_estimate* est)
{
    memset(&D, 0, sizeof(D));
    const int64_t p0 = B->part_off[f];
    const int64_t s0 = B->sub_off[f];
    const int N = B->nsub[f], M = B->mf[f];
    const int64_t nbm = 2 * (((int64_t)B->mi.K * M + 1) / 2);
    const int64_t draws = nbm + 1 + resample_draws(B->cfg.resampler, M);
    D.T = (int64_t)M * N;
    D.state = B->state + (int64_t)B->S * p0;
    D.tmp = B->tmp + (int64_t)B->S * p0;
    D.tkey = B->tkey + p0;
    D.winner = B->winner + s0;
    D.part = B->part + s0 * kPartStride;
    D.mtgp = B->mtgp + s0 * kMtgpN;
    D.ru = B->ru + B->ru_off[f];
    D.est = est;
    D.N = N;
    D.M = M;
    D.t = B->t;
    D.exchange = B->cfg.exchange;
    D.resampler = B->cfg.resampler;
    torus_dims(N, &D.dx, &D.dy);
    D.log_weights = B->cfg.log_weights ? 1 : 0;
    D.inplace = (B->cfg.resampling_freq < 1.0f || B->cfg.ess_fraction > 0.0f) ? 1 : 0;
    D.rng_fused = 1;
    D.draws = (int32_t)draws;
    D.nbm = (int32_t)nbm;
    D.ru_stride = (int32_t)(draws - nbm);
    D.mask = B->cfg.mtgp_mask;
    D.stream_base = B->cfg.stream_offset + (int32_t)s0;
    D.exch_period = B->cfg.exchange_period;
    D.freq = B->cfg.resampling_freq;
    D.ess_frac = B->cfg.ess_fraction;
    D.nnorm = (int64_t)B->mi.K * D.T;
    D.est_ctr = B->est_ctr + f;
    D.status = reinterpret_cast<int32_t*>(B->d_est + B->F);
    D.gpart = B->gpart + (int64_t)B->grp_off[f] * kPartStride;
    D.angle_mask = angle_mask_of(B->model);
    D.na = angle_count_of(B->model);
    D.mp = B->mp[f];
}

static pf_status upload_batch_descs(pf_batch* B, pf_estimate* run_est, int32_t cap)
{
    std::vector<FilterDesc> d(2 * (size_t)B->F);
    for (int f = 0; f < B->F; ++f) {
        fill_batch_desc(B, f, d[f], B->d_est + f);
        fill_batch_desc(B, f, d[B->F + f], run_est ? run_est + (int64_t)f * cap : nullptr);
    }
    CU(cudaMemcpyAsync(B->d_desc, d.data(), d.size() * sizeof(FilterDesc), cudaMemcpyHostToDevice, B->stream));
    CU(cudaStreamSynchronize(B->stream));
    return PF_OK;
}

static pf_status batch_status(int32_t st)
{
    if (st & PF_STATUS_MISALIGNED)
        return fail(PF_ERR_INVALID, "a sorted copy's rows were not 16-byte aligned (sub-filters kept their "
                                    "propagated particles)");
    if (st & PF_STATUS_WAIT_TIMEOUT)
        return fail(PF_ERR_TIMEOUT, "a bounded wait for a bulk copy ran out in a kernel (sub-filters kept their "
                                    "propagated particles)");
    return PF_OK;
}

static pf_status enqueue_batch_step(pf_batch* B, const FilterDesc* desc, InputRef in, int32_t* ctr_inc)
{
    for (const pf_batch::Group& g : B->groups) {
        const int2* map = B->map + g.map_off;  // the estimate CTAs, then the sub-filters
        CU(B->ops.sample_sort(g.M, g.E, g.TP, true, g.NS, B->stream, desc, map + g.NE, in));
        // a programmatic dependent of the sampling kernel when that pays (starts in its last wave, waits for
        // the grid)
        const int virt = dependent_launch_pays(g.NS, g.M, g.E, B->mi.S, B->cfg.device) ? 3 : 1;
        CU(B->ops.exchange_resample(g.M, g.E, B->cfg.resampler, g.NE + g.NS, B->stream, desc, map, in, nullptr,
                                    virt));
    }
    if (ctr_inc) CU(launch_counter_inc(ctr_inc, B->stream));
    return PF_OK;
}

extern "C" pf_status pf_batch_create(const pf_config* cfg, pf_model_id model, int32_t num_filters,
                                     const int32_t* num_particles, const void* params, size_t params_size,
                                     pf_batch** out)
{
    if (!cfg || !num_particles || !params || !out) return fail(PF_ERR_INVALID, "null argument");
    *out = nullptr;
    ModelInfo mi;
    if (!model_info(model, &mi)) return fail(PF_ERR_INVALID, "unknown model %d", (int)model);
    if (params_size != mi.psize)
        return fail(PF_ERR_INVALID, "model params size %zu, expected %zu", params_size, mi.psize);
    if (num_filters < 1) return fail(PF_ERR_INVALID, "num_filters must be >= 1");
    const int M = cfg->particles_per_subfilter;
    if (M < 32 || M > 1024 || (M & (M - 1)))
        return fail(PF_ERR_UNSUPPORTED, "particles per sub-filter must be a power of two in [32, 1024], got %d", M);
    const int E = cfg->particles_per_thread > 0 ? cfg->particles_per_thread : default_ppt(M, mi.S);
    if (!me_supported(M, E)) return fail(PF_ERR_UNSUPPORTED, "particles per thread %d not built for m=%d", E, M);
    if (cfg->rng != PF_RNG_SUBFILTER) return fail(PF_ERR_UNSUPPORTED, "batched filters use per-sub-filter streams");
    if (cfg->pipeline == PF_PIPELINE_PHASED)
        return fail(PF_ERR_UNSUPPORTED, "batched filters run the split pipeline, not the phased one");
    if (cfg->exchange != PF_EXCHANGE_NONE && cfg->exchange != PF_EXCHANGE_RING && cfg->exchange != PF_EXCHANGE_TORUS)
        return fail(PF_ERR_UNSUPPORTED, "batched filters exchange by ring or torus (or not at all)");
    if (cfg->num_transfer < 0) return fail(PF_ERR_INVALID, "num_transfer must be >= 0");
    if (cfg->exchange == PF_EXCHANGE_RING && 2 * cfg->num_transfer > M)
        return fail(PF_ERR_INVALID, "exchange needs 2*t <= m (t=%d, m=%d)", cfg->num_transfer, M);
    if (cfg->exchange == PF_EXCHANGE_TORUS && 5 * cfg->num_transfer > M)
        return fail(PF_ERR_INVALID, "torus exchange needs 5*t <= m (t=%d, m=%d)", cfg->num_transfer, M);
    if (cfg->resampler < PF_RESAMPLE_REFERENCE || cfg->resampler > PF_RESAMPLE_VOSE)
        return fail(PF_ERR_INVALID, "unknown resampler %d", cfg->resampler);
    if (!(cfg->resampling_freq >= 0.0f && cfg->resampling_freq <= 1.0f))
        return fail(PF_ERR_INVALID, "resampling_freq must be in [0, 1]");
    if (!(cfg->ess_fraction >= 0.0f && cfg->ess_fraction <= 1.0f))
        return fail(PF_ERR_INVALID, "ess_fraction must be in [0, 1]");
    if (cfg->stream_offset < 0 || cfg->exchange_period < 0)
        return fail(PF_ERR_INVALID, "stream_offset and exchange_period must be >= 0");
    if (cfg->threads_per_particle < 0 || cfg->threads_per_particle > 2)
        return fail(PF_ERR_INVALID, "threads_per_particle must be 1 or 2");
    if (cfg->threads_per_particle == 2 && 2 * M / E > 1024)
        return fail(PF_ERR_UNSUPPORTED, "two threads per particle need 2 m / ppt <= 1024 threads (m=%d, ppt=%d)", M,
                    E);
    int64_t P = 0, NS = 0;
    std::vector<int32_t> mf(num_filters);
    for (int f = 0; f < num_filters; ++f) {
        const int32_t n = num_particles[f];
        // the largest power of two m' <= m dividing n whose grid and exchange fit
        int mm = 0;
        for (int c = M; c >= 32 && !mm; c >>= 1) {
            if (n < c || n % c) continue;
            if (cfg->exchange == PF_EXCHANGE_TORUS) {
                int dx, dy;
                torus_dims(n / c, &dx, &dy);
                if (dx * dy != n / c || 5 * cfg->num_transfer > c) continue;
            }
            if (cfg->exchange == PF_EXCHANGE_RING && 2 * cfg->num_transfer > c) continue;
            mm = c;
        }
        if (!mm)
            return fail(PF_ERR_INVALID, "filter %d: no sub-filter size in [32, %d] divides %d particles%s", f, M, n,
                        cfg->exchange == PF_EXCHANGE_TORUS ? " into a torus" : "");
        mf[f] = mm;
        P += n;
        NS += n / mm;
    }
    if (NS > INT32_MAX / 2 || P > ((int64_t)1 << 34)) return fail(PF_ERR_INVALID, "batch too large");
    pf_status s = require_gpu(cfg->device);
    if (s != PF_OK) return s;

    pf_batch* B = new pf_batch();
    B->cfg = *cfg;
    B->model = model;
    B->mi = mi;
    B->ops = model_ops(model);
    B->F = num_filters;
    B->M = M;
    B->E = E;
    B->S = mi.S;
    B->t = cfg->exchange == PF_EXCHANGE_NONE ? 0 : cfg->num_transfer;
    B->P = P;
    B->NS = (int)NS;
    B->nsub.resize(num_filters);
    B->sub_off.resize(num_filters);
    B->part_off.resize(num_filters);
    B->grp_off.resize(num_filters);
    B->mp.resize(num_filters);
    B->mf = mf;
    B->ru_off.resize(num_filters);
    int64_t po = 0, ro = 0;
    int so = 0, go = 0;
    for (int f = 0; f < num_filters; ++f) {
        B->nsub[f] = num_particles[f] / mf[f];
        B->sub_off[f] = so;
        B->part_off[f] = po;
        B->grp_off[f] = go;
        B->ru_off[f] = ro;
        ro += (int64_t)B->nsub[f] * (1 + resample_draws(cfg->resampler, mf[f]));
        so += B->nsub[f];
        go += (B->nsub[f] + 31) / 32;
        po += num_particles[f];
        memset(&B->mp[f], 0, sizeof(ModelParams));
        memcpy(&B->mp[f], static_cast<const char*>(params) + (size_t)f * params_size, params_size);
        if (model == PF_MODEL_UNICYCLE) {
            const pf_unicycle_params& p = B->mp[f].uni;
            if (p.num_landmarks < 1 || p.num_landmarks > 8 || !(p.sigma_range > 0) || !(p.sigma_bearing > 0)) {
                release(B);
                return fail(PF_ERR_INVALID, "filter %d: 1..8 landmarks and positive sigmas", f);
            }
        } else if (model == PF_MODEL_BEACON) {
            const pf_beacon_params& p = B->mp[f].bcn;
            if (p.num_beacons < 1 || p.num_beacons > 16 || !(p.sigma_range > 0)) {
                release(B);
                return fail(PF_ERR_INVALID, "filter %d: 1..16 beacons and a positive sigma", f);
            }
        }
    }
    // one group of launches per sub-filter size, the largest first
    for (int c = M; c >= 32; c >>= 1) {
        int ns = 0, ne = 0;
        for (int f = 0; f < num_filters; ++f)
            if (mf[f] == c) {
                ns += B->nsub[f];
                ne += estimate_ctas(B->nsub[f]);
            }
        if (!ns) continue;
        const int ec = c == M ? E : (cfg->particles_per_thread > 0 && me_supported(c, cfg->particles_per_thread)
                                         ? cfg->particles_per_thread
                                         : default_ppt(c, mi.S));
        // two threads per particle where the sampling kernel's CTA stays within 1024 threads
        const int tp = cfg->threads_per_particle == 2 && 2 * c / ec <= 1024 ? 2 : 1;
        B->groups.push_back(pf_batch::Group{c, ec, tp, ns, ne, 0});
    }
    cudaError_t e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        release(B);
        return fail(PF_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
#define TRY(x)              \
    do {                    \
        pf_status s_ = (x); \
        if (s_ != PF_OK) {  \
            release(B);     \
            return s_;      \
        }                   \
    } while (0)
    TRY(balloc(B, &B->state, (size_t)B->S * P));
    TRY(balloc(B, &B->tmp, (size_t)B->S * P));
    TRY(balloc(B, &B->tkey, (size_t)P));
    TRY(balloc(B, &B->winner, (size_t)NS));
    TRY(balloc(B, &B->part, (size_t)NS * kPartStride));
    TRY(balloc(B, &B->mtgp, (size_t)NS * kMtgpN));
    TRY(balloc(B, &B->ru, (size_t)ro));
    TRY(balloc(B, &B->gpart, (size_t)go * kPartStride));
    TRY(balloc(B, &B->est_ctr, (size_t)num_filters));
    TRY(balloc(B, &B->ctr, 1));
    TRY(balloc(B, &B->map, (size_t)NS + go));
    TRY(balloc(B, &B->d_desc, 2 * (size_t)num_filters));
    TRY(balloc(B, &B->d_in, (size_t)num_filters));
    TRY(balloc(B, &B->d_est, (size_t)num_filters + 1));  // + the kernels' status word
    if (cudaMallocHost(&B->h_in, sizeof(pf_step_input) * num_filters) != cudaSuccess ||
        cudaMallocHost(&B->h_est, sizeof(pf_estimate) * (num_filters + 1)) != cudaSuccess) {
        cudaGetLastError();
        release(B);
        return fail(PF_ERR_NOMEM, "cudaMallocHost failed");
    }
    {
        // per sub-filter size, the estimate CTAs (filter, -1 - group) first --
        // they combine each group of 32 sub-filters' partials in the
        // resampling kernel's first wave -- then every sub-filter
        std::vector<int2> map;
        map.reserve((size_t)NS + go);
        for (pf_batch::Group& g : B->groups) {
            g.map_off = (int)map.size();
            for (int f = 0; f < num_filters; ++f)
                if (mf[f] == g.M)
                    for (int q = 0; q < estimate_ctas(B->nsub[f]); ++q) map.push_back(make_int2(f, -1 - q));
            for (int f = 0; f < num_filters; ++f)
                if (mf[f] == g.M)
                    for (int b = 0; b < B->nsub[f]; ++b) map.push_back(make_int2(f, b));
        }
        B->map_len = (int)map.size();
        if (cudaMemcpy(B->map, map.data(), map.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess ||
            launch_mtgp_init(B->mtgp, (int)NS, cfg->stream_offset, cfg->seed, B->stream) != cudaSuccess ||
            cudaStreamSynchronize(B->stream) != cudaSuccess) {
            cudaGetLastError();
            release(B);
            return fail(PF_ERR_CUDA, "initial upload failed");
        }
    }
    if (cudaMemset(B->est_ctr, 0, 4 * (size_t)num_filters) != cudaSuccess || cudaMemset(B->ctr, 0, 4) != cudaSuccess ||
        cudaMemset(B->d_est + num_filters, 0, sizeof(pf_estimate)) != cudaSuccess) {
        cudaGetLastError();
        release(B);
        return fail(PF_ERR_CUDA, "cudaMemset failed");
    }
    TRY(upload_batch_descs(B, nullptr, 0));
    {
        std::vector<float> init((size_t)num_filters * B->S);
        for (int f = 0; f < num_filters; ++f)
            memcpy(init.data() + (size_t)f * B->S, init_state_of(model, B->mp[f]), sizeof(float) * B->S);
        TRY(pf_batch_set_initial_states(B, init.data()));
    }
#undef TRY
    *out = B;
    return PF_OK;
}

extern "C" pf_status pf_batch_destroy(pf_batch* B)
{
    if (!B) return PF_OK;
    cudaSetDevice(B->cfg.device);
    cudaStreamSynchronize(B->stream);
    release(B);
    return PF_OK;
}

extern "C" pf_status pf_batch_set_initial_states(pf_batch* B, const float* states)
{
    if (!B || !states) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(B->cfg.device));
    CU(cudaStreamSynchronize(B->stream));
    float* d = nullptr;
    CU(cudaMalloc(&d, sizeof(float) * B->S * B->F));
    cudaError_t e = cudaMemcpy(d, states, sizeof(float) * B->S * B->F, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_batch_fill<<<B->map_len, 256, 0, B->stream>>>(B->d_desc, B->map, d, B->S);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(PF_ERR_CUDA, "set initial states: %s", cudaGetErrorString(e));
    B->steps_done = 0;
    return PF_OK;
}

extern "C" pf_status pf_batch_get_particles(pf_batch* B, int32_t filter, float* soa)
{
    if (!B || !soa) return fail(PF_ERR_INVALID, "null argument");
    if (filter < 0 || filter >= B->F) return fail(PF_ERR_INVALID, "filter %d out of range", filter);
    CU(cudaSetDevice(B->cfg.device));
    CU(cudaStreamSynchronize(B->stream));
    const int64_t T = (int64_t)B->mf[filter] * B->nsub[filter];
    for (int v = 0; v < B->S; ++v)
        CU(cudaMemcpy(soa + v * T, B->state + (int64_t)B->S * B->part_off[filter] + v * T, (size_t)T * 4,
                      cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pf_batch_step(pf_batch* B, const pf_step_input* inputs, pf_estimate* out)
{
    if (!B || !inputs) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(B->cfg.device));
    memcpy(B->h_in, inputs, sizeof(pf_step_input) * B->F);
    CU(cudaMemcpyAsync(B->d_in, B->h_in, sizeof(pf_step_input) * B->F, cudaMemcpyHostToDevice, B->stream));
    InputRef ir{B->d_in, 1, nullptr, 0, B->steps_done};
    pf_status s = enqueue_batch_step(B, B->d_desc, ir, nullptr);
    if (s != PF_OK) return s;
    // the estimates and the kernels' status word after them in one copy
    CU(cudaMemcpyAsync(out ? (void*)B->h_est : (void*)(B->h_est + B->F), out ? (void*)B->d_est : (void*)(B->d_est + B->F),
                       out ? sizeof(pf_estimate) * B->F + sizeof(int32_t) : sizeof(int32_t), cudaMemcpyDeviceToHost,
                       B->stream));
    CU(cudaStreamSynchronize(B->stream));
    B->steps_done++;
    s = batch_status(*reinterpret_cast<const int32_t*>(B->h_est + B->F));
    if (s != PF_OK) return s;
    if (out) {
        memcpy(out, B->h_est, sizeof(pf_estimate) * B->F);
        for (int f = 0; f < B->F; ++f) out[f].step = B->steps_done;
    }
    return PF_OK;
}

static pf_status capture(pf_batch* B, int steps, InputRef ir, cudaGraphExec_t* exec)
{
    cudaGraph_t g = nullptr;
    CU(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    pf_status s = PF_OK;
    for (int i = 0; i < steps && s == PF_OK; ++i) s = enqueue_batch_step(B, B->d_desc + B->F, ir, B->ctr);
    cudaError_t e = cudaStreamEndCapture(B->stream, &g);
    if (s != PF_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return fail(PF_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *exec = nullptr;
        return fail(PF_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    return PF_OK;
}

extern "C" pf_status pf_batch_submit(pf_batch* B, const pf_step_input* d_inputs, pf_estimate* d_estimates,
                                     int32_t capacity, int32_t steps)
{
    if (!B || !d_inputs || !d_estimates || capacity < 1 || steps < 0) return fail(PF_ERR_INVALID, "bad argument");
    CU(cudaSetDevice(B->cfg.device));
    if (B->graph_inputs != d_inputs || B->graph_est != d_estimates || B->graph_cap != capacity) {
        CU(cudaStreamSynchronize(B->stream));
        drop_graphs(B);
        pf_status s = upload_batch_descs(B, d_estimates, capacity);
        if (s != PF_OK) return s;
        B->graph_inputs = d_inputs;
        B->graph_est = d_estimates;
        B->graph_cap = capacity;
    }
    InputRef ir{d_inputs, capacity, B->ctr, capacity, 0};
    if (!B->graph_n && steps > 0) {
        B->graph_steps = steps < kMaxGraphSteps ? steps : kMaxGraphSteps;
        pf_status s = capture(B, B->graph_steps, ir, &B->graph_n);
        if (s != PF_OK) return s;
    }
    if (!B->graph_1 && steps % (B->graph_steps > 0 ? B->graph_steps : 1) != 0) {
        pf_status s = capture(B, 1, ir, &B->graph_1);
        if (s != PF_OK) return s;
    }
    CU(cudaMemsetAsync(B->ctr, 0, sizeof(int32_t), B->stream));
    int left = steps;
    while (left >= B->graph_steps && B->graph_steps > 0) {
        CU(cudaGraphLaunch(B->graph_n, B->stream));
        left -= B->graph_steps;
    }
    for (; left > 0; --left) CU(cudaGraphLaunch(B->graph_1, B->stream));
    B->steps_done += steps;
    return PF_OK;
}

extern "C" pf_status pf_batch_poll(pf_batch* B, int32_t* done)
{
    if (!B || !done) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(B->cfg.device));
    const cudaError_t e = cudaStreamQuery(B->stream);
    if (e == cudaSuccess) {
        *done = 1;
        return PF_OK;
    }
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        *done = 0;
        return PF_OK;
    }
    return fail(PF_ERR_CUDA, "pf_batch_poll: %s", cudaGetErrorString(e));
}

extern "C" pf_status pf_batch_synchronize(pf_batch* B)
{
    if (!B) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(B->cfg.device));
    CU(cudaStreamSynchronize(B->stream));
    int32_t st = 0;
    CU(cudaMemcpy(&st, B->d_est + B->F, sizeof(st), cudaMemcpyDeviceToHost));
    return batch_status(st);
}

extern "C" void* pf_batch_stream(pf_batch* B) { return B ? (void*)B->stream : nullptr; }

extern "C" pf_status pf_batch_info(pf_batch* B, int32_t* num_filters, int64_t* total_particles,
                                   int32_t* total_subfilters, int32_t* ppt, int64_t* bytes)
{
    if (!B) return fail(PF_ERR_INVALID, "null argument");
    if (num_filters) *num_filters = B->F;
    if (total_particles) *total_particles = B->P;
    if (total_subfilters) *total_subfilters = B->NS;
    if (ppt) *ppt = B->E;
    if (bytes) *bytes = B->dev_bytes;
    return PF_OK;
}

extern "C" pf_status pf_batch_filter_info(pf_batch* B, int32_t filter, int32_t* num_subfilters,
                                          int32_t* stream_offset, int64_t* particle_offset)
{
    if (!B) return fail(PF_ERR_INVALID, "null argument");
    if (filter < 0 || filter >= B->F) return fail(PF_ERR_INVALID, "filter %d out of range", filter);
    if (num_subfilters) *num_subfilters = B->nsub[filter];
    if (stream_offset) *stream_offset = B->cfg.stream_offset + B->sub_off[filter];
    if (particle_offset) *particle_offset = B->part_off[filter];
    return PF_OK;
}

extern "C" pf_status pf_batch_filter_shape(pf_batch* B, int32_t filter, int32_t* particles_per_subfilter,
                                           int32_t* particles_per_thread)
{
    if (!B) return fail(PF_ERR_INVALID, "null argument");
    if (filter < 0 || filter >= B->F) return fail(PF_ERR_INVALID, "filter %d out of range", filter);
    for (const pf_batch::Group& g : B->groups)
        if (g.M == B->mf[filter]) {
            if (particles_per_subfilter) *particles_per_subfilter = g.M;
            if (particles_per_thread) *particles_per_thread = g.E;
        }
    return PF_OK;
}

extern "C" pf_status pf_batch_get_sorted(pf_batch* B, int32_t filter, float* soa, float* keys)
{
    if (!B || !soa || !keys) return fail(PF_ERR_INVALID, "null argument");
    if (filter < 0 || filter >= B->F) return fail(PF_ERR_INVALID, "filter %d out of range", filter);
    CU(cudaSetDevice(B->cfg.device));
    CU(cudaStreamSynchronize(B->stream));
    const int64_t T = (int64_t)B->mf[filter] * B->nsub[filter];
    const int64_t p0 = B->part_off[filter];
    for (int v = 0; v < B->S; ++v)
        CU(cudaMemcpy(soa + v * T, B->tmp + (int64_t)B->S * p0 + v * T, (size_t)T * 4, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(keys, B->tkey + p0, (size_t)T * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: times every (m, particles per thread, threads per particle,
// exchange period) candidate
// on the caller's inputs and picks the fastest whose tracking error stays
// within a tolerance of the every-step-exchange candidates.
// ---------------------------------------------------------------------------
namespace {

struct DevMem {
    void* p = nullptr;
    ~DevMem()
    {
        if (p) cudaFree(p);
    }
};

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

// Root mean square over filters, steps >= burn_in and state variables of
// (estimate mean - truth), angular variables wrapped to (-pi, pi].
double tracking_rmse(const std::vector<pf_estimate>& est, const float* truth, int F, int steps, int burn_in, int S,
                     uint32_t amask)
{
    double acc = 0.0;
    int64_t n = 0;
    for (int f = 0; f < F; ++f)
        for (int k = burn_in; k < steps; ++k) {
            const pf_estimate& e = est[(size_t)f * steps + k];
            const float* x = truth + ((size_t)f * steps + k) * S;
            for (int v = 0; v < S; ++v) {
                double d = e.mean[v] - (double)x[v];
                if ((amask >> v) & 1u) d = std::remainder(d, 2.0 * M_PI);
                acc += d * d;
                ++n;
            }
        }
    return n ? std::sqrt(acc / (double)n) : NAN;
}

}  // namespace

extern "C" pf_status pf_batch_autotune(const pf_config* base, pf_model_id model, int32_t num_filters,
                                       const int32_t* num_particles, const void* params, size_t params_size,
                                       const pf_step_input* inputs, const float* truth, int32_t steps,
                                       int32_t burn_in, const int32_t* m_list, int32_t n_m, const int32_t* ppt_list,
                                       int32_t n_ppt, const int32_t* tpp_list, int32_t n_tpp,
                                       const int32_t* period_list, int32_t n_period, float rmse_tol,
                                       pf_tune_entry* table, int32_t table_cap, int32_t* n_table, pf_config* best)
{
    if (!base || !num_particles || !params || !inputs || !m_list || !ppt_list || !tpp_list || !period_list ||
        !table || !n_table || !best)
        return fail(PF_ERR_INVALID, "null argument");
    if (num_filters < 1 || steps < 1 || burn_in < 0 || burn_in >= steps || n_m < 1 || n_ppt < 1 || n_tpp < 1 ||
        n_period < 1)
        return fail(PF_ERR_INVALID, "bad tuning shape");
    if ((int64_t)n_m * n_ppt * n_tpp * n_period > table_cap)
        return fail(PF_ERR_INVALID, "table too small for the candidates");
    ModelInfo mi;
    if (!model_info(model, &mi)) return fail(PF_ERR_INVALID, "unknown model %d", (int)model);
    pf_status s = require_gpu(base->device);
    if (s != PF_OK) return s;
    const size_t nio = (size_t)num_filters * steps;
    DevMem din, dest;
    CU(cudaMalloc(&din.p, nio * sizeof(pf_step_input)));
    CU(cudaMalloc(&dest.p, nio * sizeof(pf_estimate)));
    CU(cudaMemcpy(din.p, inputs, nio * sizeof(pf_step_input), cudaMemcpyHostToDevice));
    EventPair ev;
    CU(cudaEventCreate(&ev.a));
    CU(cudaEventCreate(&ev.b));
    std::vector<pf_estimate> est(nio);
    std::vector<float> init((size_t)num_filters * mi.S);
    for (int f = 0; f < num_filters; ++f) {
        ModelParams mp;
        memset(&mp, 0, sizeof(mp));
        memcpy(&mp, static_cast<const char*>(params) + (size_t)f * params_size,
               std::min(params_size, sizeof(ModelParams)));
        memcpy(init.data() + (size_t)f * mi.S, init_state_of(model, mp), sizeof(float) * mi.S);
    }
    int n = 0;
    for (int im = 0; im < n_m; ++im)
        for (int ip = 0; ip < n_ppt; ++ip)
            for (int it = 0; it < n_tpp; ++it)
                for (int iq = 0; iq < n_period; ++iq) {
                    pf_tune_entry& t = table[n++];
                    memset(&t, 0, sizeof(t));
                    t.particles_per_subfilter = m_list[im];
                    t.particles_per_thread = ppt_list[ip];
                    t.threads_per_particle = tpp_list[it];
                    t.exchange_period = period_list[iq];
                    t.rmse = NAN;
                    pf_config c = *base;
                    c.particles_per_subfilter = m_list[im];
                    c.particles_per_thread = ppt_list[ip];
                    c.threads_per_particle = tpp_list[it];
                    c.exchange_period = period_list[iq];
                    pf_batch* B = nullptr;
                    t.status = pf_batch_create(&c, model, num_filters, num_particles, params, params_size, &B);
                    if (t.status != PF_OK) continue;
                    // first run captures the graph; the timed run replays it from the initial states
                    pf_status r = pf_batch_submit(B, (const pf_step_input*)din.p, (pf_estimate*)dest.p, steps, steps);
                    if (r == PF_OK) r = pf_batch_synchronize(B);
                    if (r == PF_OK) r = pf_batch_set_initial_states(B, init.data());
                    cudaError_t e = cudaSuccess;
                    if (r == PF_OK) e = cudaEventRecord(ev.a, B->stream);
                    if (r == PF_OK && e == cudaSuccess)
                        r = pf_batch_submit(B, (const pf_step_input*)din.p, (pf_estimate*)dest.p, steps, steps);
                    if (r == PF_OK && e == cudaSuccess) e = cudaEventRecord(ev.b, B->stream);
                    if (r == PF_OK && e == cudaSuccess) e = cudaEventSynchronize(ev.b);
                    float ms = 0.0f;
                    if (r == PF_OK && e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.a, ev.b);
                    if (r == PF_OK && e == cudaSuccess)
                        e = cudaMemcpy(est.data(), dest.p, nio * sizeof(pf_estimate), cudaMemcpyDeviceToHost);
                    pf_batch_destroy(B);
                    if (r != PF_OK || e != cudaSuccess) {
                        if (e != cudaSuccess) return fail(PF_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
                        t.status = r;
                        continue;
                    }
                    t.ms_per_step = ms / (float)steps;
                    int64_t P = 0;
                    for (int f = 0; f < num_filters; ++f) P += num_particles[f];
                    t.particle_steps_per_s = (double)P * steps / (ms * 1e-3);
                    if (truth)
                        t.rmse = tracking_rmse(est, truth, num_filters, steps, burn_in, mi.S, angle_mask_of(model));
                }
    *n_table = n;
    // reference error: mean over the runnable every-step-exchange candidates
    double ref = 0.0;
    int nref = 0;
    for (int i = 0; i < n; ++i)
        if (table[i].status == PF_OK && table[i].exchange_period <= 1 && std::isfinite(table[i].rmse)) {
            ref += table[i].rmse;
            ++nref;
        }
    ref = nref ? ref / nref : NAN;
    int pick = -1;
    for (int i = 0; i < n; ++i) {
        pf_tune_entry& t = table[i];
        if (t.status != PF_OK) continue;
        t.accepted = truth ? (nref > 0 && std::isfinite(t.rmse) && t.rmse <= ref * (1.0 + rmse_tol))
                           : (t.exchange_period <= 1);
        if (t.accepted && (pick < 0 || t.particle_steps_per_s > table[pick].particle_steps_per_s)) pick = i;
    }
    if (pick < 0) return fail(PF_ERR_UNSUPPORTED, "autotune: no candidate could run (last: %s)", pf_last_error());
    *best = *base;
    best->particles_per_subfilter = table[pick].particles_per_subfilter;
    best->particles_per_thread = table[pick].particles_per_thread;
    best->threads_per_particle = table[pick].threads_per_particle;
    best->exchange_period = table[pick].exchange_period;
    return PF_OK;
}
