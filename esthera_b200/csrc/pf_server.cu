// pf_server.cu -- the serving form (include/esthera_b200.h, pf_server_*): many
// independent filters kept resident on one GPU (particles, sorted copies,
// log-weights, MTGP32 streams), admitted against an HBM budget, whose
// measurement updates are batched as they arrive.
//
// Continuous batching: pf_server_update queues an update on the host; each
// pf_server_launch takes the oldest queued update of every filter that has
// none in flight and runs all of them as one batch: one host->device copy of
// the compact (slot, input) list, an expand kernel writing the CTA ->
// (slot, sub-filter) maps, the split pipeline's two kernels per model (each
// model on its own stream, forked from the server's stream after the copies
// and joined back before the gather, so the models' grids overlap), and a
// gather of the batch's estimates copied back in one transfer.  Filters are
// opened, closed and updated while batches run; everything else is ordered on
// the server's stream, so memory released by a closed filter is reused only
// after the batches that touched it.
//
// Filter memory comes from a stream-ordered pool (cudaMallocAsync), one block
// per filter; admission charges the block's size against the budget.  Each
// filter's sub-filter b uses MTGP32 parameter set b mod 200 seeded with the
// filter's seed + b + 1 -- the streams a pf_filter with that seed has -- so a
// filter's results are the same alone and in any mix.
#include <algorithm>
#include <cstring>
#include <deque>
#include <vector>

#include "pf_host.cuh"

using namespace pfdev;
using namespace pfhost;

namespace {

struct Pending {         // one update in a batch (host -> device)
    int32_t slot;
    int32_t first_lead;  // position of the slot's estimate CTAs in its model's CTA map
    int32_t first_rest;  // position of its sub-filters, after all estimate CTAs
};

// One block per batched update: copy its input into the slot's input entry
// and write the slot's CTA map entries -- group leaders (sub-filters 0, 32,
// ...) in the map's leader region, the rest after all leaders, so that the
// resampling kernel combines the estimates in its first wave.
__global__ void k_srv_expand(const Pending* __restrict__ pend, const pf_step_input* __restrict__ in, int n,
                             const FilterDesc* __restrict__ descs, pf_step_input* __restrict__ slot_in,
                             int2* __restrict__ map)
{
    const int i = blockIdx.x;
    if (i >= n) return;
    const Pending p = pend[i];
    const int N = descs[p.slot].N;
    for (int b = threadIdx.x; b < N; b += blockDim.x) map[p.first_rest + b] = make_int2(p.slot, b);
    for (int q = threadIdx.x; q < estimate_ctas(N); q += blockDim.x) map[p.first_lead + q] = make_int2(p.slot, -1 - q);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(in + i);
    uint32_t* dst = reinterpret_cast<uint32_t*>(slot_in + p.slot);
    for (int w = threadIdx.x; w < (int)(sizeof(pf_step_input) / 4); w += blockDim.x) dst[w] = src[w];
}

// Block i copies pending update i's estimate to out[i]; block n copies the
// kernels' status word into out[n] (so one D2H copy brings both back).
__global__ void k_srv_gather(const Pending* __restrict__ pend, int n, const pf_estimate* __restrict__ est_tab,
                             pf_estimate* __restrict__ out, const int32_t* __restrict__ status)
{
    const int i = blockIdx.x;
    if (i == n) {
        if (threadIdx.x == 0) *reinterpret_cast<int32_t*>(out + n) = *status;
        return;
    }
    if (i > n) return;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(est_tab + pend[i].slot);
    uint32_t* dst = reinterpret_cast<uint32_t*>(out + i);
    for (int w = threadIdx.x; w < (int)(sizeof(pf_estimate) / 4); w += blockDim.x) dst[w] = src[w];
}

// Every particle of the slot's filter set to init[v].
__global__ void k_srv_fill(const FilterDesc* __restrict__ descs, int slot, const float* __restrict__ init, int S)
{
    const FilterDesc& D = descs[slot];
    const int64_t T = D.T;
    for (int v = 0; v < S; ++v) {
        const float x = init[v];
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += (int64_t)gridDim.x * blockDim.x)
            D.state[v * T + i] = x;
    }
}

constexpr size_t kAlign = 256;
inline size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Byte offsets of a filter's arrays inside its block.
struct Layout {
    size_t state, tmp, tkey, winner, part, mtgp, ru, gpart, est_ctr, init, total;
};

Layout layout_of(int S, int M, int N, int64_t ru_stride)
{
    Layout L;
    const size_t T = (size_t)M * N;
    size_t o = 0;
    L.state = o, o += up(4 * (size_t)S * T);
    L.tmp = o, o += up(4 * (size_t)S * T);
    L.tkey = o, o += up(4 * T);
    L.winner = o, o += up(4 * (size_t)N);
    L.part = o, o += up(8 * (size_t)N * kPartStride);
    L.mtgp = o, o += up(4 * (size_t)N * kMtgpN);
    L.ru = o, o += up(4 * (size_t)N * ru_stride);
    L.gpart = o, o += up(8 * (size_t)((N + 31) / 32) * kPartStride);
    L.est_ctr = o, o += kAlign;
    L.init = o, o += up(4 * PF_MAX_STATE);
    L.total = o;
    return L;
}

struct Slot {
    bool open = false;
    int model = 0;
    int N = 0;
    int64_t T = 0;
    size_t bytes = 0;
    char* mem = nullptr;
    bool in_flight = false;
    bool in_ready = false;  // listed in its model's ready list
    int32_t steps = 0;
    std::deque<std::pair<pf_step_input, uint64_t>> queue;  // (input, caller tag)
};

}  // namespace

struct pf_server {
    pf_config cfg;
    int device = 0;
    int64_t budget = 0, used = 0;
    int max_filters = 0;
    int E[PF_NUM_MODELS] = {};  // particles per thread of each model's kernels
    int64_t nbm[PF_NUM_MODELS] = {}, draws[PF_NUM_MODELS] = {};
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaEvent_t done = nullptr;
    // each model's kernels run on their own stream, forked from and joined
    // back into `stream`, so the models' grids of a batch overlap
    cudaStream_t side[PF_NUM_MODELS] = {};
    cudaEvent_t fork = nullptr, join[PF_NUM_MODELS] = {};
    std::vector<Slot> slots;
    std::vector<int> free_slots;
    // slots with a queued update and none in flight, per model, in the order
    // they became ready (entries of closed slots are dropped at the launch)
    std::vector<int> ready[PF_NUM_MODELS];
    int64_t n_open = 0, resident_T = 0, resident_sub = 0, queued = 0;
    // device tables
    FilterDesc* d_desc = nullptr;
    pf_step_input* d_slot_in = nullptr;
    pf_estimate* d_est_tab = nullptr;
    int2* d_map[PF_NUM_MODELS] = {};
    int64_t map_cap = 0;
    Pending* d_pend = nullptr;
    pf_step_input* d_in = nullptr;
    pf_estimate* d_out = nullptr;
    int32_t* d_status = nullptr;  // PF_STATUS_* bits set by the kernels
    // pinned staging
    Pending* h_pend = nullptr;
    pf_step_input* h_in = nullptr;
    pf_estimate* h_out = nullptr;
    // the batch in flight
    bool busy = false;
    std::vector<int32_t> batch_slots;
    std::vector<uint64_t> batch_tags;
    int64_t launches = 0, updates = 0, particle_steps = 0;
};

static void srv_release(pf_server* s)
{
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& sl : s->slots)
        if (sl.mem) cudaFreeAsync(sl.mem, s->stream);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (int m = 0; m < PF_NUM_MODELS; ++m)
        if (s->d_map[m]) cudaFreeAsync(s->d_map[m], s->stream);
    if (s->stream) cudaStreamSynchronize(s->stream);
    void* dev[] = {s->d_desc, s->d_slot_in, s->d_est_tab, s->d_pend, s->d_in, s->d_out, s->d_status};
    for (void* p : dev)
        if (p) cudaFree(p);
    void* host[] = {s->h_pend, s->h_in, s->h_out};
    for (void* p : host)
        if (p) cudaFreeHost(p);
    if (s->done) cudaEventDestroy(s->done);
    if (s->fork) cudaEventDestroy(s->fork);
    for (int m = 0; m < PF_NUM_MODELS; ++m) {
        if (s->join[m]) cudaEventDestroy(s->join[m]);
        if (s->side[m]) cudaStreamDestroy(s->side[m]);
    }
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

static pf_status ensure_map(pf_server* s, int64_t need);

extern "C" pf_status pf_server_create(const pf_config* cfg, int64_t hbm_budget, int32_t max_filters,
                                      pf_server** out)
{
    if (!cfg || !out) return fail(PF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (hbm_budget <= 0 || max_filters < 1) return fail(PF_ERR_INVALID, "budget and max_filters must be positive");
    const int M = cfg->particles_per_subfilter;
    if (M < 32 || M > 1024 || (M & (M - 1)))
        return fail(PF_ERR_UNSUPPORTED, "particles per sub-filter must be a power of two in [32, 1024], got %d", M);
    int E[PF_NUM_MODELS];
    for (int m = 0; m < PF_NUM_MODELS; ++m) {
        ModelInfo mi;
        model_info(m, &mi);
        E[m] = cfg->particles_per_thread > 0 ? cfg->particles_per_thread : default_ppt(M, mi.S);
        if (!me_supported(M, E[m]))
            return fail(PF_ERR_UNSUPPORTED, "particles per thread %d not built for m=%d", E[m], M);
    }
    if (cfg->exchange != PF_EXCHANGE_NONE && cfg->exchange != PF_EXCHANGE_RING)
        return fail(PF_ERR_UNSUPPORTED, "served filters exchange by ring (or not at all)");
    if (cfg->exchange == PF_EXCHANGE_RING && (cfg->num_transfer < 0 || 2 * cfg->num_transfer > M))
        return fail(PF_ERR_INVALID, "exchange needs 0 <= 2*t <= m");
    if (cfg->exchange_period > 1) return fail(PF_ERR_UNSUPPORTED, "served filters exchange every step");
    if (cfg->resampler < PF_RESAMPLE_REFERENCE || cfg->resampler > PF_RESAMPLE_VOSE)
        return fail(PF_ERR_INVALID, "unknown resampler %d", cfg->resampler);
    if (!(cfg->resampling_freq >= 0.0f && cfg->resampling_freq <= 1.0f))
        return fail(PF_ERR_INVALID, "resampling_freq must be in [0, 1]");
    if (!(cfg->ess_fraction >= 0.0f && cfg->ess_fraction <= 1.0f))
        return fail(PF_ERR_INVALID, "ess_fraction must be in [0, 1]");
    pf_status st = require_gpu(cfg->device);
    if (st != PF_OK) return st;
    pf_server* s = new pf_server();
    s->cfg = *cfg;
    s->device = cfg->device;
    s->budget = hbm_budget;
    s->max_filters = max_filters;
    for (int m = 0; m < PF_NUM_MODELS; ++m) s->E[m] = E[m];
    for (int m = 0; m < PF_NUM_MODELS; ++m) {
        ModelInfo mi;
        model_info(m, &mi);
        s->nbm[m] = 2 * (((int64_t)mi.K * M + 1) / 2);
        s->draws[m] = s->nbm[m] + 1 + resample_draws(cfg->resampler, M);
    }
    s->slots.resize(max_filters);
    for (int i = max_filters - 1; i >= 0; --i) s->free_slots.push_back(i);
#define STRY(x)                                                           \
    do {                                                                  \
        cudaError_t e_ = (x);                                             \
        if (e_ != cudaSuccess) {                                          \
            cudaGetLastError();                                           \
            srv_release(s);                                               \
            return fail(PF_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
        }                                                                 \
    } while (0)
    STRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    STRY(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming));
    STRY(cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming));
    for (int m = 0; m < PF_NUM_MODELS; ++m) {
        STRY(cudaStreamCreateWithFlags(&s->side[m], cudaStreamNonBlocking));
        STRY(cudaEventCreateWithFlags(&s->join[m], cudaEventDisableTiming));
    }
    STRY(cudaDeviceGetDefaultMemPool(&s->pool, cfg->device));
    {
        uint64_t keep = UINT64_MAX;  // keep freed blocks in the pool for the next admission
        STRY(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    STRY(cudaMalloc(&s->d_desc, sizeof(FilterDesc) * max_filters));
    STRY(cudaMalloc(&s->d_slot_in, sizeof(pf_step_input) * max_filters));
    STRY(cudaMalloc(&s->d_est_tab, sizeof(pf_estimate) * max_filters));
    STRY(cudaMalloc(&s->d_pend, sizeof(Pending) * max_filters));
    STRY(cudaMalloc(&s->d_in, sizeof(pf_step_input) * max_filters));
    STRY(cudaMalloc(&s->d_out, sizeof(pf_estimate) * (max_filters + 1)));
    STRY(cudaMalloc(&s->d_status, sizeof(int32_t)));
    STRY(cudaMemset(s->d_status, 0, sizeof(int32_t)));
    STRY(cudaMallocHost(&s->h_pend, sizeof(Pending) * max_filters));
    STRY(cudaMallocHost(&s->h_in, sizeof(pf_step_input) * max_filters));
    STRY(cudaMallocHost(&s->h_out, sizeof(pf_estimate) * (max_filters + 1)));
#undef STRY
    {
        const pf_status ms = ensure_map(s, 1 << 20);  // 8 MB per model: a few growths at most afterwards
        if (ms != PF_OK) {
            srv_release(s);
            return ms;
        }
    }
    // Warm-up: reserve pool memory up front (growing the pool later stalls the
    // stream) and run one update of each served model, so that loading the
    // kernels does not land on the first requests.
    {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t reserve = std::min<size_t>((size_t)hbm_budget, free_b / 2) / (1 << 20) * (1 << 20);
        void* r = nullptr;
        if (reserve > 0 && cudaMallocAsync(&r, reserve, s->pool, s->stream) == cudaSuccess)
            cudaFreeAsync(r, s->stream);
        cudaGetLastError();
        pf_unicycle_params up;
        pf_dharm_params ap;
        pf_refarm_params rp;
        pf_beacon_params bp;
        pf_camarm_params cp;
        pf_unicycle_default_params(1, 4, &up);
        pf_dharm_default_params(1, &ap);
        pf_camarm_default_params(&cp);
        pf_beacon_default_params(&bp);
        memset(&rp, 0, sizeof(rp));
        rp.dt = cp.dt;
        memcpy(rp.init_state, cp.init_state, sizeof(rp.init_state));
        const void* params[PF_NUM_MODELS] = {&up, &ap, &rp, &bp, &cp};
        const size_t sizes[PF_NUM_MODELS] = {sizeof(up), sizeof(ap), sizeof(rp), sizeof(bp), sizeof(cp)};
        static_assert(PF_MODEL_REFARM == 2 && PF_MODEL_BEACON == 3 && PF_MODEL_CAMARM == 4, "warm-up table order");
        pf_step_input in;
        memset(&in, 0, sizeof(in));
        pf_server_result res;
        for (int m = 0; m < PF_NUM_MODELS; ++m) {
            int32_t id = -1, n = 0;
            pf_status w = pf_server_open(s, (pf_model_id)m, params[m], sizes[m], M, 1u, &id);
            if (w == PF_ERR_ADMISSION) continue;  // a budget below one filter: nothing to warm
            if (w == PF_OK) w = pf_server_update(s, id, &in, 0);
            if (w == PF_OK) w = pf_server_launch(s, &n);
            if (w == PF_OK) w = pf_server_poll(s, 1, &res, 1, &n);
            if (id >= 0) pf_server_close(s, id);
            if (w != PF_OK) {
                srv_release(s);
                return w;
            }
        }
        s->launches = s->updates = s->particle_steps = 0;
        if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
            srv_release(s);
            return fail(PF_ERR_CUDA, "server warm-up failed");
        }
    }
    *out = s;
    return PF_OK;
}

extern "C" pf_status pf_server_destroy(pf_server* s)
{
    if (!s) return PF_OK;
    cudaSetDevice(s->device);
    srv_release(s);
    return PF_OK;
}

// CTA-map capacity: every open filter's sub-filters fit in each model's map.
// The maps come from the stream-ordered pool: a grown map replaces the old one
// in stream order (the batches already queued keep reading the old one), so
// admission never waits for the GPU.
static pf_status ensure_map(pf_server* s, int64_t need)
{
    if (need <= s->map_cap) return PF_OK;
    const int64_t cap = std::max<int64_t>(need, 4 * s->map_cap);
    for (int m = 0; m < PF_NUM_MODELS; ++m) {
        if (s->d_map[m]) CU(cudaFreeAsync(s->d_map[m], s->stream));
        s->d_map[m] = nullptr;
        CU(cudaMallocAsync(reinterpret_cast<void**>(&s->d_map[m]), sizeof(int2) * cap, s->pool, s->stream));
    }
    s->map_cap = cap;
    return PF_OK;
}

extern "C" int64_t pf_server_footprint(const pf_server* s, pf_model_id model, int32_t num_particles)
{
    ModelInfo mi;
    if (!s || !model_info(model, &mi) || (int)model >= PF_NUM_MODELS) return -1;
    const int M = s->cfg.particles_per_subfilter;
    if (num_particles < M || num_particles % M) return -1;
    const int N = num_particles / M;
    return (int64_t)layout_of(mi.S, M, N, s->draws[model] - s->nbm[model]).total;
}

extern "C" pf_status pf_server_open(pf_server* s, pf_model_id model, const void* params, size_t params_size,
                                    int32_t num_particles, uint32_t seed, int32_t* id)
{
    if (!s || !params || !id) return fail(PF_ERR_INVALID, "null argument");
    *id = -1;
    ModelInfo mi;
    if (!model_info(model, &mi)) return fail(PF_ERR_INVALID, "unknown model %d", (int)model);
    if ((int)model >= PF_NUM_MODELS)
        return fail(PF_ERR_UNSUPPORTED, "the server runs the built-in models (0..%d); model %d is registered only "
                                        "for pf_create and batches", PF_NUM_MODELS - 1, (int)model);
    if (params_size != mi.psize) return fail(PF_ERR_INVALID, "model params size %zu, expected %zu", params_size, mi.psize);
    const int M = s->cfg.particles_per_subfilter;
    if (num_particles < M || num_particles % M)
        return fail(PF_ERR_INVALID, "%d particles is not a positive multiple of m=%d", num_particles, M);
    const int N = num_particles / M;
    if (s->cfg.exchange == PF_EXCHANGE_RING && 2 * s->cfg.num_transfer > M) return fail(PF_ERR_INVALID, "2*t > m");
    ModelParams mp;
    memset(&mp, 0, sizeof(mp));
    memcpy(&mp, params, params_size);
    if (model == PF_MODEL_UNICYCLE) {
        const pf_unicycle_params& p = mp.uni;
        if (p.num_landmarks < 1 || p.num_landmarks > 8 || !(p.sigma_range > 0) || !(p.sigma_bearing > 0))
            return fail(PF_ERR_INVALID, "1..8 landmarks and positive sigmas");
    } else if (model == PF_MODEL_DHARM) {
        if (!(mp.arm.sigma_pos > 0) || !(mp.arm.sigma_ang > 0)) return fail(PF_ERR_INVALID, "sigmas must be > 0");
    } else if (model == PF_MODEL_BEACON) {
        if (mp.bcn.num_beacons < 1 || mp.bcn.num_beacons > 16 || !(mp.bcn.sigma_range > 0))
            return fail(PF_ERR_INVALID, "1..16 beacons and a positive sigma");
    }
    const int64_t ru_stride = s->draws[model] - s->nbm[model];
    const Layout L = layout_of(mi.S, M, N, ru_stride);
    if (s->free_slots.empty()) return fail(PF_ERR_ADMISSION, "all %d filter slots are in use", s->max_filters);
    if (s->used + (int64_t)L.total > s->budget)
        return fail(PF_ERR_ADMISSION, "filter needs %zu bytes, %lld of %lld in use", L.total, (long long)s->used,
                    (long long)s->budget);
    CU(cudaSetDevice(s->device));
    pf_status st = ensure_map(s, s->resident_sub + N + estimate_ctas(N));
    if (st != PF_OK) return st;
    void* mem = nullptr;
    cudaError_t e = cudaMallocAsync(&mem, L.total, s->pool, s->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PF_ERR_ADMISSION, "device memory exhausted (%s)", cudaGetErrorString(e));
    }
    char* base = static_cast<char*>(mem);
    FilterDesc D;  // copied from pageable memory: staged before cudaMemcpyAsync returns
    memset(&D, 0, sizeof(D));
    D.T = (int64_t)M * N;
    D.state = reinterpret_cast<float*>(base + L.state);
    D.tmp = reinterpret_cast<float*>(base + L.tmp);
    D.tkey = reinterpret_cast<float*>(base + L.tkey);
    D.winner = reinterpret_cast<float*>(base + L.winner);
    D.part = reinterpret_cast<double*>(base + L.part);
    D.mtgp = reinterpret_cast<uint32_t*>(base + L.mtgp);
    D.ru = reinterpret_cast<float*>(base + L.ru);
    D.gpart = reinterpret_cast<double*>(base + L.gpart);
    D.est_ctr = reinterpret_cast<int32_t*>(base + L.est_ctr);
    D.status = s->d_status;
    const int slot = s->free_slots.back();
    D.est = s->d_est_tab + slot;
    D.N = N;
    D.M = M;
    D.t = s->cfg.exchange == PF_EXCHANGE_NONE ? 0 : s->cfg.num_transfer;
    D.exchange = s->cfg.exchange;
    D.resampler = s->cfg.resampler;
    torus_dims(N, &D.dx, &D.dy);
    D.log_weights = s->cfg.log_weights ? 1 : 0;
    D.inplace = (s->cfg.resampling_freq < 1.0f || s->cfg.ess_fraction > 0.0f) ? 1 : 0;
    D.rng_fused = 1;
    D.draws = (int32_t)s->draws[model];
    D.nbm = (int32_t)s->nbm[model];
    D.ru_stride = (int32_t)ru_stride;
    D.mask = s->cfg.mtgp_mask;
    D.stream_base = 0;
    D.exch_period = 1;
    D.freq = s->cfg.resampling_freq;
    D.ess_frac = s->cfg.ess_fraction;
    D.nnorm = (int64_t)mi.K * D.T;
    D.angle_mask = angle_mask_of(model);
    D.na = angle_count_of(model);
    D.mp = mp;
    // MTGP32 streams: sub-filter b uses parameter set b mod 200 and seed + b + 1
    e = launch_mtgp_init(D.mtgp, N, 0, seed, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_desc + slot, &D, sizeof(D), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(D.est_ctr, 0, 4, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(base + L.init, init_state_of(model, mp), 4 * (size_t)mi.S, cudaMemcpyHostToDevice,
                            s->stream);
    if (e == cudaSuccess) {
        k_srv_fill<<<std::min<int64_t>((D.T + 255) / 256, 1184), 256, 0, s->stream>>>(
            s->d_desc, slot, reinterpret_cast<const float*>(base + L.init), mi.S);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        cudaFreeAsync(mem, s->stream);
        return fail(PF_ERR_CUDA, "open: %s", cudaGetErrorString(e));
    }
    s->free_slots.pop_back();
    Slot& sl = s->slots[slot];
    sl.open = true;
    sl.model = model;
    sl.N = N;
    sl.T = D.T;
    sl.bytes = L.total;
    sl.mem = base;
    sl.in_flight = false;
    sl.in_ready = false;
    sl.steps = 0;
    sl.queue.clear();
    s->used += (int64_t)L.total;
    s->n_open++;
    s->resident_T += D.T;
    s->resident_sub += N + estimate_ctas(N);  // map entries: sub-filters and estimate CTAs
    *id = slot;
    return PF_OK;
}

extern "C" pf_status pf_server_close(pf_server* s, int32_t id)
{
    if (!s || id < 0 || id >= s->max_filters || !s->slots[id].open) return fail(PF_ERR_NOT_FOUND, "no open filter %d", id);
    CU(cudaSetDevice(s->device));
    Slot& sl = s->slots[id];
    if (sl.in_flight) return fail(PF_ERR_BUSY, "filter %d has an update in flight (poll first)", id);
    CU(cudaFreeAsync(sl.mem, s->stream));  // stream-ordered: reused only after the work queued before
    s->used -= (int64_t)sl.bytes;
    s->n_open--;
    s->resident_T -= sl.T;
    s->resident_sub -= sl.N + estimate_ctas(sl.N);
    s->queued -= (int64_t)sl.queue.size();
    sl = Slot();
    s->free_slots.push_back(id);
    return PF_OK;
}

extern "C" pf_status pf_server_update(pf_server* s, int32_t id, const pf_step_input* in, uint64_t tag)
{
    if (!s || !in) return fail(PF_ERR_INVALID, "null argument");
    if (id < 0 || id >= s->max_filters || !s->slots[id].open) return fail(PF_ERR_NOT_FOUND, "no open filter %d", id);
    Slot& sl = s->slots[id];
    sl.queue.emplace_back(*in, tag);
    s->queued++;
    if (!sl.in_flight && !sl.in_ready) {
        s->ready[sl.model].push_back(id);
        sl.in_ready = true;
    }
    return PF_OK;
}

extern "C" pf_status pf_server_launch(pf_server* s, int32_t* n_launched)
{
    if (!s || !n_launched) return fail(PF_ERR_INVALID, "null argument");
    *n_launched = 0;
    if (s->busy) return PF_OK;  // one batch in flight at a time
    CU(cudaSetDevice(s->device));
    int n = 0;
    int64_t ctas[PF_NUM_MODELS] = {}, ests[PF_NUM_MODELS] = {};
    s->batch_slots.clear();
    s->batch_tags.clear();
    // group the batch by model so each model's kernels see one contiguous CTA map
    for (int m = 0; m < PF_NUM_MODELS; ++m) {
        const int first = n;
        int64_t leads = 0;
        for (const int i : s->ready[m]) {
            Slot& sl = s->slots[i];
            sl.in_ready = false;
            if (!sl.open || sl.model != m || sl.in_flight || sl.queue.empty()) continue;  // closed since
            s->h_pend[n] = Pending{i, (int32_t)leads, 0};
            s->h_in[n] = sl.queue.front().first;
            s->batch_slots.push_back(i);
            s->batch_tags.push_back(sl.queue.front().second);
            sl.queue.pop_front();
            s->queued--;
            sl.in_flight = true;
            leads += estimate_ctas(sl.N);
            ctas[m] += sl.N;
            ++n;
        }
        s->ready[m].clear();
        ests[m] = leads;
        int64_t rest = leads;  // the sub-filters follow all of the model's estimate CTAs
        for (int q = first; q < n; ++q) {
            s->h_pend[q].first_rest = (int32_t)rest;
            rest += s->slots[s->h_pend[q].slot].N;
        }
    }
    if (n == 0) return PF_OK;
    const int M = s->cfg.particles_per_subfilter;
    cudaStream_t st = s->stream;
    CU(cudaMemcpyAsync(s->d_pend, s->h_pend, sizeof(Pending) * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(s->d_in, s->h_in, sizeof(pf_step_input) * n, cudaMemcpyHostToDevice, st));
    // one expand launch per model group (each writes its own map), each group
    // on its model's stream after everything queued on `stream` so far
    CU(cudaEventRecord(s->fork, st));
    bool used[PF_NUM_MODELS] = {};
    int first = 0;
    for (int m = 0; m < PF_NUM_MODELS; ++m) {
        int cnt = 0;
        while (first + cnt < n && s->slots[s->h_pend[first + cnt].slot].model == m) ++cnt;
        if (cnt == 0) continue;
        cudaStream_t ms = s->side[m];
        CU(cudaStreamWaitEvent(ms, s->fork, 0));
        k_srv_expand<<<cnt, 128, 0, ms>>>(s->d_pend + first, s->d_in + first, cnt, s->d_desc, s->d_slot_in,
                                          s->d_map[m]);
        CU(cudaGetLastError());
        const ModelOps ops = model_ops(m);
        const int E = s->E[m];
        InputRef ir{s->d_slot_in, 1, nullptr, 0, 0};
        CU(ops.sample_sort(M, E, 1, true, (int)ctas[m], ms, s->d_desc, s->d_map[m] + ests[m], ir));
        ModelInfo mi;
        model_info(m, &mi);
        const int virt = dependent_launch_pays((int)ctas[m], M, E, mi.S, s->device) ? 3 : 1;
        CU(ops.exchange_resample(M, E, s->cfg.resampler, (int)(ests[m] + ctas[m]), ms, s->d_desc, s->d_map[m], ir,
                                 nullptr, virt));
        CU(cudaEventRecord(s->join[m], ms));
        used[m] = true;
        first += cnt;
    }
    for (int m = 0; m < PF_NUM_MODELS; ++m)
        if (used[m]) CU(cudaStreamWaitEvent(st, s->join[m], 0));
    k_srv_gather<<<n + 1, 64, 0, st>>>(s->d_pend, n, s->d_est_tab, s->d_out, s->d_status);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(s->h_out, s->d_out, sizeof(pf_estimate) * n + sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CU(cudaEventRecord(s->done, st));
    s->busy = true;
    s->launches++;
    *n_launched = n;
    return PF_OK;
}

extern "C" pf_status pf_server_poll(pf_server* s, int32_t wait, pf_server_result* out, int32_t cap, int32_t* n)
{
    if (!s || !n || (cap > 0 && !out)) return fail(PF_ERR_INVALID, "null argument");
    *n = 0;
    if (!s->busy) return PF_OK;
    CU(cudaSetDevice(s->device));
    if (wait) {
        CU(cudaEventSynchronize(s->done));
    } else {
        const cudaError_t e = cudaEventQuery(s->done);
        if (e == cudaErrorNotReady) {
            cudaGetLastError();
            return PF_OK;
        }
        if (e != cudaSuccess) return fail(PF_ERR_CUDA, "poll: %s", cudaGetErrorString(e));
    }
    const int nb = (int)s->batch_slots.size();
    if (cap < nb) return fail(PF_ERR_INVALID, "result buffer holds %d, the batch has %d", cap, nb);
    if (*reinterpret_cast<const int32_t*>(s->h_out + nb) & PF_STATUS_MISALIGNED)
        return fail(PF_ERR_INVALID, "a sorted copy's rows were not 16-byte aligned (sub-filters kept their "
                                    "propagated particles)");
    if (*reinterpret_cast<const int32_t*>(s->h_out + nb) & PF_STATUS_WAIT_TIMEOUT)
        return fail(PF_ERR_TIMEOUT, "a bounded wait for a bulk copy ran out in a kernel (sub-filters kept their "
                                    "propagated particles)");
    for (int i = 0; i < nb; ++i) {
        Slot& sl = s->slots[s->batch_slots[i]];
        sl.in_flight = false;
        sl.steps++;
        if (!sl.queue.empty() && !sl.in_ready) {
            s->ready[sl.model].push_back(s->batch_slots[i]);
            sl.in_ready = true;
        }
        out[i].filter = s->batch_slots[i];
        out[i].step = sl.steps;
        out[i].tag = s->batch_tags[i];
        out[i].particles = sl.T;
        out[i].estimate = s->h_out[i];
        out[i].estimate.step = sl.steps;
        s->particle_steps += sl.T;
    }
    s->updates += nb;
    s->busy = false;
    *n = nb;
    return PF_OK;
}

extern "C" pf_status pf_server_stats_get(pf_server* s, pf_server_stats* st)
{
    if (!s || !st) return fail(PF_ERR_INVALID, "null argument");
    memset(st, 0, sizeof(*st));
    st->open_filters = (int32_t)s->n_open;
    st->resident_particles = s->resident_T;
    st->queued_updates = s->queued;
    st->bytes_in_use = s->used;
    st->budget = s->budget;
    st->launches = s->launches;
    st->updates = s->updates;
    st->particle_steps = s->particle_steps;
    st->in_flight = s->busy ? (int32_t)s->batch_slots.size() : 0;
    return PF_OK;
}

extern "C" pf_status pf_server_get_particles(pf_server* s, int32_t id, float* soa, float* sorted_soa, float* keys)
{
    if (!s) return fail(PF_ERR_INVALID, "null argument");
    if (id < 0 || id >= s->max_filters || !s->slots[id].open) return fail(PF_ERR_NOT_FOUND, "no open filter %d", id);
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    FilterDesc D;
    CU(cudaMemcpy(&D, s->d_desc + id, sizeof(D), cudaMemcpyDeviceToHost));
    ModelInfo mi;
    model_info(s->slots[id].model, &mi);
    if (soa) CU(cudaMemcpy(soa, D.state, 4 * (size_t)mi.S * D.T, cudaMemcpyDeviceToHost));
    if (sorted_soa) CU(cudaMemcpy(sorted_soa, D.tmp, 4 * (size_t)mi.S * D.T, cudaMemcpyDeviceToHost));
    if (keys) CU(cudaMemcpy(keys, D.tkey, 4 * (size_t)D.T, cudaMemcpyDeviceToHost));
    return PF_OK;
}

// ---------------------------------------------------------------------------
// per-filter snapshot / restore
// layout: int64 header[4] = {magic, model, T, N}, state S*T floats, stream
// words N*351, int32 updates completed.
// ---------------------------------------------------------------------------
static const int64_t kSrvSnapMagic = 0x5046535256534e31LL;

static pf_status idle_filter(const pf_server* s, int32_t id)
{
    if (!s) return fail(PF_ERR_INVALID, "null argument");
    if (id < 0 || id >= s->max_filters || !s->slots[id].open) return fail(PF_ERR_NOT_FOUND, "no open filter %d", id);
    const Slot& sl = s->slots[id];
    if (sl.in_flight || !sl.queue.empty()) return fail(PF_ERR_BUSY, "filter %d has updates queued or in flight", id);
    return PF_OK;
}

extern "C" int64_t pf_server_snapshot_size(const pf_server* s, int32_t id)
{
    if (!s || id < 0 || id >= s->max_filters || !s->slots[id].open) return -1;
    const Slot& sl = s->slots[id];
    ModelInfo mi;
    model_info(sl.model, &mi);
    return 32 + 4 * (int64_t)mi.S * sl.T + 4 * (int64_t)sl.N * kMtgpN + 4;
}

extern "C" pf_status pf_server_snapshot(pf_server* s, int32_t id, void* buf)
{
    pf_status st = idle_filter(s, id);
    if (st != PF_OK) return st;
    if (!buf) return fail(PF_ERR_INVALID, "null argument");
    const Slot& sl = s->slots[id];
    ModelInfo mi;
    model_info(sl.model, &mi);
    const Layout L = layout_of(mi.S, s->cfg.particles_per_subfilter, sl.N, s->draws[sl.model] - s->nbm[sl.model]);
    CU(cudaSetDevice(s->device));
    char* p = static_cast<char*>(buf);
    const int64_t hdr[4] = {kSrvSnapMagic, sl.model, sl.T, sl.N};
    memcpy(p, hdr, 32);
    p += 32;
    const size_t sb = 4 * (size_t)mi.S * sl.T, mb = 4 * (size_t)sl.N * kMtgpN;
    CU(cudaMemcpyAsync(p, sl.mem + L.state, sb, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(p + sb, sl.mem + L.mtgp, mb, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    memcpy(p + sb + mb, &sl.steps, 4);
    return PF_OK;
}

extern "C" pf_status pf_server_restore(pf_server* s, int32_t id, const void* buf, size_t size)
{
    pf_status st = idle_filter(s, id);
    if (st != PF_OK) return st;
    if (!buf) return fail(PF_ERR_INVALID, "null argument");
    const int64_t want = pf_server_snapshot_size(s, id);
    if (size < 32 || (int64_t)size != want)
        return fail(PF_ERR_INVALID, "snapshot of %zu bytes; filter %d takes %lld", size, id, (long long)want);
    Slot& sl = s->slots[id];
    const char* p = static_cast<const char*>(buf);
    int64_t hdr[4];
    memcpy(hdr, p, 32);
    if (hdr[0] != kSrvSnapMagic || hdr[1] != sl.model || hdr[2] != sl.T || hdr[3] != sl.N)
        return fail(PF_ERR_INVALID, "snapshot does not match filter %d (model, particle count)", id);
    p += 32;
    ModelInfo mi;
    model_info(sl.model, &mi);
    const Layout L = layout_of(mi.S, s->cfg.particles_per_subfilter, sl.N, s->draws[sl.model] - s->nbm[sl.model]);
    CU(cudaSetDevice(s->device));
    const size_t sb = 4 * (size_t)mi.S * sl.T, mb = 4 * (size_t)sl.N * kMtgpN;
    // pageable source: each copy is staged before the call returns, and runs
    // in stream order before any later batch of this filter
    CU(cudaMemcpyAsync(sl.mem + L.state, p, sb, cudaMemcpyHostToDevice, s->stream));
    CU(cudaMemcpyAsync(sl.mem + L.mtgp, p + sb, mb, cudaMemcpyHostToDevice, s->stream));
    int32_t steps = 0;
    memcpy(&steps, p + sb + mb, 4);
    sl.steps = steps;
    return PF_OK;
}
