// pf_api.cu -- the C ABI (include/esthera_b200.h): filter lifecycle, device
// memory, the per-step launch sequence, CUDA-graph replay, snapshot/restore
// and the kernel-level entry points used by the parity tests.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_set>
#include <atomic>
#include <vector>

#include "pf_host.cuh"

using namespace pfdev;
using namespace pfhost;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

pf_status pfhost::fail(pf_status s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

extern "C" const char* pf_last_error(void) { return g_err.c_str(); }

pf_status pfi_fail(pf_status s, const char* msg) { return fail(s, "%s", msg); }

extern "C" const char* pf_status_string(pf_status s)
{
    switch (s) {
    case PF_OK: return "ok";
    case PF_ERR_INVALID: return "invalid argument";
    case PF_ERR_CUDA: return "CUDA error";
    case PF_ERR_NOMEM: return "out of memory";
    case PF_ERR_UNSUPPORTED: return "unsupported configuration";
    case PF_ERR_IO: return "I/O error";
    case PF_ERR_ADMISSION: return "admission rejected";
    case PF_ERR_TIMEOUT: return "timeout";
    case PF_ERR_NOT_FOUND: return "not found";
    case PF_ERR_BUSY: return "busy";
    }
    return "unknown";
}

extern "C" int32_t pf_version(void) { return 100; }

extern "C" int32_t pf_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

pf_status pfhost::require_gpu(int device)
{
    const int n = pf_device_count();
    if (n <= 0) return fail(PF_ERR_CUDA, "no CUDA device available (this engine has no CPU path)");
    if (device < 0 || device >= n) return fail(PF_ERR_INVALID, "device %d out of range (%d devices)", device, n);
    CU(cudaSetDevice(device));
    return PF_OK;
}

// ---------------------------------------------------------------------------
// model table
// ---------------------------------------------------------------------------

// The registry: a fixed table filled by the registrations that run when the
// library is loaded (PF_REGISTER_MODEL / PF_MODEL), read-only afterwards.
namespace {
constexpr int kMaxModels = 64;
struct Registry {
    std::mutex mu;
    pfhost::ModelEntry e[kMaxModels];
    int n = 0;
};
Registry& registry()
{
    static Registry r;
    return r;
}
}  // namespace

bool pfhost::register_model(const ModelEntry& e)
{
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    if (e.id < 0 || r.n >= kMaxModels) return false;
    for (int i = 0; i < r.n; ++i)
        if (r.e[i].id == e.id) return false;
    r.e[r.n++] = e;
    return true;
}

const pfhost::ModelEntry* pfhost::find_model(int id)
{
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    for (int i = 0; i < r.n; ++i)
        if (r.e[i].id == id) return &r.e[i];
    return nullptr;
}

int pfhost::registered_models(int* ids, int cap)
{
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    for (int i = 0; i < r.n && i < cap; ++i) ids[i] = r.e[i].id;
    return r.n;
}

bool pfhost::model_info(int model, ModelInfo* mi)
{
    const ModelEntry* e = find_model(model);
    if (!e) return false;
    *mi = e->info;
    return true;
}

bool pfhost::dependent_launch_pays(int grid, int M, int E, int S, int device)
{
    static std::atomic<int> sms[64] = {};  // SM count per device, read once (any thread)
    if (device < 0 || device >= 64) return false;
    int n = sms[device].load(std::memory_order_relaxed);
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        sms[device].store(n, std::memory_order_relaxed);
    }
    return grid > n * pf_min_blocks(M / E, pf_k1_warps(S, E));
}

extern "C" pf_status pf_model_info(pf_model_id model, int32_t* S, int32_t* K, int32_t* C, int32_t* Z)
{
    ModelInfo mi;
    if (!model_info(model, &mi)) return fail(PF_ERR_INVALID, "unknown model %d", (int)model);
    if (S) *S = mi.S;
    if (K) *K = mi.K;
    if (C) *C = mi.C;
    if (Z) *Z = mi.Z;
    return PF_OK;
}

const float* pfhost::init_state_of(int model, const ModelParams& mp)
{
    const ModelEntry* e = find_model(model);
    return reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(&mp) + (e ? e->init_offset : 0));
}

uint32_t pfhost::angle_mask_of(int model)
{
    const ModelEntry* e = find_model(model);
    return e ? e->angle_mask : 0u;
}

int pfhost::angle_count_of(int model)
{
    const ModelEntry* e = find_model(model);
    return e ? e->angle_count : 0;
}

ModelOps pfhost::model_ops(int model)
{
    const ModelEntry* e = find_model(model);
    return e ? e->ops : ModelOps{};
}

extern "C" int32_t pf_model_list(int32_t* ids, int32_t cap)
{
    std::vector<int> v(kMaxModels);
    const int n = registered_models(v.data(), kMaxModels);
    for (int i = 0; i < n && i < cap && ids; ++i) ids[i] = v[i];
    return n;
}

extern "C" const char* pf_model_name(int32_t model)
{
    const ModelEntry* e = find_model(model);
    return e ? e->name : nullptr;
}

// ---------------------------------------------------------------------------
// MTGP32 stream initialisation on the host (mtgp32_init_state,
// src/partfilt/cuda/mtgp/mtgp32-fast.c:119-137): the same 351 words the
// reference seeds stream g with (seed + g + 1).
// ---------------------------------------------------------------------------
static const uint32_t kHostParams[200 * 52] = {
#include "mtgp32_params_11213.inc"
};

void pfhost::mtgp_init_state_host(uint32_t* st, int set, uint32_t seed)
{
    const uint32_t* tbl = kHostParams + set * 52 + 4;
    const uint32_t hidden = tbl[4] ^ (tbl[8] << 16);
    uint32_t tmp = hidden;
    tmp += tmp >> 16;
    tmp += tmp >> 8;
    const uint32_t b = tmp & 0xffu;
    const uint32_t fill = b | (b << 8) | (b << 16) | (b << 24);
    for (int i = 0; i < kMtgpN; ++i) st[i] = fill;
    st[0] = seed;
    st[1] = hidden;
    for (int i = 1; i < kMtgpN; ++i) st[i] ^= 1812433253u * (st[i - 1] ^ (st[i - 1] >> 30)) + (uint32_t)i;
}

// ---------------------------------------------------------------------------
// filter
// ---------------------------------------------------------------------------
struct pf_filter {
    pf_config cfg;
    int model;
    ModelParams mp;
    ModelInfo mi;
    ModelOps ops;
    int M, E, N, t, dx, dy, streams, na, pipe;
    int tp = 1;  // threads per particle of the sampling kernel
    StepState X{};
    uint32_t angle_mask;
    int64_t T, rtotal, draws, nbm;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    float *state = nullptr, *tmp = nullptr, *tkey = nullptr, *key = nullptr, *winner = nullptr, *ru = nullptr,
          *rbuf = nullptr;
    double* part = nullptr;
    uint32_t* mtgp = nullptr;
    int32_t *a2a = nullptr, *sel = nullptr, *ctr = nullptr, *est_ctr = nullptr;
    double* gpart = nullptr;
    pf_estimate* d_est = nullptr;
    pf_step_input* d_in = nullptr;
    FilterDesc* d_desc = nullptr;  // [0]: pf_step, [1]: pf_run_device
    FilterDesc h_desc;
    pf_estimate* h_est = nullptr;
    pf_step_input* h_in = nullptr;
    int64_t dev_bytes = 0;
    int32_t steps_done = 0;
    cudaGraphExec_t graph = nullptr;
    const pf_step_input* graph_inputs = nullptr;
    pf_estimate* graph_est = nullptr;
    int32_t graph_cap = 0;
    // submit / collect queue (pf_step_submit): pinned and device rings of
    // inputs and estimates, an upload and a download stream, events per slot
    pf_step_input *h_q_in = nullptr, *d_q_in = nullptr;
    pf_estimate *h_q_est = nullptr, *d_q_est = nullptr;
    cudaStream_t q_up = nullptr, q_down = nullptr;
    cudaEvent_t q_ev_up[PF_QUEUE_DEPTH] = {}, q_ev_done[PF_QUEUE_DEPTH] = {}, q_ev_got[PF_QUEUE_DEPTH] = {};
    int q_active = 0;   // the device counter holds q_next (else set it before the next submit)
    int q_pending = 0;  // submitted, not yet collected
    int32_t q_next = 0; // step number (and slot, modulo the depth) of the next submit
    // a shard of a larger filter (pf_shard_*): global sub-filters b0 ..
    // b0 + N - 1 (rows r0 .. of the global dx x gdy torus of gN sub-filters)
    int shard = 0, b0 = 0, r0 = 0, gdy = 0, gN = 0;
    float *halo_in = nullptr, *halo_out = nullptr;  // [2][1+S][dx*t] each
    double* rows = nullptr;                         // the last step's group rows [ng][kPartStride]
    float* states = nullptr;                        // and their winners' states [ng][S]
    cudaEvent_t ev_sampled = nullptr;
    // per-phase timing: events recorded between the launches of a step
    int timing = 0;
    cudaEvent_t ev[8] = {};
    const char* phase[8] = {};
    int nphase = 0;
};

template <class T>
static pf_status dalloc(pf_filter* f, T** p, size_t count)
{
    void* q = nullptr;
    const size_t bytes = count * sizeof(T);
    if (bytes == 0) {
        *p = nullptr;
        return PF_OK;
    }
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PF_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    f->allocs.push_back(q);
    f->dev_bytes += (int64_t)bytes;
    *p = static_cast<T*>(q);
    return PF_OK;
}

static void release(pf_filter* f)
{
    if (!f) return;
    if (f->graph) cudaGraphExecDestroy(f->graph);
    if (f->ev_sampled) cudaEventDestroy(f->ev_sampled);
    for (cudaEvent_t e : f->ev)
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < PF_QUEUE_DEPTH; ++i) {
        if (f->q_ev_up[i]) cudaEventDestroy(f->q_ev_up[i]);
        if (f->q_ev_done[i]) cudaEventDestroy(f->q_ev_done[i]);
        if (f->q_ev_got[i]) cudaEventDestroy(f->q_ev_got[i]);
    }
    if (f->q_up) cudaStreamDestroy(f->q_up);
    if (f->q_down) cudaStreamDestroy(f->q_down);
    if (f->h_q_in) cudaFreeHost(f->h_q_in);
    if (f->h_q_est) cudaFreeHost(f->h_q_est);
    for (void* p : f->allocs) cudaFree(p);
    if (f->h_est) cudaFreeHost(f->h_est);
    if (f->h_in) cudaFreeHost(f->h_in);
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
}

extern "C" pf_status pf_config_default(pf_config* c)
{
    if (!c) return fail(PF_ERR_INVALID, "null config");
    memset(c, 0, sizeof(*c));
    c->particles_per_subfilter = 512;
    c->num_subfilters = 16;
    c->num_transfer = 1;
    c->exchange = PF_EXCHANGE_RING;
    c->resampler = PF_RESAMPLE_SYSTEMATIC;
    c->resampling_freq = 1.0f;
    c->seed = 0xF000000Du;
    c->rng = PF_RNG_SUBFILTER;
    c->mtgp_streams = 96;
    c->mtgp_mask = PF_MTGP_MASK_PARAMS;
    c->log_weights = 1;
    c->pipeline = PF_PIPELINE_FUSED;
    c->particles_per_thread = 0;
    c->device = 0;
    c->stream_offset = 0;
    c->exchange_period = 1;
    c->ess_fraction = 0.0f;
    return PF_OK;
}

int pfhost::default_ppt(int M, int S)
{
    if (M <= 32) return 1;
    if (M <= 64) return 2;
    return S > 3 ? 2 : 4;  // large states: two particles per thread (pf_k1_warps)
}

void pfhost::torus_dims(int N, int* dx, int* dy)
{
    int x = 1;
    while ((int64_t)(2 * x) * (2 * x) <= N) x *= 2;
    *dx = x;
    *dy = N / x;
}

static pf_status validate(const pf_config* c, int model, const ModelInfo& mi, int* E)
{
    const int M = c->particles_per_subfilter;
    if (M < 32 || M > 1024 || (M & (M - 1)))
        return fail(PF_ERR_UNSUPPORTED, "particles per sub-filter must be a power of two in [32, 1024], got %d", M);
    if (c->num_subfilters < 1) return fail(PF_ERR_INVALID, "num_subfilters must be >= 1");
    if ((int64_t)M * c->num_subfilters > (int64_t)1 << 30) return fail(PF_ERR_INVALID, "too many particles");
    if (c->num_transfer < 0) return fail(PF_ERR_INVALID, "num_transfer must be >= 0");
    if (c->exchange < PF_EXCHANGE_NONE || c->exchange > PF_EXCHANGE_ALL2ALL)
        return fail(PF_ERR_INVALID, "unknown exchange %d", c->exchange);
    if (c->exchange == PF_EXCHANGE_TORUS && 5 * c->num_transfer > M)
        return fail(PF_ERR_INVALID, "torus exchange needs 5*t <= m (t=%d, m=%d)", c->num_transfer, M);
    if (c->exchange == PF_EXCHANGE_TORUS) {
        int dx, dy;
        torus_dims(c->num_subfilters, &dx, &dy);
        if (dx * dy != c->num_subfilters)
            return fail(PF_ERR_INVALID, "torus exchange needs N = dx*dy with dx = 2^floor(log2 sqrt N) (N=%d)",
                        c->num_subfilters);
    }
    if ((c->exchange == PF_EXCHANGE_RING || c->exchange == PF_EXCHANGE_ALL2ALL) && 2 * c->num_transfer > M)
        return fail(PF_ERR_INVALID, "exchange needs 2*t <= m (t=%d, m=%d)", c->num_transfer, M);
    if (c->exchange == PF_EXCHANGE_ALL2ALL && (c->num_subfilters > 8192 || c->num_transfer > c->num_subfilters * M))
        return fail(PF_ERR_UNSUPPORTED, "all-to-all exchange supports at most 8192 sub-filters");
    if (c->resampler < PF_RESAMPLE_REFERENCE || c->resampler > PF_RESAMPLE_VOSE)
        return fail(PF_ERR_INVALID, "unknown resampler %d", c->resampler);
    if (!(c->resampling_freq >= 0.0f && c->resampling_freq <= 1.0f))
        return fail(PF_ERR_INVALID, "resampling_freq must be in [0, 1]");
    if (!(c->ess_fraction >= 0.0f && c->ess_fraction <= 1.0f))
        return fail(PF_ERR_INVALID, "ess_fraction must be in [0, 1]");
    if (c->rng != PF_RNG_SUBFILTER && c->rng != PF_RNG_REFLAYOUT) return fail(PF_ERR_INVALID, "unknown rng layout");
    if (c->stream_offset < 0) return fail(PF_ERR_INVALID, "stream_offset must be >= 0");
    if (c->exchange_period < 0) return fail(PF_ERR_INVALID, "exchange_period must be >= 0");
    if (c->exchange_period > 1 && c->pipeline == PF_PIPELINE_PHASED)
        return fail(PF_ERR_UNSUPPORTED, "the phased pipeline exchanges every step (exchange_period <= 1)");
    if (c->rng == PF_RNG_REFLAYOUT && (c->mtgp_streams < 1 || c->mtgp_streams > 200))
        return fail(PF_ERR_INVALID, "mtgp_streams must be in [1, 200]");
    if (c->pipeline == PF_PIPELINE_PHASED && c->rng != PF_RNG_REFLAYOUT)
        return fail(PF_ERR_INVALID, "the phased pipeline uses the reference RNG layout (rng = PF_RNG_REFLAYOUT)");
    if (c->pipeline != PF_PIPELINE_FUSED && c->pipeline != PF_PIPELINE_PHASED && c->pipeline != PF_PIPELINE_SPLIT)
        return fail(PF_ERR_INVALID, "unknown pipeline");
    *E = c->particles_per_thread > 0 ? c->particles_per_thread : default_ppt(M, mi.S);
    if (!me_supported(M, *E))
        return fail(PF_ERR_UNSUPPORTED, "particles per thread %d not built for m=%d", *E, M);
    if (c->threads_per_particle < 0 || c->threads_per_particle > 2)
        return fail(PF_ERR_INVALID, "threads_per_particle must be 1 or 2");
    if (c->threads_per_particle == 2 &&
        (c->rng != PF_RNG_SUBFILTER || c->pipeline == PF_PIPELINE_PHASED || 2 * M / *E > 1024))
        return fail(PF_ERR_UNSUPPORTED, "two threads per particle run the split pipeline with per-sub-filter "
                                        "streams and 2 m / ppt <= 1024 threads");
    (void)model;
    (void)mi;
    return PF_OK;
}

// The kernels' status word (PF_STATUS_* bits), stored right after the
// estimate so that pf_step's estimate copy brings it along.
static int32_t* status_word(pf_filter* f) { return reinterpret_cast<int32_t*>(f->d_est + 1); }

static pf_status check_status(int32_t st)
{
    if (st & PF_STATUS_MISALIGNED)
        return fail(PF_ERR_INVALID, "a sorted copy's rows were not 16-byte aligned (sub-filters kept their "
                                    "propagated particles)");
    if (st & PF_STATUS_WAIT_TIMEOUT)
        return fail(PF_ERR_TIMEOUT, "a bounded wait for a bulk copy ran out in a kernel (sub-filters kept their "
                                    "propagated particles)");
    return PF_OK;
}

static void fill_desc(pf_filter* f, FilterDesc& D, pf_estimate* est)
{
    memset(&D, 0, sizeof(D));
    D.state = f->state;
    D.tmp = f->tmp;
    D.tkey = f->tkey;
    D.key = f->key;
    D.winner = f->winner;
    D.part = f->part;
    D.mtgp = f->mtgp;
    D.ru = f->ru;
    D.rbuf = f->rbuf;
    D.a2a = f->a2a;
    D.sel = f->sel;
    D.est = est;
    D.T = f->T;
    D.N = f->N;
    D.M = f->M;
    D.t = f->t;
    D.exchange = f->cfg.exchange;
    D.resampler = f->cfg.resampler;
    D.dx = f->dx;
    D.dy = f->dy;
    D.log_weights = f->cfg.log_weights ? 1 : 0;
    D.inplace = (f->cfg.resampling_freq < 1.0f || f->cfg.ess_fraction > 0.0f || f->pipe == PF_PIPELINE_PHASED) ? 1 : 0;
    D.rng_fused = f->cfg.rng == PF_RNG_SUBFILTER ? 1 : 0;
    D.draws = (int32_t)f->draws;
    D.nbm = (int32_t)f->nbm;
    D.ru_stride = (int32_t)(f->draws - f->nbm);
    D.mask = f->cfg.mtgp_mask;
    D.stream_base = f->cfg.stream_offset;
    D.exch_period = f->cfg.exchange_period;
    D.freq = f->cfg.resampling_freq;
    D.ess_frac = f->cfg.ess_fraction;
    D.nnorm = (int64_t)f->mi.K * f->T;
    D.est_ctr = f->est_ctr;
    D.status = status_word(f);
    D.gpart = f->gpart;
    D.angle_mask = f->angle_mask;
    D.na = f->na;
    D.shard = f->shard;
    D.b0 = f->b0;
    D.r0 = f->r0;
    D.gdy = f->gdy;
    D.halo = f->halo_in;
    D.mp = f->mp;
}

static pf_status upload_descs(pf_filter* f, pf_estimate* run_est)
{
    FilterDesc d[2];
    fill_desc(f, d[0], f->d_est);
    fill_desc(f, d[1], run_est);
    f->h_desc = d[0];
    CU(cudaMemcpyAsync(f->d_desc, d, sizeof(d), cudaMemcpyHostToDevice, f->stream));
    CU(cudaStreamSynchronize(f->stream));
    return PF_OK;
}

int64_t pfhost::resample_draws(int res, int M)
{
    return res == PF_RESAMPLE_REFERENCE ? M : (res == PF_RESAMPLE_VOSE ? 2 * (int64_t)M : 1);
}

static pf_status init_streams(pf_filter* f)
{
    std::vector<uint32_t> st((size_t)f->streams * kMtgpN);
    const int off = f->cfg.rng == PF_RNG_SUBFILTER ? f->cfg.stream_offset : 0;
    for (int g = 0; g < f->streams; ++g)
        mtgp_init_state_host(st.data() + (size_t)g * kMtgpN, (off + g) % kMtgpSets,
                             f->cfg.seed + (uint32_t)(off + g) + 1u);
    CU(cudaMemcpy(f->mtgp, st.data(), st.size() * 4, cudaMemcpyHostToDevice));
    return PF_OK;
}

extern "C" pf_status pf_create(const pf_config* cfg, pf_model_id model, const void* params, size_t params_size,
                               pf_filter** out)
{
    if (!cfg || !out) return fail(PF_ERR_INVALID, "null argument");
    *out = nullptr;
    ModelInfo mi;
    if (!model_info(model, &mi)) return fail(PF_ERR_INVALID, "unknown model %d", (int)model);
    if (!params || params_size != mi.psize)
        return fail(PF_ERR_INVALID, "model params size %zu, expected %zu", params_size, mi.psize);
    int E = 0;
    pf_status s = validate(cfg, model, mi, &E);
    if (s != PF_OK) return s;
    if (model == PF_MODEL_UNICYCLE) {
        const pf_unicycle_params* p = (const pf_unicycle_params*)params;
        if (p->num_landmarks < 1 || p->num_landmarks > 8) return fail(PF_ERR_INVALID, "1..8 landmarks");
        if (!(p->sigma_range > 0) || !(p->sigma_bearing > 0)) return fail(PF_ERR_INVALID, "sigmas must be > 0");
    } else if (model == PF_MODEL_DHARM) {
        const pf_dharm_params* p = (const pf_dharm_params*)params;
        if (!(p->sigma_pos > 0) || !(p->sigma_ang > 0)) return fail(PF_ERR_INVALID, "sigmas must be > 0");
    } else if (model == PF_MODEL_BEACON) {
        const pf_beacon_params* p = (const pf_beacon_params*)params;
        if (p->num_beacons < 1 || p->num_beacons > 16) return fail(PF_ERR_INVALID, "1..16 beacons");
        if (!(p->sigma_range > 0)) return fail(PF_ERR_INVALID, "sigma_range must be > 0");
    }
    s = require_gpu(cfg->device);
    if (s != PF_OK) return s;

    pf_filter* f = new pf_filter();
    f->cfg = *cfg;
    f->model = model;
    memset(&f->mp, 0, sizeof(f->mp));
    memcpy(&f->mp, params, params_size);
    f->mi = mi;
    f->ops = model_ops(model);
    f->tp = cfg->threads_per_particle == 2 ? 2 : 1;
    f->pipe = (cfg->pipeline == PF_PIPELINE_FUSED && cfg->rng == PF_RNG_SUBFILTER && cfg->exchange_period <= 1 &&
               f->tp == 1)
                  ? PF_PIPELINE_FUSED
                  : (cfg->pipeline == PF_PIPELINE_PHASED ? PF_PIPELINE_PHASED : PF_PIPELINE_SPLIT);
    f->angle_mask = angle_mask_of(model);
    f->na = angle_count_of(model);
    f->M = cfg->particles_per_subfilter;
    f->E = E;
    f->N = cfg->num_subfilters;
    f->t = cfg->exchange == PF_EXCHANGE_NONE ? 0 : cfg->num_transfer;
    f->T = (int64_t)f->M * f->N;
    torus_dims(f->N, &f->dx, &f->dy);
    f->nbm = 2 * (((int64_t)mi.K * f->M + 1) / 2);
    f->draws = f->nbm + 1 + resample_draws(cfg->resampler, f->M);
    f->streams = cfg->rng == PF_RNG_SUBFILTER ? f->N : cfg->mtgp_streams;
    if (cfg->rng == PF_RNG_REFLAYOUT) {
        const int64_t nn = (int64_t)mi.K * f->T;
        const int64_t nu = cfg->resampler == PF_RESAMPLE_VOSE ? (int64_t)(2 * f->M + 1) * f->N
                                                              : (int64_t)(f->M + 1) * f->N;
        const int64_t unit = 768LL * cfg->mtgp_streams;
        f->rtotal = ((nn + nu + unit - 1) / unit) * unit;
        if (f->rtotal / cfg->mtgp_streams > INT32_MAX) {
            release(f);
            return fail(PF_ERR_UNSUPPORTED, "random buffer too large for the reference layout");
        }
    }
    cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        release(f);
        return fail(PF_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    const int S = mi.S;
#define TRY(x)                 \
    do {                       \
        pf_status s_ = (x);    \
        if (s_ != PF_OK) {     \
            release(f);        \
            return s_;         \
        }                      \
    } while (0)
    TRY(dalloc(f, &f->state, (size_t)S * f->T));
    TRY(dalloc(f, &f->tmp, (size_t)S * f->T));
    TRY(dalloc(f, &f->tkey, (size_t)f->T));
    if (cfg->pipeline == PF_PIPELINE_PHASED) TRY(dalloc(f, &f->key, (size_t)f->T));
    TRY(dalloc(f, &f->winner, (size_t)f->N));
    TRY(dalloc(f, &f->part, (size_t)f->N * kPartStride));
    TRY(dalloc(f, &f->mtgp, (size_t)f->streams * kMtgpN));
    if (cfg->rng == PF_RNG_SUBFILTER) TRY(dalloc(f, &f->ru, (size_t)f->N * (f->draws - f->nbm)));
    else TRY(dalloc(f, &f->rbuf, (size_t)f->rtotal));
    if (cfg->exchange == PF_EXCHANGE_ALL2ALL) TRY(dalloc(f, &f->a2a, (size_t)(f->t > 0 ? f->t : 1)));
    if (f->pipe == PF_PIPELINE_FUSED) {
        TRY(dalloc(f, &f->X.tmp2, (size_t)S * f->T));
        TRY(dalloc(f, &f->X.tkey2, (size_t)f->T));
        TRY(dalloc(f, &f->X.steps, 1));
        TRY(dalloc(f, &f->X.need_init, 1));
        TRY(dalloc(f, &f->X.grp_ctr, (size_t)((f->N + 31) / 32)));
        if (cudaMemset(f->X.steps, 0, 4) != cudaSuccess ||
            cudaMemset(f->X.grp_ctr, 0, (size_t)((f->N + 31) / 32) * 4) != cudaSuccess) {
            cudaGetLastError();
            release(f);
            return fail(PF_ERR_CUDA, "cudaMemset failed");
        }
    }
    TRY(dalloc(f, &f->ctr, 1));
    TRY(dalloc(f, &f->est_ctr, 1));
    TRY(dalloc(f, &f->gpart, (size_t)((f->N + 31) / 32) * kPartStride));
    TRY(dalloc(f, &f->d_est, 2));  // [0] the estimate, then the kernels' status word
    TRY(dalloc(f, &f->d_in, 1));
    TRY(dalloc(f, &f->d_desc, 2));
    if (cudaMallocHost(&f->h_est, 2 * sizeof(pf_estimate)) != cudaSuccess ||
        cudaMallocHost(&f->h_in, sizeof(pf_step_input)) != cudaSuccess) {
        cudaGetLastError();
        release(f);
        return fail(PF_ERR_NOMEM, "cudaMallocHost failed");
    }
    TRY(init_streams(f));
    if (cudaMemset(f->est_ctr, 0, 4) != cudaSuccess || cudaMemset(f->ctr, 0, 4) != cudaSuccess ||
        cudaMemset(f->d_est, 0, 2 * sizeof(pf_estimate)) != cudaSuccess) {
        cudaGetLastError();
        release(f);
        return fail(PF_ERR_CUDA, "cudaMemset failed");
    }
    TRY(upload_descs(f, nullptr));
    TRY(pf_set_initial_state(f, init_state_of(model, f->mp)));
#undef TRY
    *out = f;
    return PF_OK;
}

extern "C" pf_status pf_destroy(pf_filter* f)
{
    if (!f) return PF_OK;
    cudaSetDevice(f->cfg.device);
    cudaStreamSynchronize(f->stream);
    release(f);
    return PF_OK;
}

// Single-kernel pipeline: the next step starts from `state` instead of resampling.
static pf_status mark_need_init(pf_filter* f)
{
    if (f->pipe != PF_PIPELINE_FUSED) return PF_OK;
    const int32_t one = 1;
    CU(cudaMemcpy(f->X.need_init, &one, 4, cudaMemcpyHostToDevice));
    return PF_OK;
}

// Single-kernel pipeline: materialise the particles after the last step's
// resampling into `state` (deferred to the next step otherwise).
static pf_status materialise(pf_filter* f)
{
    if (f->pipe != PF_PIPELINE_FUSED) return PF_OK;
    InputRef none{nullptr, 0, nullptr, 0};
    CU(f->ops.step(f->M, f->E, f->cfg.resampler, f->N, f->stream, f->d_desc, f->X, none, nullptr, true));
    CU(cudaStreamSynchronize(f->stream));
    return PF_OK;
}

extern "C" pf_status pf_set_initial_state(pf_filter* f, const float* state)
{
    if (!f || !state) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    std::vector<float> h((size_t)f->mi.S * f->T);
    for (int v = 0; v < f->mi.S; ++v)
        for (int64_t i = 0; i < f->T; ++i) h[(size_t)v * f->T + i] = state[v];
    CU(cudaStreamSynchronize(f->stream));
    CU(cudaMemcpy(f->state, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
    f->steps_done = 0;
    f->q_active = 0;
    return mark_need_init(f);
}

extern "C" pf_status pf_set_particles(pf_filter* f, const float* soa)
{
    if (!f || !soa) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    CU(cudaMemcpy(f->state, soa, (size_t)f->mi.S * f->T * 4, cudaMemcpyHostToDevice));
    return mark_need_init(f);
}

extern "C" pf_status pf_get_particles(pf_filter* f, float* soa)
{
    if (!f || !soa) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    pf_status s = materialise(f);
    if (s != PF_OK) return s;
    CU(cudaMemcpy(soa, f->state, (size_t)f->mi.S * f->T * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pf_get_sorted(pf_filter* f, float* soa, float* keys)
{
    if (!f) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    const float* tmp = f->tmp;
    const float* tkey = f->tkey;
    if (f->pipe == PF_PIPELINE_FUSED) {  // the half written by the last step
        int32_t steps = 0;
        CU(cudaMemcpy(&steps, f->X.steps, 4, cudaMemcpyDeviceToHost));
        if (((steps & 1) ^ 1) == 1) {
            tmp = f->X.tmp2;
            tkey = f->X.tkey2;
        }
    }
    if (soa) CU(cudaMemcpy(soa, tmp, (size_t)f->mi.S * f->T * 4, cudaMemcpyDeviceToHost));
    if (keys) CU(cudaMemcpy(keys, tkey, (size_t)f->T * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pf_record_selection(pf_filter* f, int32_t enable)
{
    if (!f) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    if (enable && !f->sel) {
        pf_status s = dalloc(f, &f->sel, (size_t)f->T);
        if (s != PF_OK) return s;
    }
    if (!enable) f->sel = nullptr;  // the buffer stays allocated until destroy
    if (f->graph) {
        cudaGraphExecDestroy(f->graph);
        f->graph = nullptr;
    }
    return upload_descs(f, f->graph_est);
}

extern "C" pf_status pf_get_selection(pf_filter* f, int32_t* sel)
{
    if (!f || !sel) return fail(PF_ERR_INVALID, "null argument");
    if (!f->sel) return fail(PF_ERR_INVALID, "selection recording is off (pf_record_selection)");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    pf_status s = materialise(f);
    if (s != PF_OK) return s;
    CU(cudaMemcpy(sel, f->sel, (size_t)f->T * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

// The launch sequence of one step on f->stream.  desc: device descriptor to use.
// With timing on, an event is recorded before the first and after every launch
// (also inside a captured graph, as event-record nodes).
static pf_status enqueue_step(pf_filter* f, const FilterDesc* desc, InputRef in, int32_t* ctr_inc)
{
    const int M = f->M, E = f->E, N = f->N;
    cudaStream_t st = f->stream;
    const pf_config& c = f->cfg;
    int np = 0;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (f->timing) CU(cudaStreamIsCapturing(st, &cap));
    auto mark = [&](const char* name) -> cudaError_t {
        if (!f->timing) return cudaSuccess;
        if (name) f->phase[np - 1] = name;
        if (np >= 8) return cudaSuccess;
        // inside a capture the record must become an event node of the graph
        return cudaEventRecordWithFlags(f->ev[np++], st,
                                        cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                             : cudaEventRecordDefault);
    };
    CU(mark(nullptr));
    if (c.rng == PF_RNG_REFLAYOUT) {
        const int G = c.mtgp_streams;
        CU(launch_mtgp_blocks(G, f->mtgp, reinterpret_cast<uint32_t*>(f->rbuf), f->rtotal / G, c.mtgp_mask, 1, 0, st));
        CU(mark("mtgp32"));
        CU(launch_boxmuller(f->rbuf, (int64_t)f->mi.K * f->T, st));
        CU(mark("boxmuller"));
    }
    if (f->pipe == PF_PIPELINE_FUSED) {
        CU(f->ops.step(M, E, c.resampler, N, st, desc, f->X, in, ctr_inc, false));
        CU(mark("step"));
        if (c.exchange == PF_EXCHANGE_ALL2ALL && f->t > 0) {
            CU(launch_a2a_merge_step(desc, f->X, st));
            CU(mark("a2a_merge"));
        }
    } else if (f->pipe == PF_PIPELINE_SPLIT) {
        CU(f->ops.sample_sort(M, E, f->tp, c.rng == PF_RNG_SUBFILTER, N, st, desc, nullptr, in));
        CU(mark("sample_sort"));
        if (c.exchange == PF_EXCHANGE_ALL2ALL && f->t > 0) {
            CU(launch_a2a_merge(1, desc, st));
            CU(mark("a2a_merge"));
        }
        // with an exchange period every CTA of the resampling kernel reads the
        // step counter, so it advances in a launch of its own after the kernel
        const bool late = ctr_inc && c.exchange_period > 1;
        // a programmatic dependent of the sampling kernel when that pays (its
        // CTAs start during the sampling kernel's last wave and wait there)
        const int virt = dependent_launch_pays(N, M, E, f->mi.S, c.device) ? 3 : 1;
        CU(f->ops.exchange_resample(M, E, c.resampler, N + estimate_ctas(N), st, desc, nullptr, in,
                                    late ? nullptr : ctr_inc, virt));
        CU(mark("exchange_resample"));
        if (late) CU(launch_counter_inc(ctr_inc, st));
    } else {
        CU(f->ops.sample_weight(M, E, N, st, desc, nullptr, in));
        CU(mark("sample_weight"));
        CU(f->ops.block_sort(M, E, N, st, desc, nullptr));
        CU(mark("block_sort"));
        if (c.exchange == PF_EXCHANGE_ALL2ALL && f->t > 0) {
            CU(launch_a2a_merge(1, desc, st));
            CU(mark("a2a_merge"));
        }
        if (c.exchange != PF_EXCHANGE_NONE && f->t > 0) {
            const int nx = c.exchange == PF_EXCHANGE_TORUS ? 4 * f->t : f->t;
            CU(f->ops.exchange_inplace(N, nx < 1024 ? ((nx + 31) / 32) * 32 : 1024, st, desc, nullptr));
            CU(mark("exchange"));
        }
        CU(f->ops.exchange_resample(M, E, c.resampler, N + estimate_ctas(N), st, desc, nullptr, in, ctr_inc, 0));
        CU(mark("resample"));
    }
    if (f->timing) f->nphase = np - 1;
    return PF_OK;
}

extern "C" pf_status pf_set_timing(pf_filter* f, int32_t enable)
{
    if (!f) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    if (enable && !f->ev[0])
        for (auto& e : f->ev) CU(cudaEventCreate(&e));
    if ((enable != 0) != (f->timing != 0) && f->graph) {
        cudaGraphExecDestroy(f->graph);
        f->graph = nullptr;
    }
    f->timing = enable ? 1 : 0;
    return PF_OK;
}

extern "C" pf_status pf_last_step_timing(pf_filter* f, float* ms, int32_t cap, int32_t* n)
{
    if (!f || !n) return fail(PF_ERR_INVALID, "null argument");
    if (!f->timing || f->nphase <= 0) return fail(PF_ERR_INVALID, "timing is off or no step ran");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaEventSynchronize(f->ev[f->nphase]));
    *n = f->nphase;
    for (int i = 0; i < f->nphase && i < cap; ++i) CU(cudaEventElapsedTime(&ms[i], f->ev[i], f->ev[i + 1]));
    return PF_OK;
}

extern "C" const char* pf_phase_name(pf_filter* f, int32_t i)
{
    if (!f || i < 0 || i >= f->nphase) return "";
    return f->phase[i];
}

extern "C" pf_status pf_step(pf_filter* f, const pf_step_input* in, pf_estimate* out)
{
    if (!f || !in) return fail(PF_ERR_INVALID, "null argument");
    if (f->shard) return fail(PF_ERR_INVALID, "a shard steps through pf_shard_sample / pf_shard_resample");
    CU(cudaSetDevice(f->cfg.device));
    *f->h_in = *in;
    CU(cudaMemcpyAsync(f->d_in, f->h_in, sizeof(pf_step_input), cudaMemcpyHostToDevice, f->stream));
    InputRef ir{f->d_in, 0, nullptr, 0, f->steps_done};
    pf_status s = enqueue_step(f, f->d_desc, ir, nullptr);
    if (s != PF_OK) return s;
    CU(cudaMemcpyAsync(f->h_est, f->d_est, sizeof(pf_estimate) + sizeof(int32_t), cudaMemcpyDeviceToHost,
                       f->stream));
    CU(cudaStreamSynchronize(f->stream));
    f->steps_done++;
    s = check_status(*reinterpret_cast<const int32_t*>(f->h_est + 1));
    if (s != PF_OK) return s;
    if (out) {
        *out = *f->h_est;
        out->step = f->steps_done;
    }
    return PF_OK;
}

// The graph of one step reading inputs[ctr % capacity] and writing
// estimates[ctr % capacity] (ctr: the filter's device step counter), rebuilt
// when the arrays change.
static pf_status ensure_run_graph(pf_filter* f, const pf_step_input* d_inputs, pf_estimate* d_estimates,
                                  int32_t capacity)
{
    if (f->graph && f->graph_inputs == d_inputs && f->graph_est == d_estimates && f->graph_cap == capacity)
        return PF_OK;
    CU(cudaStreamSynchronize(f->stream));
    if (f->graph) {
        cudaGraphExecDestroy(f->graph);
        f->graph = nullptr;
    }
    pf_status s = upload_descs(f, d_estimates);
    if (s != PF_OK) return s;
    cudaGraph_t g = nullptr;
    CU(cudaStreamBeginCapture(f->stream, cudaStreamCaptureModeThreadLocal));
    InputRef ir{d_inputs, 0, f->ctr, capacity};
    s = enqueue_step(f, f->d_desc + 1, ir, f->ctr);
    cudaError_t e = cudaStreamEndCapture(f->stream, &g);
    if (s != PF_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return fail(PF_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&f->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        f->graph = nullptr;
        return fail(PF_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    f->graph_inputs = d_inputs;
    f->graph_est = d_estimates;
    f->graph_cap = capacity;
    return PF_OK;
}

extern "C" pf_status pf_run_device(pf_filter* f, const pf_step_input* d_inputs, pf_estimate* d_estimates,
                                   int32_t capacity, int32_t steps)
{
    if (!f || !d_inputs || !d_estimates || capacity < 1 || steps < 0) return fail(PF_ERR_INVALID, "bad argument");
    if (f->shard) return fail(PF_ERR_INVALID, "a shard steps through pf_shard_sample / pf_shard_resample");
    CU(cudaSetDevice(f->cfg.device));
    pf_status s = ensure_run_graph(f, d_inputs, d_estimates, capacity);
    if (s != PF_OK) return s;
    CU(cudaMemsetAsync(f->ctr, 0, sizeof(int32_t), f->stream));
    f->q_active = 0;
    for (int i = 0; i < steps; ++i) CU(cudaGraphLaunch(f->graph, f->stream));
    f->steps_done += steps;
    return PF_OK;
}

static pf_status queue_setup(pf_filter* f)
{
    if (f->d_q_in) return PF_OK;
    void* h = nullptr;
    if (!f->h_q_in) {
        CU(cudaMallocHost(&h, PF_QUEUE_DEPTH * sizeof(pf_step_input)));
        f->h_q_in = static_cast<pf_step_input*>(h);
    }
    if (!f->h_q_est) {
        CU(cudaMallocHost(&h, PF_QUEUE_DEPTH * sizeof(pf_estimate)));
        f->h_q_est = static_cast<pf_estimate*>(h);
    }
    if (!f->q_up) CU(cudaStreamCreateWithFlags(&f->q_up, cudaStreamNonBlocking));
    if (!f->q_down) CU(cudaStreamCreateWithFlags(&f->q_down, cudaStreamNonBlocking));
    for (int i = 0; i < PF_QUEUE_DEPTH; ++i) {
        if (!f->q_ev_up[i]) CU(cudaEventCreateWithFlags(&f->q_ev_up[i], cudaEventDisableTiming));
        if (!f->q_ev_done[i]) CU(cudaEventCreateWithFlags(&f->q_ev_done[i], cudaEventDisableTiming));
        if (!f->q_ev_got[i]) CU(cudaEventCreateWithFlags(&f->q_ev_got[i], cudaEventDisableTiming));
    }
    if (!f->d_q_est) {
        pf_status s = dalloc(f, &f->d_q_est, PF_QUEUE_DEPTH);
        if (s != PF_OK) return s;
    }
    pf_step_input* di = nullptr;
    pf_status s = dalloc(f, &di, PF_QUEUE_DEPTH);
    if (s != PF_OK) return s;
    f->d_q_in = di;  // set last: marks the queue as set up
    return PF_OK;
}

extern "C" pf_status pf_step_submit(pf_filter* f, const pf_step_input* in)
{
    if (!f || !in) return fail(PF_ERR_INVALID, "null argument");
    if (f->shard) return fail(PF_ERR_INVALID, "a shard steps through pf_shard_sample / pf_shard_resample");
    CU(cudaSetDevice(f->cfg.device));
    pf_status s = queue_setup(f);
    if (s != PF_OK) return s;
    if (f->q_pending >= PF_QUEUE_DEPTH)
        return fail(PF_ERR_BUSY, "%d steps pending: collect before submitting more", PF_QUEUE_DEPTH);
    if (!f->q_active || f->q_next != f->steps_done) {
        // another call stepped the filter or reset its counter since the last submit
        if (f->q_pending > 0)
            return fail(PF_ERR_BUSY, "collect the pending steps before submitting after another step call");
        s = ensure_run_graph(f, f->d_q_in, f->d_q_est, PF_QUEUE_DEPTH);
        if (s != PF_OK) return s;
        CU(launch_counter_set(f->ctr, f->steps_done, f->stream));
        f->q_next = f->steps_done;
        f->q_active = 1;
    }
    const int slot = (int)((uint32_t)f->q_next % PF_QUEUE_DEPTH);  // as the device maps its counter
    f->h_q_in[slot] = *in;
    CU(cudaMemcpyAsync(f->d_q_in + slot, f->h_q_in + slot, sizeof(pf_step_input), cudaMemcpyHostToDevice, f->q_up));
    CU(cudaEventRecord(f->q_ev_up[slot], f->q_up));
    CU(cudaStreamWaitEvent(f->stream, f->q_ev_up[slot], 0));
    CU(cudaGraphLaunch(f->graph, f->stream));
    CU(cudaEventRecord(f->q_ev_done[slot], f->stream));
    CU(cudaStreamWaitEvent(f->q_down, f->q_ev_done[slot], 0));
    CU(cudaMemcpyAsync(f->h_q_est + slot, f->d_q_est + slot, sizeof(pf_estimate), cudaMemcpyDeviceToHost,
                       f->q_down));
    CU(cudaEventRecord(f->q_ev_got[slot], f->q_down));
    f->q_next++;
    f->steps_done++;
    f->q_pending++;
    return PF_OK;
}

extern "C" pf_status pf_step_collect(pf_filter* f, pf_estimate* out, int32_t max, int32_t wait, int32_t* count)
{
    if (!f || !count || (max > 0 && !out)) return fail(PF_ERR_INVALID, "null argument");
    *count = 0;
    if (f->q_pending == 0 || max <= 0) return PF_OK;
    CU(cudaSetDevice(f->cfg.device));
    while (*count < max && f->q_pending > 0) {
        const int32_t k = f->q_next - f->q_pending;  // oldest pending step
        const int slot = (int)((uint32_t)k % PF_QUEUE_DEPTH);
        if (wait) {
            CU(cudaEventSynchronize(f->q_ev_got[slot]));
        } else {
            const cudaError_t e = cudaEventQuery(f->q_ev_got[slot]);
            if (e == cudaErrorNotReady) break;
            CU(e);
        }
        out[(*count)++] = f->h_q_est[slot];
        f->q_pending--;
    }
    return PF_OK;
}

// One step of a run already set up by pf_run_device (graph replay with the
// counter continuing); used to time steps one by one.
extern "C" pf_status pf_run_device_continue(pf_filter* f, int32_t steps)
{
    if (!f || !f->graph) return fail(PF_ERR_INVALID, "no run set up (call pf_run_device first)");
    CU(cudaSetDevice(f->cfg.device));
    for (int i = 0; i < steps; ++i) CU(cudaGraphLaunch(f->graph, f->stream));
    f->steps_done += steps;
    return PF_OK;
}

extern "C" pf_status pf_synchronize(pf_filter* f)
{
    if (!f) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    int32_t st = 0;
    CU(cudaMemcpy(&st, status_word(f), sizeof(st), cudaMemcpyDeviceToHost));
    return check_status(st);
}

extern "C" void* pf_stream(pf_filter* f) { return f ? (void*)f->stream : nullptr; }

extern "C" pf_status pf_get_info(pf_filter* f, int32_t* pipe, int32_t* ppt, int32_t* dx, int32_t* dy,
                                  int64_t* bytes)
{
    if (!f) return fail(PF_ERR_INVALID, "null argument");
    if (pipe) *pipe = f->pipe;
    if (ppt) *ppt = f->E;
    if (dx) *dx = f->dx;
    if (dy) *dy = f->dy;
    if (bytes) *bytes = f->dev_bytes;
    return PF_OK;
}

// snapshot layout: int64 header[4] = {magic, S, T, streams}, state S*T floats,
// stream words streams*351, int32 steps_done.
static const int64_t kSnapMagic = 0x5046534e41503031LL;

extern "C" int64_t pf_snapshot_size(pf_filter* f)
{
    if (!f) return -1;
    return 32 + (int64_t)f->mi.S * f->T * 4 + (int64_t)f->streams * kMtgpN * 4 + 4;
}

extern "C" pf_status pf_snapshot(pf_filter* f, void* buf)
{
    if (!f || !buf) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    pf_status ms = materialise(f);
    if (ms != PF_OK) return ms;
    char* p = (char*)buf;
    int64_t hdr[4] = {kSnapMagic, f->mi.S, f->T, f->streams};
    memcpy(p, hdr, 32);
    p += 32;
    const size_t sb = (size_t)f->mi.S * f->T * 4, mb = (size_t)f->streams * kMtgpN * 4;
    CU(cudaMemcpy(p, f->state, sb, cudaMemcpyDeviceToHost));
    p += sb;
    CU(cudaMemcpy(p, f->mtgp, mb, cudaMemcpyDeviceToHost));
    p += mb;
    memcpy(p, &f->steps_done, 4);
    return PF_OK;
}

extern "C" pf_status pf_restore(pf_filter* f, const void* buf, size_t size)
{
    if (!f || !buf) return fail(PF_ERR_INVALID, "null argument");
    const int64_t want = pf_snapshot_size(f);
    if (size < 32 || (int64_t)size != want)
        return fail(PF_ERR_INVALID, "snapshot of %zu bytes; this filter takes %lld", size, (long long)want);
    const char* p = (const char*)buf;
    int64_t hdr[4];
    memcpy(hdr, p, 32);
    if (hdr[0] != kSnapMagic || hdr[1] != f->mi.S || hdr[2] != f->T || hdr[3] != f->streams)
        return fail(PF_ERR_INVALID, "snapshot does not match this filter");
    p += 32;
    CU(cudaSetDevice(f->cfg.device));
    CU(cudaStreamSynchronize(f->stream));
    const size_t sb = (size_t)f->mi.S * f->T * 4, mb = (size_t)f->streams * kMtgpN * 4;
    CU(cudaMemcpy(f->state, p, sb, cudaMemcpyHostToDevice));
    p += sb;
    CU(cudaMemcpy(f->mtgp, p, mb, cudaMemcpyHostToDevice));
    p += mb;
    memcpy(&f->steps_done, p, 4);
    f->q_active = 0;
    return mark_need_init(f);
}

// ---------------------------------------------------------------------------
// kernel-level entry points (host arrays in/out)
// ---------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

static pf_status dev_buf(DevBuf& b, size_t bytes)
{
    CU(cudaMalloc(&b.p, bytes ? bytes : 4));
    return PF_OK;
}

#define TRYS(x)                 \
    do {                        \
        pf_status s_ = (x);     \
        if (s_ != PF_OK) return s_; \
    } while (0)

extern "C" pf_status pfk_mtgp_generate(int32_t G, uint32_t seed, uint32_t mask, int32_t kind, int64_t per_stream,
                                       int32_t calls, uint32_t* out)
{
    if (G < 1 || G > 200 || per_stream < 0 || per_stream > INT32_MAX || calls < 1 || !out)
        return fail(PF_ERR_INVALID, "bad argument");
    TRYS(require_gpu(0));
    std::vector<uint32_t> st((size_t)G * kMtgpN);
    for (int g = 0; g < G; ++g) mtgp_init_state_host(st.data() + (size_t)g * kMtgpN, g, seed + (uint32_t)g + 1u);
    DevBuf ds, dout;
    TRYS(dev_buf(ds, st.size() * 4));
    TRYS(dev_buf(dout, (size_t)G * per_stream * 4));
    CU(cudaMemcpy(ds.p, st.data(), st.size() * 4, cudaMemcpyHostToDevice));
    for (int c = 0; c < calls; ++c) {
        CU(launch_mtgp_blocks(G, (uint32_t*)ds.p, (uint32_t*)dout.p, per_stream, mask, kind ? 1 : 0, 0, 0));
        CU(cudaMemcpy(out + (size_t)c * G * per_stream, dout.p, (size_t)G * per_stream * 4, cudaMemcpyDeviceToHost));
    }
    return PF_OK;
}

extern "C" pf_status pfk_bounded_wait_test(int32_t limit, int32_t* status)
{
    if (!status || limit < 1 || limit > (1 << 20)) return fail(PF_ERR_INVALID, "bad argument");
    TRYS(require_gpu(0));
    DevBuf d;
    TRYS(dev_buf(d, 4));
    CU(cudaMemset(d.p, 0xff, 4));
    CU(launch_test_bounded_wait(limit, (int32_t*)d.p, 0));
    CU(cudaMemcpy(status, d.p, 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pfk_bounded_wait_mixed_test(const int32_t* limits, int32_t nthreads, int32_t* outcome,
                                                 int32_t* copied)
{
    if (!limits || !outcome || !copied || nthreads < 32 || nthreads > 1024 || nthreads % 32)
        return fail(PF_ERR_INVALID, "bad argument");
    for (int i = 0; i < nthreads; ++i)
        if (limits[i] < 0 || limits[i] > (1 << 20)) return fail(PF_ERR_INVALID, "poll limits must be in [0, 2^20]");
    TRYS(require_gpu(0));
    std::vector<uint32_t> src(kMixedWaitSrcBytes / 4);
    for (size_t i = 0; i < src.size(); ++i) src[i] = 0x9e3779b9u * (uint32_t)(i + 1);
    DevBuf dl, ds, dout;
    TRYS(dev_buf(dl, (size_t)nthreads * 4));
    TRYS(dev_buf(ds, kMixedWaitSrcBytes));
    TRYS(dev_buf(dout, (size_t)(nthreads + 1) * 4));
    CU(cudaMemcpy(dl.p, limits, (size_t)nthreads * 4, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(ds.p, src.data(), kMixedWaitSrcBytes, cudaMemcpyHostToDevice));
    CU(cudaMemset(dout.p, 0x7f, (size_t)(nthreads + 1) * 4));
    int32_t* o = static_cast<int32_t*>(dout.p);
    CU(launch_test_bounded_wait_mixed(static_cast<const int32_t*>(dl.p), nthreads, ds.p, o, o + nthreads, 0));
    CU(cudaMemcpy(outcome, o, (size_t)nthreads * 4, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(copied, o + nthreads, 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pfk_boxmuller(float* data, int64_t n)
{
    if (!data || n < 0) return fail(PF_ERR_INVALID, "bad argument");
    TRYS(require_gpu(0));
    const size_t cnt = (size_t)(2 * ((n + 1) / 2));
    DevBuf d;
    TRYS(dev_buf(d, cnt * 4));
    CU(cudaMemcpy(d.p, data, cnt * 4, cudaMemcpyHostToDevice));
    CU(launch_boxmuller((float*)d.p, n, 0));
    CU(cudaMemcpy(data, d.p, cnt * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

static int pick_ppt(int m, int ppt) { return ppt > 0 ? ppt : default_ppt(m, 1); }

extern "C" pf_status pfk_bitonic_sort(float* keys, int32_t* idx, int32_t m, int32_t nsub, int32_t ppt)
{
    if (!keys || !idx || nsub < 1) return fail(PF_ERR_INVALID, "bad argument");
    const int E = pick_ppt(m, ppt);
    if (!me_supported(m, E)) return fail(PF_ERR_UNSUPPORTED, "m=%d ppt=%d not built", m, E);
    TRYS(require_gpu(0));
    const size_t n = (size_t)m * nsub;
    DevBuf dk, di;
    TRYS(dev_buf(dk, n * 4));
    TRYS(dev_buf(di, n * 4));
    CU(cudaMemcpy(dk.p, keys, n * 4, cudaMemcpyHostToDevice));
    CU(launch_test_sort(m, E, nsub, (float*)dk.p, (int32_t*)di.p, 0, nullptr, 0));
    CU(cudaMemcpy(keys, dk.p, n * 4, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(idx, di.p, n * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pfk_rank_sort(float* keys, int32_t* idx, int32_t m, int32_t nsub, int32_t ppt,
                                   int32_t* fallbacks)
{
    if (!keys || !idx || !fallbacks || nsub < 1) return fail(PF_ERR_INVALID, "bad argument");
    const int E = pick_ppt(m, ppt);
    if (!me_supported(m, E)) return fail(PF_ERR_UNSUPPORTED, "m=%d ppt=%d not built", m, E);
    TRYS(require_gpu(0));
    const size_t n = (size_t)m * nsub;
    DevBuf dk, di, dc;
    TRYS(dev_buf(dk, n * 4));
    TRYS(dev_buf(di, n * 4));
    TRYS(dev_buf(dc, 4));
    CU(cudaMemcpy(dk.p, keys, n * 4, cudaMemcpyHostToDevice));
    CU(cudaMemset(dc.p, 0, 4));
    CU(launch_test_sort(m, E, nsub, (float*)dk.p, (int32_t*)di.p, 1, (int32_t*)dc.p, 0));
    CU(cudaMemcpy(keys, dk.p, n * 4, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(idx, di.p, n * 4, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(fallbacks, dc.p, 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

static pf_status test_resample(int res, const float* w, const float* u, int m, int nsub, int ppt, int32_t* sel,
                               float* prob, uint32_t* alias)
{
    const int E = pick_ppt(m, ppt);
    if (!me_supported(m, E)) return fail(PF_ERR_UNSUPPORTED, "m=%d ppt=%d not built", m, E);
    TRYS(require_gpu(0));
    const size_t n = (size_t)m * nsub;
    const size_t nu = res == PF_RESAMPLE_SYSTEMATIC ? (size_t)nsub : (res == PF_RESAMPLE_VOSE ? 2 * n : n);
    DevBuf dw, du, ds, dp, da;
    TRYS(dev_buf(dw, n * 4));
    TRYS(dev_buf(du, nu * 4));
    TRYS(dev_buf(ds, n * 4));
    CU(cudaMemcpy(dw.p, w, n * 4, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(du.p, u, nu * 4, cudaMemcpyHostToDevice));
    if (prob) {
        TRYS(dev_buf(dp, n * 4));
        TRYS(dev_buf(da, n * 4));
    }
    CU(launch_test_resample(res, m, E, nsub, (const float*)dw.p, (const float*)du.p, (int32_t*)ds.p,
                            (float*)dp.p, (uint32_t*)da.p, 0));
    if (sel) CU(cudaMemcpy(sel, ds.p, n * 4, cudaMemcpyDeviceToHost));
    if (prob) {
        CU(cudaMemcpy(prob, dp.p, n * 4, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(alias, da.p, n * 4, cudaMemcpyDeviceToHost));
    }
    return PF_OK;
}

extern "C" pf_status pfk_resample(int32_t resampler, const float* w, const float* u, int32_t m, int32_t nsub,
                                  int32_t ppt, int32_t* sel)
{
    if (!w || !u || !sel || nsub < 1 || resampler < 0 || resampler > 2) return fail(PF_ERR_INVALID, "bad argument");
    return test_resample(resampler, w, u, m, nsub, ppt, sel, nullptr, nullptr);
}

extern "C" pf_status pfk_vose_build(const float* w, int32_t m, int32_t nsub, int32_t ppt, float* prob,
                                    uint32_t* alias)
{
    if (!w || !prob || !alias || nsub < 1) return fail(PF_ERR_INVALID, "bad argument");
    std::vector<float> u((size_t)2 * m * nsub, 0.0f);
    return test_resample(PF_RESAMPLE_VOSE, w, u.data(), m, nsub, ppt, nullptr, prob, alias);
}

extern "C" pf_status pfk_exchange_sources(int32_t mode, int32_t N, int32_t m, int32_t t, const float* sorted_keys,
                                          int32_t* src)
{
    // Routing is evaluated by the same device function the step kernels use.
    if (!src || N < 1 || m < 1 || t < 0) return fail(PF_ERR_INVALID, "bad argument");
    if (mode == PF_EXCHANGE_ALL2ALL && (!sorted_keys || N > 8192)) return fail(PF_ERR_INVALID, "bad argument");
    TRYS(require_gpu(0));
    const int64_t T = (int64_t)m * N;
    DevBuf dkeys, da2a, dsrc, ddesc;
    TRYS(dev_buf(dkeys, (size_t)T * 4));
    TRYS(dev_buf(da2a, (size_t)(t > 0 ? t : 1) * 4));
    TRYS(dev_buf(dsrc, (size_t)T * 4));
    TRYS(dev_buf(ddesc, sizeof(FilterDesc)));
    if (sorted_keys) CU(cudaMemcpy(dkeys.p, sorted_keys, (size_t)T * 4, cudaMemcpyHostToDevice));
    FilterDesc D;
    memset(&D, 0, sizeof(D));
    D.tkey = (float*)dkeys.p;
    D.a2a = (int32_t*)da2a.p;
    D.T = T;
    D.N = N;
    D.M = m;
    D.t = t;
    D.exchange = mode;
    torus_dims(N, &D.dx, &D.dy);
    CU(cudaMemcpy(ddesc.p, &D, sizeof(D), cudaMemcpyHostToDevice));
    if (mode == PF_EXCHANGE_ALL2ALL && t > 0) CU(launch_a2a_merge(1, (const FilterDesc*)ddesc.p, 0));
    CU(launch_exchange_sources((const FilterDesc*)ddesc.p, (int32_t*)dsrc.p, 0));
    CU(cudaMemcpy(src, dsrc.p, (size_t)T * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pfk_model_step(pf_model_id model, const void* params, size_t params_size,
                                    const pf_step_input* in, int32_t n, float* state, const float* noise,
                                    float* loglik)
{
    ModelInfo mi;
    if (!model_info(model, &mi)) return fail(PF_ERR_INVALID, "unknown model");
    if (!params || params_size != mi.psize || !in || n < 1 || !state || !noise || !loglik)
        return fail(PF_ERR_INVALID, "bad argument");
    TRYS(require_gpu(0));
    ModelParams mp;
    memset(&mp, 0, sizeof(mp));
    memcpy(&mp, params, params_size);
    DevBuf din, ds, dn, dl;
    TRYS(dev_buf(din, sizeof(pf_step_input)));
    TRYS(dev_buf(ds, (size_t)mi.S * n * 4));
    TRYS(dev_buf(dn, (size_t)mi.K * n * 4));
    TRYS(dev_buf(dl, (size_t)n * 4));
    CU(cudaMemcpy(din.p, in, sizeof(pf_step_input), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(ds.p, state, (size_t)mi.S * n * 4, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(dn.p, noise, (size_t)mi.K * n * 4, cudaMemcpyHostToDevice));
    CU(model_ops(model).test_model(mp, (const pf_step_input*)din.p, n, (float*)ds.p, (const float*)dn.p,
                                   (float*)dl.p, 0));
    CU(cudaMemcpy(state, ds.p, (size_t)mi.S * n * 4, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(loglik, dl.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

// ---------------------------------------------------------------------------
// Shards: one filter's torus rows spread over several filters (devices,
// processes).  The reference runs one filter per process
// (src/partfilt/cuda/pf_generic_soa.cu:686); its torus exchange
// (src/partfilt/cuda/pf_generic.cu:352-393, dims :682-683) is what crosses
// the shard boundaries here: between a step's sampling and its resampling
// each shard hands the sorted top t of its first and last rows to the shards
// above and below, and the group partial rows of all shards are combined into
// the filter's estimate in group order.  With shard boundaries on whole rows
// and on multiples of 32 sub-filters, the shards' particles, sorted copies and
// estimate equal the unsharded filter's bit for bit.
// ---------------------------------------------------------------------------
static_assert(PF_SHARD_ROW == kPartStride, "group row width");
static int64_t halo_block_floats(const pf_filter* f) { return (int64_t)(1 + f->mi.S) * f->dx * f->t; }

extern "C" pf_status pf_shard_create(const pf_config* cfg, pf_model_id model, const void* params, size_t params_size,
                                     int32_t row0, int32_t row1, pf_filter** out)
{
    if (!cfg || !out) return fail(PF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->exchange != PF_EXCHANGE_TORUS || cfg->num_transfer < 1)
        return fail(PF_ERR_UNSUPPORTED, "shards run the torus exchange (t >= 1)");
    if (cfg->rng != PF_RNG_SUBFILTER) return fail(PF_ERR_UNSUPPORTED, "shards draw one MTGP32 stream per sub-filter");
    if (cfg->exchange_period > 1) return fail(PF_ERR_UNSUPPORTED, "shards exchange every step");
    const int N = cfg->num_subfilters;
    ModelInfo mi;
    if (!model_info(model, &mi)) return fail(PF_ERR_INVALID, "unknown model %d", (int)model);
    int E = 0;
    TRYS(validate(cfg, model, mi, &E));  // the whole filter's configuration (torus dims, 5 t <= m)
    int dx = 0, dy = 0;
    torus_dims(N, &dx, &dy);
    if (row0 < 0 || row1 <= row0 || row1 > dy)
        return fail(PF_ERR_INVALID, "rows [%d, %d) outside the %d x %d torus", row0, row1, dx, dy);
    if (row1 - row0 == dy) return fail(PF_ERR_INVALID, "a shard holding every row is the whole filter: use pf_create");
    const int b0 = row0 * dx, n = (row1 - row0) * dx;
    if (b0 % 32 != 0 || (n % 32 != 0 && b0 + n != N))
        return fail(PF_ERR_UNSUPPORTED, "shard boundaries must fall on multiples of 32 sub-filters (the estimate's "
                                        "groups); rows [%d, %d) of width %d start at sub-filter %d", row0, row1, dx, b0);
    pf_config c = *cfg;
    c.num_subfilters = n;
    c.stream_offset = cfg->stream_offset + b0;  // global sub-filter b draws the stream of the whole filter's b
    c.pipeline = PF_PIPELINE_SPLIT;
    c.exchange = PF_EXCHANGE_RING;  // the shard's rows need not form a torus of their own
    pf_filter* f = nullptr;
    pf_status s = pf_create(&c, model, params, params_size, &f);
    if (s != PF_OK) return s;
    f->cfg.exchange = PF_EXCHANGE_TORUS;
    f->shard = 1;
    f->b0 = b0;
    f->r0 = row0;
    f->gdy = dy;
    f->gN = N;
    f->dx = dx;
    f->dy = row1 - row0;
    const int64_t hb = halo_block_floats(f);
    const int ng = (n + 31) / 32;
#define TRYR(x)              \
    do {                     \
        pf_status s_ = (x);  \
        if (s_ != PF_OK) {   \
            release(f);      \
            return s_;       \
        }                    \
    } while (0)
    TRYR(dalloc(f, &f->halo_in, 2 * (size_t)hb));
    TRYR(dalloc(f, &f->halo_out, 2 * (size_t)hb));
    TRYR(dalloc(f, &f->rows, (size_t)ng * kPartStride));
    TRYR(dalloc(f, &f->states, (size_t)ng * f->mi.S));
    if (cudaMemset(f->halo_in, 0, 2 * (size_t)hb * 4) != cudaSuccess ||
        cudaEventCreateWithFlags(&f->ev_sampled, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        release(f);
        return fail(PF_ERR_CUDA, "shard set-up failed");
    }
    TRYR(upload_descs(f, nullptr));
#undef TRYR
    *out = f;
    return PF_OK;
}

static pf_status need_shard(const pf_filter* f)
{
    if (!f) return fail(PF_ERR_INVALID, "null argument");
    if (!f->shard) return fail(PF_ERR_INVALID, "not a shard (pf_shard_create)");
    return PF_OK;
}

extern "C" pf_status pf_shard_info(pf_filter* f, int32_t* row0, int32_t* row1, int32_t* first_subfilter,
                                   int32_t* num_groups, int64_t* halo_bytes)
{
    TRYS(need_shard(f));
    if (row0) *row0 = f->r0;
    if (row1) *row1 = f->r0 + f->dy;
    if (first_subfilter) *first_subfilter = f->b0;
    if (num_groups) *num_groups = (f->N + 31) / 32;
    if (halo_bytes) *halo_bytes = 4 * halo_block_floats(f);
    return PF_OK;
}

extern "C" pf_status pf_shard_sample(pf_filter* f, const pf_step_input* in)
{
    TRYS(need_shard(f));
    if (!in) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    *f->h_in = *in;
    CU(cudaMemcpyAsync(f->d_in, f->h_in, sizeof(pf_step_input), cudaMemcpyHostToDevice, f->stream));
    InputRef ir{f->d_in, 0, nullptr, 0, f->steps_done};
    CU(f->ops.sample_sort(f->M, f->E, f->tp, true, f->N, f->stream, f->d_desc, nullptr, ir));
    CU(launch_shard_pack(f->d_desc, f->halo_out, f->mi.S, f->dx * f->t, f->stream));
    CU(cudaEventRecord(f->ev_sampled, f->stream));
    return PF_OK;
}

extern "C" pf_status pf_shard_halo_out(pf_filter* f, int32_t dir, void* host_buf)
{
    TRYS(need_shard(f));
    if (!host_buf || (dir != 0 && dir != 1)) return fail(PF_ERR_INVALID, "bad argument");
    CU(cudaSetDevice(f->cfg.device));
    const int64_t hb = halo_block_floats(f);
    CU(cudaMemcpyAsync(host_buf, f->halo_out + dir * hb, 4 * (size_t)hb, cudaMemcpyDeviceToHost, f->stream));
    CU(cudaStreamSynchronize(f->stream));
    return PF_OK;
}

extern "C" pf_status pf_shard_halo_in(pf_filter* f, int32_t dir, const void* host_buf)
{
    TRYS(need_shard(f));
    if (!host_buf || (dir != 0 && dir != 1)) return fail(PF_ERR_INVALID, "bad argument");
    CU(cudaSetDevice(f->cfg.device));
    const int64_t hb = halo_block_floats(f);
    CU(cudaMemcpyAsync(f->halo_in + dir * hb, host_buf, 4 * (size_t)hb, cudaMemcpyHostToDevice, f->stream));
    CU(cudaStreamSynchronize(f->stream));
    return PF_OK;
}

extern "C" pf_status pf_shard_halo_copy(pf_filter* from, int32_t dir, pf_filter* to)
{
    TRYS(need_shard(from));
    TRYS(need_shard(to));
    if (dir != 0 && dir != 1) return fail(PF_ERR_INVALID, "dir must be 0 or 1");
    if (from->gN != to->gN || from->dx != to->dx || from->t != to->t || from->mi.S != to->mi.S || from->M != to->M)
        return fail(PF_ERR_INVALID, "the shards belong to different filters");
    // block 0 carries from's last row to the shard below it (its row above),
    // block 1 from's first row to the shard above it (its row below)
    const int gdy = from->gdy;
    const bool adjacent = dir == 0 ? to->r0 == (from->r0 + from->dy) % gdy : (to->r0 + to->dy) % gdy == from->r0;
    if (!adjacent)
        return fail(PF_ERR_INVALID, "the shard at rows [%d, %d) is not the %s neighbour of the shard at rows [%d, %d)",
                    to->r0, to->r0 + to->dy, dir == 0 ? "lower" : "upper", from->r0, from->r0 + from->dy);
    const int64_t hb = halo_block_floats(from);
    CU(cudaSetDevice(to->cfg.device));
    CU(cudaStreamWaitEvent(to->stream, from->ev_sampled, 0));
    if (from->cfg.device == to->cfg.device)
        CU(cudaMemcpyAsync(to->halo_in + dir * hb, from->halo_out + dir * hb, 4 * (size_t)hb,
                           cudaMemcpyDeviceToDevice, to->stream));
    else
        CU(cudaMemcpyPeerAsync(to->halo_in + dir * hb, to->cfg.device, from->halo_out + dir * hb, from->cfg.device,
                               4 * (size_t)hb, to->stream));
    return PF_OK;
}

extern "C" pf_status pf_shard_resample(pf_filter* f)
{
    TRYS(need_shard(f));
    CU(cudaSetDevice(f->cfg.device));
    InputRef ir{f->d_in, 0, nullptr, 0, f->steps_done};
    CU(f->ops.exchange_resample(f->M, f->E, f->cfg.resampler, f->N + estimate_ctas(f->N), f->stream, f->d_desc,
                                nullptr, ir, nullptr, 1));
    const int ng = (f->N + 31) / 32;
    CU(launch_shard_rows(f->d_desc, ng, f->rows, f->states, f->mi.S, 2 + f->mi.S + f->na, f->stream));
    CU(cudaMemcpyAsync(f->h_est, f->d_est, sizeof(pf_estimate) + sizeof(int32_t), cudaMemcpyDeviceToHost, f->stream));
    CU(cudaStreamSynchronize(f->stream));
    f->steps_done++;
    return check_status(*reinterpret_cast<const int32_t*>(f->h_est + 1));
}

extern "C" pf_status pf_shard_group_rows(pf_filter* f, double* rows, float* states)
{
    TRYS(need_shard(f));
    if (!rows || !states) return fail(PF_ERR_INVALID, "null argument");
    CU(cudaSetDevice(f->cfg.device));
    const int ng = (f->N + 31) / 32;
    CU(cudaMemcpy(rows, f->rows, (size_t)ng * kPartStride * 8, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(states, f->states, (size_t)ng * f->mi.S * 4, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pf_shard_estimate(pf_filter* f, const double* rows, const float* states, int32_t num_groups,
                                       pf_estimate* out)
{
    TRYS(need_shard(f));
    const int S = f->mi.S, ngt = (f->gN + 31) / 32, NV = 2 + S + f->na;
    if (!rows || !states || !out || num_groups != ngt)
        return fail(PF_ERR_INVALID, "the estimate takes the rows of all %d groups", ngt);
    CU(cudaSetDevice(f->cfg.device));
    // winner states at their filter-wide sub-filter index (rows[g][NV+1])
    std::vector<float> best((size_t)S * f->gN, 0.0f);
    for (int g = 0; g < ngt; ++g) {
        const double wi = rows[(size_t)g * kPartStride + NV + 1];
        if (!(wi >= 0.0) || wi >= (double)f->gN) continue;
        for (int v = 0; v < S; ++v) best[(size_t)v * f->gN + (size_t)wi] = states[(size_t)g * S + v];
    }
    DevBuf dr, db, de;
    TRYS(dev_buf(dr, (size_t)ngt * kPartStride * 8));
    TRYS(dev_buf(db, best.size() * 4));
    TRYS(dev_buf(de, sizeof(pf_estimate)));
    CU(cudaMemcpy(dr.p, rows, (size_t)ngt * kPartStride * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(db.p, best.data(), best.size() * 4, cudaMemcpyHostToDevice));
    FilterDesc D;
    fill_desc(f, D, static_cast<pf_estimate*>(de.p));
    D.gpart = static_cast<double*>(dr.p);
    D.N = f->gN;
    D.T = f->gN;
    D.M = 1;
    D.b0 = 0;
    CU(launch_shard_estimate(D, S, static_cast<const float*>(db.p), static_cast<pf_estimate*>(de.p), ngt,
                             f->steps_done, 0));
    CU(cudaMemcpy(out, de.p, sizeof(pf_estimate), cudaMemcpyDeviceToHost));
    return PF_OK;
}
