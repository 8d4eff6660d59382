/*
 * pf_serve.c -- the served tracking load (host C over the pf_server_* ABI).
 *
 * Requests arrive as a Poisson process; each is a unicycle or a DH-arm
 * tracking filter with a log-uniform particle count and a stream of
 * measurement updates spaced uniformly in [min_gap, max_gap] ms, generated
 * from the load's seed (SplitMix64; request r's model parameters, ground
 * truth and measurements come from pf_make_trace with seed  seed * 1000003 + r,
 * which also seeds the filter's MTGP32 streams).  One host thread runs the
 * loop in real time:
 *   arrivals -> admission queue (FIFO; pf_server_open fails with
 *   PF_ERR_ADMISSION while the HBM budget or the slots are full) ->
 *   due updates queued with pf_server_update -> pf_server_launch whenever no
 *   batch is in flight -> pf_server_poll without blocking -> a request whose
 *   last update returned is closed, freeing its memory for the queue.
 * Latency of an update = time its result is back on the host minus the time
 * its measurement became due (waiting for admission counts).
 * Every k-th request (norm_check_every) stays open until the end; its last
 * log normalisation is compared with an FP64 log-sum-exp of its sorted keys.
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "esthera_b200.h"

typedef struct {
    uint64_t s;
} srng_t;

static uint64_t srng_next(srng_t* r)
{
    uint64_t z = (r->s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static double srng_unif(srng_t* r) { return (double)(srng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

typedef struct {
    int32_t model, particles, n_updates, next_issue, returned, slot, sampled, traced;
    double arrival;
    double* due;            /* due time of each update (relative to the run start) */
    pf_step_input* inputs;  /* [n_updates] */
    double last_log_norm;
} request_t;

/* binary min-heap of (due time, request index) */
typedef struct {
    double t;
    int32_t r;
} due_t;

typedef struct {
    due_t* a;
    int64_t n, cap;
} heap_t;

static int heap_push(heap_t* h, double t, int32_t r)
{
    if (h->n == h->cap) {
        int64_t cap = h->cap ? 2 * h->cap : 1024;
        due_t* a = (due_t*)realloc(h->a, (size_t)cap * sizeof(due_t));
        if (!a) return -1;
        h->a = a;
        h->cap = cap;
    }
    int64_t i = h->n++;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (h->a[p].t <= t) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i].t = t;
    h->a[i].r = r;
    return 0;
}

static due_t heap_pop(heap_t* h)
{
    due_t top = h->a[0];
    due_t last = h->a[--h->n];
    int64_t i = 0;
    for (;;) {
        int64_t c = 2 * i + 1;
        if (c >= h->n) break;
        if (c + 1 < h->n && h->a[c + 1].t < h->a[c].t) ++c;
        if (last.t <= h->a[c].t) break;
        h->a[i] = h->a[c];
        i = c;
    }
    if (h->n > 0) h->a[i] = last;
    return top;
}

static int cmp_float(const void* a, const void* b)
{
    const float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

static double pct(const float* sorted, int64_t n, double p)
{
    if (n <= 0) return 0.0;
    int64_t i = (int64_t)ceil(p / 100.0 * (double)n) - 1;
    if (i < 0) i = 0;
    if (i >= n) i = n - 1;
    return sorted[i];
}

pf_status pf_load_default(pf_load_config* c)
{
    if (!c) return PF_ERR_INVALID;
    memset(c, 0, sizeof(*c));
    c->rate = 2000.0;
    c->duration_s = 10.0;
    c->frac_unicycle = 0.7;
    c->min_particles = 1024;
    c->max_particles = 262144;
    c->min_updates = 50;
    c->max_updates = 500;
    c->min_gap_ms = 1.0;
    c->max_gap_ms = 20.0;
    c->seed = 5;
    c->hbm_budget = 150LL * 1000 * 1000 * 1000;
    c->max_filters = 16384;
    c->norm_check_every = 64;
    c->drain_limit_s = 30.0;
    return PF_OK;
}

static pf_status make_request(const pf_load_config* lc, int m, srng_t* rng, double arrival, request_t* q)
{
    memset(q, 0, sizeof(*q));
    q->arrival = arrival;
    q->slot = -1;
    q->model = srng_unif(rng) < lc->frac_unicycle ? PF_MODEL_UNICYCLE : PF_MODEL_DHARM;
    const double lo = log((double)lc->min_particles), hi = log((double)lc->max_particles);
    int64_t n = (int64_t)llround(exp(lo + (hi - lo) * srng_unif(rng)) / m) * m;
    if (n < m) n = m;
    q->particles = (int32_t)n;
    q->n_updates = lc->min_updates + (int32_t)(srng_unif(rng) * (double)(lc->max_updates - lc->min_updates + 1));
    if (q->n_updates > lc->max_updates) q->n_updates = lc->max_updates;
    q->due = (double*)malloc(sizeof(double) * (size_t)q->n_updates);
    q->inputs = (pf_step_input*)malloc(sizeof(pf_step_input) * (size_t)q->n_updates);
    if (!q->due || !q->inputs) return PF_ERR_NOMEM;
    double t = arrival;
    for (int j = 0; j < q->n_updates; ++j) {
        t += 1e-3 * (lc->min_gap_ms + (lc->max_gap_ms - lc->min_gap_ms) * srng_unif(rng));
        q->due[j] = t;
    }
    return PF_OK;
}

static pf_status fill_trace(request_t* q, uint32_t rseed, void* params)
{
    float* truth = (float*)malloc(sizeof(float) * PF_MAX_STATE * (size_t)q->n_updates);
    if (!truth) return PF_ERR_NOMEM;
    pf_status s;
    if (q->model == PF_MODEL_UNICYCLE) {
        s = pf_unicycle_default_params(rseed, 4, (pf_unicycle_params*)params);
    } else {
        s = pf_dharm_default_params(rseed, (pf_dharm_params*)params);
    }
    if (s == PF_OK) s = pf_make_trace((pf_model_id)q->model, params, rseed, q->n_updates, q->inputs, truth);
    free(truth);
    return s;
}

pf_status pf_serve_load(const pf_config* filter_cfg, const pf_load_config* lc, pf_load_report* rep)
{
    if (!filter_cfg || !lc || !rep) return PF_ERR_INVALID;
    if (!(lc->rate > 0) || !(lc->duration_s > 0) || lc->min_particles < 1 || lc->max_particles < lc->min_particles ||
        lc->min_updates < 1 || lc->max_updates < lc->min_updates || lc->max_gap_ms < lc->min_gap_ms)
        return PF_ERR_INVALID;
    memset(rep, 0, sizeof(*rep));
    const int m = filter_cfg->particles_per_subfilter;
    pf_server* srv = NULL;
    pf_status st = pf_server_create(filter_cfg, lc->hbm_budget, lc->max_filters, &srv);
    if (st != PF_OK) return st;
    pf_server_result* res = (pf_server_result*)malloc(sizeof(pf_server_result) * (size_t)lc->max_filters);
    int64_t req_cap = (int64_t)(lc->rate * lc->duration_s * 1.2) + 1024;
    request_t* reqs = (request_t*)calloc((size_t)req_cap, sizeof(request_t));
    int32_t* adm = (int32_t*)malloc(sizeof(int32_t) * (size_t)req_cap);  /* admission FIFO */
    int64_t lat_cap = 1 << 20, nlat = 0;
    float* lat = (float*)malloc(sizeof(float) * (size_t)lat_cap);
    heap_t heap = {0};
    if (!res || !reqs || !adm || !lat) {
        st = PF_ERR_NOMEM;
        goto done;
    }
    srng_t rng = {0x5345525645ULL ^ ((uint64_t)lc->seed << 24)};
    int64_t nreq = 0, adm_head = 0, adm_tail = 0, open_now = 0, finished = 0;
    double next_arrival = -log(1.0 - srng_unif(&rng)) / lc->rate;
    double demanded = 0.0, batch_sum = 0.0;
    const double t0 = now_s();
    double t = 0.0;
    union {
        pf_unicycle_params u;
        pf_dharm_params a;
    } params;
    for (;;) {
        t = now_s() - t0;
        /* arrivals */
        while (next_arrival <= t && next_arrival < lc->duration_s && nreq < req_cap) {
            request_t* q = &reqs[nreq];
            st = make_request(lc, m, &rng, next_arrival, q);
            if (st != PF_OK) goto done;
            demanded += (double)q->particles * q->n_updates;
            adm[adm_tail++] = (int32_t)nreq;
            ++nreq;
            next_arrival += -log(1.0 - srng_unif(&rng)) / lc->rate;
        }
        /* admissions, in arrival order */
        while (adm_head < adm_tail) {
            request_t* q = &reqs[adm[adm_head]];
            const uint32_t rseed = lc->seed * 1000003u + (uint32_t)adm[adm_head];
            if (!q->traced) {
                st = fill_trace(q, rseed, &params);
                if (st != PF_OK) goto done;
                q->traced = 1;
            } else if (q->model == PF_MODEL_UNICYCLE) {
                pf_unicycle_default_params(rseed, 4, &params.u);
            } else {
                pf_dharm_default_params(rseed, &params.a);
            }
            int32_t id = -1;
            st = pf_server_open(srv, (pf_model_id)q->model, &params,
                                q->model == PF_MODEL_UNICYCLE ? sizeof(pf_unicycle_params) : sizeof(pf_dharm_params),
                                q->particles, rseed, &id);
            if (st == PF_ERR_ADMISSION) {
                rep->admission_waits++;
                st = PF_OK;
                break;
            }
            if (st != PF_OK) goto done;
            q->slot = id;
            q->sampled = lc->norm_check_every > 0 && (adm[adm_head] % lc->norm_check_every) == 0;
            if (heap_push(&heap, q->due[0], adm[adm_head])) {
                st = PF_ERR_NOMEM;
                goto done;
            }
            ++adm_head;
            ++open_now;
            rep->admitted++;
        }
        /* due updates */
        while (heap.n > 0 && heap.a[0].t <= t) {
            due_t d = heap_pop(&heap);
            request_t* q = &reqs[d.r];
            const int j = q->next_issue++;
            st = pf_server_update(srv, q->slot, &q->inputs[j], ((uint64_t)(uint32_t)d.r << 32) | (uint32_t)j);
            if (st != PF_OK) goto done;
            if (q->next_issue < q->n_updates && heap_push(&heap, q->due[q->next_issue], d.r)) {
                st = PF_ERR_NOMEM;
                goto done;
            }
        }
        /* completions */
        int32_t n = 0;
        st = pf_server_poll(srv, 0, res, lc->max_filters, &n);
        if (st != PF_OK) goto done;
        if (n > 0) {
            const double tr = now_s() - t0;
            for (int i = 0; i < n; ++i) {
                const int32_t r = (int32_t)(res[i].tag >> 32);
                const int32_t j = (int32_t)(res[i].tag & 0xffffffffu);
                request_t* q = &reqs[r];
                if (nlat == lat_cap) {
                    float* l2 = (float*)realloc(lat, sizeof(float) * (size_t)(2 * lat_cap));
                    if (!l2) {
                        st = PF_ERR_NOMEM;
                        goto done;
                    }
                    lat = l2;
                    lat_cap *= 2;
                }
                lat[nlat++] = (float)(1e3 * (tr - q->due[j]));
                rep->particle_steps += (double)res[i].particles;
                q->returned++;
                q->last_log_norm = res[i].estimate.log_norm;
                if (q->returned == q->n_updates) {
                    ++finished;
                    if (!q->sampled) {
                        st = pf_server_close(srv, q->slot);
                        if (st != PF_OK) goto done;
                        q->slot = -1;
                        --open_now;
                    }
                    free(q->due);
                    q->due = NULL;
                    free(q->inputs);
                    q->inputs = NULL;
                }
            }
        }
        /* next batch */
        int32_t launched = 0;
        st = pf_server_launch(srv, &launched);
        if (st != PF_OK) goto done;
        if (launched > 0) {
            rep->launches++;
            batch_sum += launched;
        }
        pf_server_stats ss;
        pf_server_stats_get(srv, &ss);
        if (ss.resident_particles > rep->max_resident_particles) rep->max_resident_particles = ss.resident_particles;
        if (ss.bytes_in_use > rep->max_bytes_in_use) rep->max_bytes_in_use = ss.bytes_in_use;
        if (ss.open_filters > rep->max_open_filters) rep->max_open_filters = ss.open_filters;
        const int arrivals_over = next_arrival >= lc->duration_s || nreq >= req_cap;
        if (arrivals_over && finished == nreq && ss.in_flight == 0) break;
        if (arrivals_over && t > lc->duration_s + lc->drain_limit_s) {
            rep->incomplete = 1;
            break;
        }
    }
    rep->wall_s = now_s() - t0;
    /* drain a batch still in flight */
    {
        int32_t n = 0;
        pf_server_poll(srv, 1, res, lc->max_filters, &n);
    }
    rep->requests = nreq;
    rep->completed_requests = finished;
    rep->updates = nlat;
    rep->demanded_particle_steps_per_s = demanded / lc->duration_s;
    rep->particle_steps_per_s = rep->particle_steps / rep->wall_s;
    rep->mean_batch = rep->launches ? batch_sum / (double)rep->launches : 0.0;
    qsort(lat, (size_t)nlat, sizeof(float), cmp_float);
    rep->lat_p50_ms = pct(lat, nlat, 50.0);
    rep->lat_p99_ms = pct(lat, nlat, 99.0);
    rep->lat_p999_ms = pct(lat, nlat, 99.9);
    rep->lat_max_ms = nlat ? lat[nlat - 1] : 0.0;
    /* FP64 check of the sampled filters' last normalisation */
    {
        double emax = 0.0, esum = 0.0;
        int64_t nc = 0;
        for (int64_t r = 0; r < nreq; ++r) {
            request_t* q = &reqs[r];
            if (!q->sampled || q->slot < 0 || q->returned == 0) continue;
            float* keys = (float*)malloc(sizeof(float) * (size_t)q->particles);
            if (!keys) break;
            if (pf_server_get_particles(srv, q->slot, NULL, NULL, keys) == PF_OK) {
                double mx = -INFINITY;
                for (int i = 0; i < q->particles; ++i)
                    if ((double)keys[i] > mx) mx = keys[i];
                double sum = 0.0;
                for (int i = 0; i < q->particles; ++i) sum += exp((double)keys[i] - mx);
                const double ln = mx + log(sum);
                const double e = fabs(q->last_log_norm - ln) / (fabs(ln) > 1.0 ? fabs(ln) : 1.0);
                if (e > emax) emax = e;
                esum += e;
                ++nc;
            }
            free(keys);
        }
        rep->norm_checked = nc;
        rep->norm_err_max = emax;
        rep->norm_err_mean = nc ? esum / (double)nc : 0.0;
    }
    st = PF_OK;
done:
    if (reqs) {
        for (int64_t r = 0; r < req_cap; ++r) {
            free(reqs[r].due);
            free(reqs[r].inputs);
        }
    }
    free(reqs);
    free(adm);
    free(lat);
    free(res);
    free(heap.a);
    pf_server_destroy(srv);
    return st;
}
