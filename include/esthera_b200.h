/*
 * esthera_b200.h -- C ABI of the B200 particle-filter engine.
 *
 * The engine replaces the filter step of Esthera's distributed (sub-filter)
 * particle filter: MTGP32 random numbers -> Box-Muller -> per-particle
 * propagate + importance weight -> per-sub-filter bitonic sort -> global
 * winner -> exchange of the best particles between sub-filters -> resampling.
 * Everything runs as hand-written CUDA for sm_100a; there is no CPU fallback:
 * every call that needs the GPU returns PF_ERR_CUDA when none is usable.
 *
 * Conventions: plain pointers and sizes, no C++ or framework types; every
 * function returns a pf_status (never exit()); pf_last_error() gives a
 * thread-local message for the last failure.  A pf_filter is used by one
 * host thread at a time and owns one CUDA stream.
 *
 * Reference interfaces replaced (paths in the Esthera tree):
 *   driver call  int particle_filter(num_particles, num_blocks, num_transfer,
 *                resampling_freq, input_file)  src/partfilt/cuda/pf_generic_soa.cu:686,
 *                src/partfilt/opencl/pf_generic.c:245
 *   model hooks  sampling_iw / particle_set   src/models/robotarm/cuda/pf_model_soa.cuh:93-184
 *                read_trace / estimate_error  pf_model_soa.cuh:276-316,
 *                                             src/models/robotarm/opencl/pf_model_host.h:30-69
 */
#ifndef ESTHERA_B200_H
#define ESTHERA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PF_OK = 0,
    PF_ERR_INVALID = 1,     /* bad argument / configuration */
    PF_ERR_CUDA = 2,        /* CUDA runtime failure or no usable GPU */
    PF_ERR_NOMEM = 3,       /* device or host allocation failed */
    PF_ERR_UNSUPPORTED = 4, /* valid but not built (e.g. particle count not a power of two) */
    PF_ERR_IO = 5,          /* trace file missing or malformed */
    PF_ERR_ADMISSION = 6,   /* serving: request does not fit the memory budget */
    PF_ERR_TIMEOUT = 7,     /* a bounded wait ran out */
    PF_ERR_NOT_FOUND = 8,   /* serving: unknown request id */
    PF_ERR_BUSY = 9         /* serving: no free slot right now */
} pf_status;

typedef enum {
    PF_MODEL_UNICYCLE = 0, /* (x, y, theta), range/bearing to landmarks */
    PF_MODEL_DHARM = 1,    /* 6-joint Denavit-Hartenberg arm, q[6] + qdot[6] */
    PF_MODEL_REFARM = 2,   /* the reference's 5-angle camera arm on a cart */
    PF_MODEL_BEACON = 3,   /* the reference's unicycle tracked by range-only beacons (x, y, theta) */
    PF_MODEL_CAMARM = 4    /* the reference's camera arm seen through a pinhole camera with lens distortion */
} pf_model_id;
#define PF_NUM_MODELS 5

typedef enum {
    PF_EXCHANGE_NONE = 0,
    PF_EXCHANGE_RING = 1,    /* slot m-1-j <- sub-filter b-1 slot j          (exchange_ring) */
    PF_EXCHANGE_TORUS = 2,   /* slot m-1-j-k*t <- neighbour k slot j, k = R,L,B,T */
    PF_EXCHANGE_ALL2ALL = 3  /* slot m-1-j <- j-th best of all sub-filters' top t */
} pf_exchange;

typedef enum {
    PF_RESAMPLE_REFERENCE = 0,  /* multinomial, FP32 Blelloch scan + binary search (resampling) */
    PF_RESAMPLE_SYSTEMATIC = 1, /* systematic, FP64 scan */
    PF_RESAMPLE_VOSE = 2        /* Vose alias build + draw (resampling_valias) */
} pf_resampler;

typedef enum {
    PF_RNG_SUBFILTER = 0, /* one MTGP32 stream per sub-filter, generated inside the step kernel */
    PF_RNG_REFLAYOUT = 1  /* G streams materialised in the reference's block layout */
} pf_rng_layout;

typedef enum {
    PF_PIPELINE_FUSED = 0,  /* one kernel per step, one CTA per sub-filter, the resampling deferred to
                               the next step (needs PF_RNG_SUBFILTER and exchange_period <= 1;
                               other configurations run PF_PIPELINE_SPLIT) */
    PF_PIPELINE_PHASED = 1, /* one kernel per reference phase */
    PF_PIPELINE_SPLIT = 2   /* sample+weight+sort kernel, then exchange+resample+estimate kernel */
} pf_pipeline;

#define PF_MAX_STATE 16
#define PF_MAX_CONTROL 8
#define PF_MAX_MEAS 16
#define PF_MTGP_MASK_PARAMS 0u            /* use each parameter set's own mask (0xfff80000) */
#define PF_MTGP_MASK_CUDA_REF 0xff800000u /* constant hard-wired in the reference CUDA kernel */

typedef struct {
    int32_t particles_per_subfilter; /* m: power of two, 32..1024 (reference -m) */
    int32_t num_subfilters;          /* N (reference -N) */
    int32_t num_transfer;            /* t (reference -t) */
    int32_t exchange;                /* pf_exchange */
    int32_t resampler;               /* pf_resampler */
    float resampling_freq;           /* sub-filter b resamples iff its uniform u <= freq (reference -r) */
    uint32_t seed;                   /* stream g / sub-filter b seeded with seed + g + 1 */
    int32_t rng;                     /* pf_rng_layout */
    int32_t mtgp_streams;            /* G for PF_RNG_REFLAYOUT (1..200; reference: 96 OpenCL, 120 CUDA) */
    uint32_t mtgp_mask;              /* PF_MTGP_MASK_PARAMS or PF_MTGP_MASK_CUDA_REF */
    int32_t log_weights;             /* 1: FP32 max-subtracted log weights; 0: linear FP32 weights */
    int32_t pipeline;                /* pf_pipeline */
    int32_t particles_per_thread;    /* 0 = pick (1 for m = 32, 2 for m = 64, else 4 for states of up to
                                        3 variables and 2 for larger ones); built pairs
                                        (m, ppt): (32,1) (64,2) (128,2|4) (256,2|4|8) (512,2|4|16)
                                        (1024,2|4) */
    int32_t device;                  /* CUDA device ordinal */
    int32_t stream_offset;           /* PF_RNG_SUBFILTER: sub-filter b uses stream offset + b (parameter
                                        set (offset + b) mod 200, seed + offset + b + 1); 0 by default */
    int32_t exchange_period;         /* exchange on run steps s with s mod period == 0 (<= 1: every step;
                                        s counts pf_step calls since the initial state was set, or the
                                        steps of the current pf_run_device run); single-kernel and
                                        split pipelines only */
    float ess_fraction;              /* > 0: a sub-filter resamples only while its effective sample
                                        size (sum w)^2 / sum w^2 (FP64) is below ess_fraction * m,
                                        otherwise it keeps its propagated particles; 0: always (the
                                        reference's ADAPTIVE_RESAMPLING test sum p^2 <= thr,
                                        resampling-valias.cl:273-284, is ess_fraction = 1 / (thr m)) */
    int32_t threads_per_particle;    /* 0 or 1: one thread per particle; 2: two adjacent threads share each
                                        particle's propagate + weight (the unicycle and beacon models split
                                        their measurement sums, the DH arm its forward-kinematics chain; other
                                        models compute it on both) and sort together.  Split pipeline with
                                        PF_RNG_SUBFILTER, 2 m / ppt <= 1024 */
} pf_config;

/* One step's inputs.  control/meas are interpreted by the model:
 *   unicycle: control {v, omega};        meas {range[L], bearing[L]}
 *   dharm:    control {};                 meas {px, py, pz, yaw, pitch, roll}
 *   refarm:   control {joint rates[5]};   meas {angles[5], x, y}
 *   beacon:   control {v, omega};         meas {range[L]}
 *   camarm:   control {joint rates[5]};   meas {angles[5], pixel x, pixel y}
 * dt <= 0 uses the model's dt. */
typedef struct {
    float dt;
    float control[PF_MAX_CONTROL];
    float meas[PF_MAX_MEAS];
    float pad[7];
} pf_step_input; /* 128 bytes */

typedef struct {
    double mean[PF_MAX_STATE];  /* weighted posterior mean (circular mean for angles) */
    double log_norm;            /* log of the global normalisation sum (FP64) */
    float best[PF_MAX_STATE];   /* the reference's estimate: best particle of the best sub-filter */
    float best_key;             /* its weight (log or linear, per config) */
    int32_t best_subfilter;     /* first maximum (thrust::max_element semantics) */
    int32_t step;               /* steps completed */
    int32_t flags;              /* nonzero: device-side anomaly (NaN weights ...) */
} pf_estimate;

typedef struct {
    float dt;
    float sigma_q[3];            /* process noise std on x, y, theta */
    float sigma_range;
    float sigma_bearing;
    int32_t num_landmarks;       /* 1..8 */
    float landmarks[8][2];
    float init_state[3];
} pf_unicycle_params;

typedef struct {
    float dt;
    float sigma_qd;              /* process noise std on joint velocities */
    float sigma_pos;             /* end-effector position measurement std */
    float sigma_ang;             /* yaw/pitch/roll measurement std */
    float a[6], alpha[6], d[6];  /* standard DH parameters (theta is the joint state) */
    float init_state[12];        /* q[6], qdot[6] */
} pf_dharm_params;

typedef struct {
    float dt;
    float init_state[9];         /* angles[5], x, y, vX, vY */
} pf_refarm_params;

/* The reference's unicycle program (src/models/unicycle/particle_filter.cu:
 * 314-359): v += noise[0] n0, omega += noise[1] n1, gamma = noise[2] n2;
 * x += v/omega (sin(theta + omega dt) - sin theta),
 * y -= v/omega (cos(theta + omega dt) - cos theta), theta += (omega + gamma) dt;
 * weight = norm exp(-sum_i (|p - s_i| - z_i)^2 / (2 sigma_range^2)) with p = (x, y, 0)
 * and the reference's norm = 1e5 / (2 pi)^(L/2) (L/2 an integer division).
 * pf_beacon_default_params gives the reference's constants: 10 beacons, noise
 * (0.5, 0.1, 0.01), sigma_range = sqrt(1/2) (its exp(-sum e^2)), dt = 1, start
 * (20, 40, -pi/2). */
typedef struct {
    float dt;
    float noise[3];              /* std of the velocity, turn-rate and heading (gamma) noise */
    float sigma_range;
    int32_t num_beacons;         /* 1..16 */
    float beacons[16][3];        /* beacon positions (x, y, z) */
    float init_state[3];         /* x, y, theta */
} pf_beacon_params;

/* The reference's pinhole-camera variant of the arm
 * (src/models/robotarm/cuda/pf_model_soa_packed_code.cuh:61-145): the
 * refarm chain, then the cart's camera coordinates (cx, cy, cz) are
 * projected, xn = cx/cz, yn = cy/cz, r2 = xn^2 + yn^2, distorted
 * xd = (1 + kc1 r2 + kc2 r2^2) xn + 2 kc3 xn yn + kc4 (3 xn^2 + yn^2),
 * yd = (1 + kc1 r2 + kc2 r2^2) yn + kc3 (3 yn^2 + xn^2) + 2 kc4 xn yn, and
 * mapped to pixels (fc_x xd + cc_x, fc_y yd + cc_y).  Log weight
 * -(sum 0.1 e^2).  pf_camarm_default_params gives the reference's
 * calibration (:33-42), dt = 1 and the refarm start state. */
typedef struct {
    float dt;
    float init_state[9];         /* angles[5], x, y, vX, vY */
    float fc[2];                 /* focal lengths (pixels) */
    float cc[2];                 /* principal point (pixels) */
    float kc[4];                 /* radial kc1, kc2; tangential kc3, kc4 */
} pf_camarm_params;

typedef struct pf_filter pf_filter;

/* ---- library ---- */
const char* pf_status_string(pf_status s);
const char* pf_last_error(void);
int32_t pf_version(void);
/* Number of usable CUDA devices (0 when none). */
int32_t pf_device_count(void);
/* Model sizes: state floats, normals per particle per step, control and measurement floats. */
pf_status pf_model_info(pf_model_id model, int32_t* num_state, int32_t* num_noise,
                        int32_t* num_control, int32_t* num_meas);
/* Models compiled into the library: the built-in ones above and any added
 * with PF_MODEL (esthera_b200_model.cuh, ids >= PF_MODEL_USER_BASE).  The
 * reference's model plugin is a compile-time #include of one model header
 * (src/partfilt/cuda/pf_generic_soa.cu:43, src/models/robotarm/cuda/
 * pf_model_soa.cuh); here every model registers itself into one table when
 * the library loads.  pf_model_list writes up to cap ids and returns how many
 * are registered; pf_model_name gives a model's name (NULL if unknown). */
#define PF_MODEL_USER_BASE 64
int32_t pf_model_list(int32_t* ids, int32_t cap);
const char* pf_model_name(int32_t model);

/* ---- plain filter (replaces particle_filter()'s step loop body) ---- */
pf_status pf_config_default(pf_config* cfg);
pf_status pf_create(const pf_config* cfg, pf_model_id model, const void* params, size_t params_size,
                    pf_filter** out);
pf_status pf_destroy(pf_filter* f);
/* Every particle set to the same state (the reference's init, pf_generic_soa.cu:756-767). */
pf_status pf_set_initial_state(pf_filter* f, const float* state);
/* Host SoA arrays, num_state x (m*N) floats. */
pf_status pf_set_particles(pf_filter* f, const float* soa);
pf_status pf_get_particles(pf_filter* f, float* soa);
/* After a step: the sorted (pre-exchange) state, sorted keys, and the slot each
 * output particle was resampled from (-1: the sub-filter skipped resampling). */
pf_status pf_get_sorted(pf_filter* f, float* soa, float* keys);
pf_status pf_get_selection(pf_filter* f, int32_t* sel);
/* Turn recording of the resampling selections on or off (off by default: it costs 4 bytes per particle-step). */
pf_status pf_record_selection(pf_filter* f, int32_t enable);
/* One step with host inputs (copied H2D) and a host estimate (copied D2H); synchronous. */
pf_status pf_step(pf_filter* f, const pf_step_input* in, pf_estimate* out);
/* Device-resident run: d_inputs[capacity] and d_estimates[capacity] in device
 * memory; resets the step counter and runs `steps` steps (step k reads
 * d_inputs[k % capacity], writes d_estimates[k % capacity]).  Asynchronous on
 * the filter's stream: one step is captured into a CUDA graph (once per
 * argument set) and replayed with a device step counter.  pf_synchronize() waits. */
pf_status pf_run_device(pf_filter* f, const pf_step_input* d_inputs, pf_estimate* d_estimates,
                        int32_t capacity, int32_t steps);
/* Replays `steps` more steps of the run set up by pf_run_device (the step
 * counter continues), e.g. to time steps one at a time. */
pf_status pf_run_device_continue(pf_filter* f, int32_t steps);
/* Pipelined host stepping (no counterpart in the reference, whose driver loop
 * copies each step's estimate back before the next step starts,
 * pf_generic_soa.cu:858-1154).  pf_step_submit copies the input into a pinned
 * ring slot and returns without waiting: the slot is uploaded on a copy stream,
 * the step (the CUDA graph of pf_run_device, over device rings of
 * PF_QUEUE_DEPTH inputs and estimates) runs on the filter's stream once the
 * upload landed, and the estimate is downloaded into a pinned ring slot on a
 * second copy stream, so uploads and downloads overlap the neighbouring steps.
 * Results equal pf_step's on the same inputs (the step counter is the number of
 * steps since the initial state, as for pf_step).  At most PF_QUEUE_DEPTH steps
 * may be pending: a further submit returns PF_ERR_BUSY, as does a submit after
 * another call stepped the filter while steps are pending.
 * pf_step_collect returns up to `max` estimates in submission order; wait != 0
 * blocks until that many are done (or all pending ones), wait == 0 returns the
 * finished ones only.  One host thread per filter. */
#define PF_QUEUE_DEPTH 64
pf_status pf_step_submit(pf_filter* f, const pf_step_input* in);
pf_status pf_step_collect(pf_filter* f, pf_estimate* out, int32_t max, int32_t wait, int32_t* count);
pf_status pf_synchronize(pf_filter* f);
/* Per-launch timing: with timing on, every step records a CUDA event before its
 * first launch and after each launch (graph replays included).
 * pf_last_step_timing waits for the last step and returns the duration of
 * each launch in ms; pf_phase_name(i) names launch i ("sample_sort", ...). */
pf_status pf_set_timing(pf_filter* f, int32_t enable);
pf_status pf_last_step_timing(pf_filter* f, float* ms, int32_t cap, int32_t* n);
const char* pf_phase_name(pf_filter* f, int32_t i);
/* The filter's CUDA stream (a cudaStream_t), for timing with events. */
void* pf_stream(pf_filter* f);
/* Resolved configuration: pipeline actually used, particles per thread, torus dims, device bytes. */
pf_status pf_get_info(pf_filter* f, int32_t* pipeline, int32_t* particles_per_thread, int32_t* torus_dx,
                      int32_t* torus_dy, int64_t* device_bytes);
/* Snapshot / restore of particles, MTGP stream words and the step count (host buffer of
 * pf_snapshot_size bytes; restore rejects a buffer whose size differs with PF_ERR_INVALID,
 * before reading past it). */
int64_t pf_snapshot_size(pf_filter* f);
pf_status pf_snapshot(pf_filter* f, void* host_buf);
pf_status pf_restore(pf_filter* f, const void* host_buf, size_t size);

/* ---- shards: one filter's torus rows spread over several filters ----
 * The reference runs a filter in one process (particle_filter,
 * pf_generic_soa.cu:686) with the torus exchange of pf_generic.cu:352-393 on
 * a dx x dy grid (pf_generic_soa.cu:682-683).  A shard holds rows
 * [row0, row1) of that grid (cfg->num_subfilters is the WHOLE filter's N; the
 * exchange must be the torus, every step, with per-sub-filter streams).  Its
 * first sub-filter row0*dx and its size must be multiples of 32 (the size may
 * instead end at N).  A step is:
 *   pf_shard_sample on every shard;
 *   pf_shard_halo_copy(s, 0, lower(s)) and pf_shard_halo_copy(s, 1, upper(s))
 *     for every shard s (or pf_shard_halo_out / pf_shard_halo_in through host
 *     buffers of halo_bytes, e.g. across processes), where lower(s) is the
 *     shard whose first row follows s's last row and upper(s) the shard whose
 *     last row precedes s's first row (both on the torus);
 *   pf_shard_resample on every shard;
 *   pf_shard_group_rows on every shard, concatenated in row order into
 *     num_groups = ceil(N / 32) rows of PF_SHARD_ROW doubles and
 *     num_groups x S winner states, then pf_shard_estimate on any shard.
 * The shards' particles and the estimate then equal the whole filter's bit for
 * bit.  pf_step, pf_run_device and pf_step_submit reject a shard. */
#define PF_SHARD_ROW 32
pf_status pf_shard_create(const pf_config* cfg, pf_model_id model, const void* params, size_t params_size,
                          int32_t row0, int32_t row1, pf_filter** out);
pf_status pf_shard_info(pf_filter* f, int32_t* row0, int32_t* row1, int32_t* first_subfilter, int32_t* num_groups,
                        int64_t* halo_bytes);
pf_status pf_shard_sample(pf_filter* f, const pf_step_input* in);
pf_status pf_shard_halo_out(pf_filter* f, int32_t dir, void* host_buf);
pf_status pf_shard_halo_in(pf_filter* f, int32_t dir, const void* host_buf);
pf_status pf_shard_halo_copy(pf_filter* from, int32_t dir, pf_filter* to);
pf_status pf_shard_resample(pf_filter* f);
pf_status pf_shard_group_rows(pf_filter* f, double* rows, float* states);
pf_status pf_shard_estimate(pf_filter* f, const double* rows, const float* states, int32_t num_groups,
                            pf_estimate* out);

/* ---- batched filters: many independent filters of uneven sizes stepped together ----
 * The reference runs one filter per process (particle_filter, pf_generic_soa.cu:686);
 * these calls have no counterpart there.  Every filter shares cfg's model,
 * resampler and exchange settings (exchange stays inside each filter: none,
 * ring, or torus when every filter's N = dx*dy; all-to-all is not offered) and
 * runs the split pipeline with per-sub-filter streams.  Filter f has
 * num_particles[f] particles and params + f (params_size bytes each).  cfg's m
 * is the largest sub-filter size: filter f runs sub-filters of m_f particles,
 * the largest power of two in [32, m] that divides num_particles[f] (and for
 * the torus gives N = dx*dy and 5t <= m_f; for the ring 2t <= m_f), with cfg's
 * particles per thread where that is built for m_f, else the default
 * (pf_batch_filter_shape).  Its sub-filter b uses stream cfg.stream_offset +
 * first(f) + b, first(f) = sub-filters of filters 0..f-1 (pf_batch_filter_info),
 * so a pf_filter created with that stream_offset, m_f and ppt reproduces
 * filter f exactly. */
typedef struct pf_batch pf_batch;
pf_status pf_batch_create(const pf_config* cfg, pf_model_id model, int32_t num_filters,
                          const int32_t* num_particles, const void* params, size_t params_size, pf_batch** out);
pf_status pf_batch_destroy(pf_batch* b);
/* states: num_filters x S floats (host); every particle of filter f starts at states[f*S..]. */
pf_status pf_batch_set_initial_states(pf_batch* b, const float* states);
/* Filter f's particles (host, SoA, S x num_particles[f]). */
pf_status pf_batch_get_particles(pf_batch* b, int32_t filter, float* soa);
/* One step of every filter from host inputs[num_filters]; estimates to out[num_filters] (may be NULL). */
pf_status pf_batch_step(pf_batch* b, const pf_step_input* inputs, pf_estimate* out);
/* Enqueues `steps` steps on the batch's stream and returns: step k of filter f
 * reads d_inputs[f*capacity + k % capacity] and writes d_estimates[f*capacity +
 * k % capacity] (device arrays).  The steps are captured once into a CUDA graph
 * of up to 256 steps and replayed; pf_batch_poll reports completion without
 * blocking, pf_batch_synchronize waits. */
pf_status pf_batch_submit(pf_batch* b, const pf_step_input* d_inputs, pf_estimate* d_estimates,
                          int32_t capacity, int32_t steps);
pf_status pf_batch_poll(pf_batch* b, int32_t* done);
pf_status pf_batch_synchronize(pf_batch* b);
void* pf_batch_stream(pf_batch* b);
pf_status pf_batch_info(pf_batch* b, int32_t* num_filters, int64_t* total_particles, int32_t* total_subfilters,
                        int32_t* particles_per_thread, int64_t* device_bytes);
pf_status pf_batch_filter_info(pf_batch* b, int32_t filter, int32_t* num_subfilters, int32_t* stream_offset,
                               int64_t* particle_offset);
/* Filter f's sub-filter size m_f and particles per thread. */
pf_status pf_batch_filter_shape(pf_batch* b, int32_t filter, int32_t* particles_per_subfilter,
                                int32_t* particles_per_thread);
/* Filter f's sorted (pre-exchange) particles and keys of the last step (host, SoA). */
pf_status pf_batch_get_sorted(pf_batch* b, int32_t filter, float* soa, float* keys);

/* Autotuner for batched filters (project-written; no reference counterpart).
 * Every candidate (m from m_list x particles per thread from ppt_list x threads
 * per particle from tpp_list x exchange period from period_list) runs `steps` steps of the whole batch on `inputs`
 * (host, [F][steps]) twice -- the first run captures the CUDA graph, the second
 * is timed with CUDA events -- and, when `truth` ([F][steps][S], host) is given,
 * its tracking RMSE over steps >= burn_in is computed (angles wrapped).  A
 * candidate is accepted when its RMSE is within (1 + rmse_tol) of the mean
 * RMSE of the period-1 candidates (without truth: period-1 candidates only);
 * *best = base with the fastest accepted candidate's m, ppt, threads per
 * particle and period.  Candidates that cannot run (no sub-filter size
 * dividing some count, ppt not built for m) keep their pf_status in the
 * table. */
typedef struct {
    int32_t particles_per_subfilter;
    int32_t particles_per_thread;
    int32_t threads_per_particle;
    int32_t exchange_period;
    int32_t status;
    float ms_per_step;
    int32_t accepted;
    double particle_steps_per_s;
    double rmse;
} pf_tune_entry;
pf_status pf_batch_autotune(const pf_config* base, pf_model_id model, int32_t num_filters,
                            const int32_t* num_particles, const void* params, size_t params_size,
                            const pf_step_input* inputs, const float* truth, int32_t steps, int32_t burn_in,
                            const int32_t* m_list, int32_t n_m, const int32_t* ppt_list, int32_t n_ppt,
                            const int32_t* tpp_list, int32_t n_tpp, const int32_t* period_list, int32_t n_period,
                            float rmse_tol,
                            pf_tune_entry* table, int32_t table_cap, int32_t* n_table, pf_config* best);

/* ---- serving: many resident filters, updates batched as they arrive ----
 * No counterpart in the reference (one filter per process there).  Filters
 * of any compiled-in model share the server's pf_config template (m,
 * particles per thread, ring/no exchange, resampler, resampling_freq,
 * log_weights, mtgp_mask); each has its own particle count (a multiple of m),
 * parameters and seed (sub-filter b: parameter set b mod 200, seed + b + 1, as
 * a pf_filter with that seed).  Device memory per filter comes from a
 * stream-ordered pool; pf_server_open fails with PF_ERR_ADMISSION when the
 * filter's block (pf_server_footprint) does not fit the HBM budget or no slot
 * is free.  pf_server_update queues an update; pf_server_launch runs the
 * oldest queued update of every filter without one in flight as one batch
 * (no-op while a batch is in flight); pf_server_poll returns the finished
 * batch's results (wait = 0: without blocking).  A handle is used by one
 * host thread at a time. */
typedef struct pf_server pf_server;
typedef struct {
    int32_t filter;       /* id from pf_server_open */
    int32_t step;         /* updates completed by this filter */
    uint64_t tag;         /* the caller's tag of the update */
    int64_t particles;
    pf_estimate estimate;
} pf_server_result;
typedef struct {
    int32_t open_filters;
    int32_t in_flight;
    int64_t resident_particles;
    int64_t queued_updates;
    int64_t bytes_in_use;
    int64_t budget;
    int64_t launches;
    int64_t updates;
    int64_t particle_steps;
} pf_server_stats;
pf_status pf_server_create(const pf_config* filter_cfg, int64_t hbm_budget, int32_t max_filters, pf_server** out);
pf_status pf_server_destroy(pf_server* s);
int64_t pf_server_footprint(const pf_server* s, pf_model_id model, int32_t num_particles);
pf_status pf_server_open(pf_server* s, pf_model_id model, const void* params, size_t params_size,
                         int32_t num_particles, uint32_t seed, int32_t* id);
pf_status pf_server_close(pf_server* s, int32_t id);
pf_status pf_server_update(pf_server* s, int32_t id, const pf_step_input* in, uint64_t tag);
pf_status pf_server_launch(pf_server* s, int32_t* n_launched);
pf_status pf_server_poll(pf_server* s, int32_t wait, pf_server_result* out, int32_t cap, int32_t* n);
pf_status pf_server_stats_get(pf_server* s, pf_server_stats* st);
/* Current particles, sorted copy and sorted keys of filter id (host; any may be NULL). */
pf_status pf_server_get_particles(pf_server* s, int32_t id, float* soa, float* sorted_soa, float* keys);
/* Per-filter snapshot / restore (no counterpart in the reference), e.g. to move
 * a filter to another server or GPU: the snapshot holds the filter's model,
 * particle count, particles, MTGP32 stream words and update count.  Both need
 * the filter idle (no update queued or in flight: PF_ERR_BUSY otherwise).
 * Restore targets an open filter of the same model and particle count (opened
 * with the same parameters for the same results) and replaces its particles,
 * streams and update count; its next updates then give the results the
 * snapshotted filter would have given.  Restore takes the buffer's size and
 * rejects one that is not pf_server_snapshot_size bytes (a truncated transfer)
 * with PF_ERR_INVALID before reading past it. */
int64_t pf_server_snapshot_size(const pf_server* s, int32_t id);
pf_status pf_server_snapshot(pf_server* s, int32_t id, void* host_buf);
pf_status pf_server_restore(pf_server* s, int32_t id, const void* host_buf, size_t size);

/* ---- the served tracking load (request loop over pf_server_*, host C) ----
 * Poisson arrivals at `rate` per second for `duration_s`; each request is a
 * unicycle (probability frac_unicycle) or DH-arm filter with a log-uniform
 * particle count in [min_particles, max_particles] (rounded to m), a uniform
 * number of updates in [min_updates, max_updates] spaced uniformly in
 * [min_gap_ms, max_gap_ms].  Everything is generated from `seed`.  The loop
 * runs in real time on the calling thread and fills the report; it stops
 * drain_limit_s after the last arrival if work is left (report.incomplete). */
typedef struct {
    double rate;
    double duration_s;
    double frac_unicycle;
    int32_t min_particles, max_particles;
    int32_t min_updates, max_updates;
    double min_gap_ms, max_gap_ms;
    uint32_t seed;
    int32_t max_filters;
    int64_t hbm_budget;
    int32_t norm_check_every;  /* every k-th request: FP64 check of its last normalisation (0: off) */
    int32_t pad0;
    double drain_limit_s;
} pf_load_config;
typedef struct {
    int64_t requests, admitted, admission_waits, completed_requests, updates, launches;
    int64_t max_resident_particles, max_bytes_in_use;
    int32_t max_open_filters, incomplete;
    double wall_s, particle_steps, particle_steps_per_s, demanded_particle_steps_per_s, mean_batch;
    double lat_p50_ms, lat_p99_ms, lat_p999_ms, lat_max_ms;
    int64_t norm_checked;
    double norm_err_max, norm_err_mean;  /* |log_norm - FP64 log-sum-exp| / max(1, |.|) */
} pf_load_report;
pf_status pf_load_default(pf_load_config* c);
pf_status pf_serve_load(const pf_config* filter_cfg, const pf_load_config* load, pf_load_report* report);

/* ---- kernel-level entry points (device work on host arrays; used by parity tests) ---- */
/* MTGP32 in the reference block layout: streams g = 0..G-1 with parameter set g,
 * seed + g + 1; out[g*per_stream + i].  kind 0: uint32, 1: float bits in [1,2).
 * Replaces mtgp32_uint32_kernel / mtgp32_single_kernel (mtgp32-cuda.cu:180-306). */
pf_status pfk_mtgp_generate(int32_t G, uint32_t seed, uint32_t mask, int32_t kind,
                            int64_t per_stream, int32_t calls, uint32_t* out);
/* Failure detection without a fault (no counterpart in the reference): one
 * CTA waits, at most `limit` polls (1..2^20), on an mbarrier phase that
 * nothing completes -- the bounded wait the resampling kernels use for their
 * bulk copies -- and *status receives the kernel's report: 1 (the wait ran out;
 * the kernels set the same bit in a filter's status word, which pf_step /
 * pf_synchronize return as PF_ERR_TIMEOUT), 0 had it completed.  The context
 * stays usable. */
pf_status pfk_bounded_wait_test(int32_t limit, int32_t* status);
/* The same wait made CTA-wide, with a bulk copy of 32 KB really in flight
 * into shared memory and a poll limit per thread (limits[nthreads], 0..2^20;
 * 0: that thread gives up at once while the others may see the copy land).
 * The threads agree on one outcome: outcome[tid] = 1 (landed within the
 * first wait), 0 (some thread ran out; the copy landed in the second wait, so
 * the kernels report PF_ERR_TIMEOUT and keep their propagated particles) or
 * -1 (the copy may still be in flight: the kernel leaves that shared memory
 * alone).  *copied = 1 when the shared words equal the source once the block
 * went on, 0 when not, -1 after outcome -1.  nthreads: 32..1024, a multiple
 * of 32.  No counterpart in the reference. */
pf_status pfk_bounded_wait_mixed_test(const int32_t* limits, int32_t nthreads, int32_t* outcome, int32_t* copied);
/* In-place Box-Muller over pairs (2i, 2i+1), 2i < n (boxmuller, pf_generic_soa.cu:481-500).
 * data must hold 2*ceil(n/2) floats. */
pf_status pfk_boxmuller(float* data, int64_t n);
/* nsub independent descending bitonic sorts of m keys; idx receives the permutation
 * (block_sort + bitonic_sort, pf_generic_soa.cu:289-323, bitonic-sort.cu:11-61). */
pf_status pfk_bitonic_sort(float* keys, int32_t* idx, int32_t m, int32_t nsub, int32_t ppt);
/* The same sort as the sampling kernels run it for models whose keys rarely
 * tie (unicycle, beacon): the network on the keys alone, the permutation
 * recovered by rank; a sub-filter with equal keys (ties, +0/-0, repeated
 * -inf) or a NaN key falls back to the (key, index) network, so the result
 * equals pfk_bitonic_sort's in every case.  *fallbacks receives how many
 * sub-filters fell back.  (No counterpart in the reference.) */
pf_status pfk_rank_sort(float* keys, int32_t* idx, int32_t m, int32_t nsub, int32_t ppt, int32_t* fallbacks);
/* nsub sub-filters of m weights (linear FP32, slot order) -> sel[nsub*m].
 * u: REFERENCE: m raw uniforms in [1,2) per sub-filter; SYSTEMATIC: 1 value in [0,1);
 * VOSE: 2m values in [0,1) (x, y pairs).  ppt: particles per thread (scan grouping). */
pf_status pfk_resample(int32_t resampler, const float* w, const float* u, int32_t m, int32_t nsub,
                       int32_t ppt, int32_t* sel);
/* Vose tables (prob, alias) of nsub sub-filters (vose_alias_init, resampling-valias.cl:111-195). */
pf_status pfk_vose_build(const float* w, int32_t m, int32_t nsub, int32_t ppt, float* prob,
                         uint32_t* alias);
/* Slot sources after exchange for N sub-filters (identity where not replaced). */
pf_status pfk_exchange_sources(int32_t mode, int32_t N, int32_t m, int32_t t,
                               const float* sorted_keys, int32_t* src);
/* One model propagate + log-likelihood for n particles (SoA state in/out, noise SoA K x n). */
pf_status pfk_model_step(pf_model_id model, const void* params, size_t params_size,
                         const pf_step_input* in, int32_t n, float* state, const float* noise,
                         float* loglik);

/* Posterior estimate of num_particles particles (keys[T] log or linear weights, state SoA
 * num_state x T, m per sub-filter): FP64 weighted mean (circular for the variables in
 * angle_mask), log normalisation sum, first-maximum winner.  Host arrays. */
pf_status pfk_estimate(const float* keys, const float* state, int32_t num_state, int64_t num_particles,
                       int32_t m, uint32_t angle_mask, int32_t log_weights, pf_estimate* out);

/* pfk_estimate for callers that cannot allocate device memory (a pool or arena
 * owns every allocation, the allocator is locked after start-up, or no
 * allocation may happen between stream captures).  No counterpart in the
 * reference.  Inputs and output are device pointers the caller owns; it calls
 * no cudaMalloc/cudaFree: its per-sub-filter scratch is a static device array
 * sized for at most 4096 sub-filters (num_particles / m), about 1.15 MB held
 * by every GPU that loads the library.  Larger inputs return PF_ERR_INVALID.
 * The first call on a device looks up the array's device address (make that
 * call before any stream capture); the address is kept per device and CUDA
 * context, so the first call after cudaDeviceReset (or from another context
 * on the same device) looks it up again.  All calls share the array and every call
 * overwrites the entries it reads, so nothing needs clearing; calls that
 * overlap on the GPU (other streams, other threads) race on it.
 * Asynchronous on `stream` (a cudaStream_t, NULL = default stream). */
pf_status pfk_estimate_noalloc(const float* d_keys, const float* d_state, int32_t num_state,
                               int64_t num_particles, int32_t m, uint32_t angle_mask,
                               int32_t log_weights, pf_estimate* d_out, void* stream);

/* ---- synthetic traces (seeded ground truth + measurements) ---- */
/* Unicycle: landmarks uniform in [-10,10]^2, truth from (0,0,0), v=1, omega=0.3 sin(0.05 t). */
pf_status pf_unicycle_default_params(uint32_t seed, int32_t num_landmarks, pf_unicycle_params* p);
pf_status pf_dharm_default_params(uint32_t seed, pf_dharm_params* p);
/* The reference unicycle program's constants (particle_filter.cu:60-76, 708-716). */
pf_status pf_beacon_default_params(pf_beacon_params* p);
/* The reference's camera calibration (pf_model_soa_packed_code.cuh:33-42). */
pf_status pf_camarm_default_params(pf_camarm_params* p);
/* steps x pf_step_input and steps x num_state truth floats. */
pf_status pf_make_trace(pf_model_id model, const void* params, uint32_t seed, int32_t steps,
                        pf_step_input* inputs, float* truth);

/* ---- reference-compatible driver (reference trace files, C host) ---- */
/* Parses one line of a reference trace.  PF_MODEL_REFARM and PF_MODEL_CAMARM:
 * robot-arm format "x y angles[5] controls[5] dt actual_x actual_y
 * actual_angles[5]" (pf_model_soa.cuh:276-301; pf_model_soa_packed_code.c:57-82,
 * where x y are pixels).  PF_MODEL_BEACON: unicycle format
 * "ranges[10] v omega dt actual_x actual_y actual_theta"
 * (src/models/unicycle/particle_filter.cu:756-772).  Returns PF_OK,
 * PF_ERR_IO at end of file / bad line, PF_ERR_UNSUPPORTED for the models
 * without a reference trace format (unicycle, DH arm). */
pf_status pf_read_trace_line(void* file, pf_model_id model, pf_step_input* in, float* actual);
/* The reference's estimate_error for the robot-arm model (pf_model_soa.cuh:303-316). */
float pf_refarm_estimate_error(const float* est, const float* actual);
/* The unicycle program's error: position distance |est.xy - actual.xy|
 * (particle_filter.cu:1044). */
float pf_beacon_estimate_error(const float* est, const float* actual);
/* Drop-in for the reference driver: runs the robot-arm filter over a trace file with
 * the reference's defaults (ring exchange, multinomial resampling) and returns the
 * mean estimate error through *mean_error. */
pf_status pf_particle_filter(int32_t num_particles, int32_t num_blocks, int32_t num_transfer,
                             float resampling_freq, const char* input_file, float* mean_error);
/* Drop-in for the unicycle program's main loop (particle_filter.cu:596-1160):
 * the beacon filter with the default constants over a unicycle trace file
 * (ring exchange of num_transfer particles, multinomial resampling every
 * step), returning the mean position error of the best particle. */
pf_status pf_beacon_particle_filter(int32_t num_particles, int32_t num_blocks, int32_t num_transfer,
                                    const char* input_file, float* mean_error);

#ifdef __cplusplus
}
#endif
#endif
