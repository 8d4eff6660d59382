/*
 * pf_oracle.h -- CPU restatement of the Esthera distributed particle-filter
 * step, used ONLY as test infrastructure: the parity checker for the CUDA
 * path and the timed CPU baseline.  Nothing in the product links this.
 *
 * Every function cites the reference routine it restates (paths relative to
 * the Esthera source tree).  Parity pinning: the MTGP32 restatement is
 * checked against the reference's own CPU generator (mtgp32-fast.c, built
 * by oracle/build_ref.sh into oracle/_ref/) and against committed golden
 * vectors; the sort / scan / resampling restatements are checked against
 * golden vectors produced by this oracle and against hand-derived cases.
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- MTGP32-11213 ---------------- */
#define ORC_MTGP_N 351        /* state words (mexp/32 + 1) */
#define ORC_MTGP_SETS 200     /* parameter sets in the dynamic-creator table */
#define ORC_MTGP_MASK 0xfff80000u   /* mask stored in every parameter set */
#define ORC_MTGP_MASK_CUDA_REF 0xff800000u /* constant hard-wired in the reference CUDA kernel */

/* Fill st[351] for parameter set `set` and `seed`.
 * Restates mtgp32_init_state (src/partfilt/cuda/mtgp/mtgp32-fast.c:119-137). */
void orc_mtgp_init_state(uint32_t* st, int set, uint32_t seed);

/* Sequential generation of n outputs from the stream whose 351-word state is
 * st (advanced in place).  kind 0: tempered uint32 (mtgp32_genrand_uint32,
 * mtgp32-fast.h:248-263); kind 1: float bits in [1,2)
 * (mtgp32_genrand_close1_open2, mtgp32-fast.h:274-289).  mask 0 means the
 * parameter set's own mask. */
void orc_mtgp_generate(uint32_t* st, int set, uint32_t mask, int kind, int64_t n, uint32_t* out);

/* Reference block layout (mtgp32_single_kernel, mtgp32-cuda.cu:259-306;
 * mtgp32-opencl.cl:186): G streams, stream g uses parameter set g and writes
 * out[g*(total/G) + i].  states holds G*351 words, advanced in place. */
void orc_mtgp_generate_blocks(uint32_t* states, int G, uint32_t mask, int kind,
                              int64_t total, uint32_t* out);

/* ---------------- Box-Muller ---------------- */
/* In-place over pairs (2i, 2i+1) for all i with 2i < n, inputs in [1,2):
 * u1 = 2-x, u2 = 2-y, z = sqrt(-2 ln u1) * (cos 2 pi u2, sin 2 pi u2).
 * Restates boxmuller (src/partfilt/cuda/pf_generic_soa.cu:481-500;
 * src/partfilt/opencl/pf_generic.cl:465-483), evaluated in double. */
void orc_boxmuller(float* data, int64_t n);

/* ---------------- sub-filter primitives ---------------- */
/* Descending bitonic key+index sort of m (power of two) elements, the exact
 * comparator network of bitonic_sort with dir=0 (equal keys are swapped).
 * Restates src/partfilt/cuda/bitonic-sort.cu:11-61. */
void orc_bitonic_sort_desc(float* key, int32_t* idx, int m);

/* FP32 Blelloch work-efficient exclusive scan in place; returns the total.
 * Restates prefix_sum (src/partfilt/cuda/pf_generic_soa.cu:169-216). */
float orc_blelloch_scan(float* w, int m);

/* Last index i with hay[i] <= needle (0 if none).
 * Restates binary_search (pf_generic_soa.cu:221-240). */
int orc_binary_search(const float* hay, float needle, int m);

/* Reference multinomial resampling of one sub-filter: w (m FP32 weights in
 * slot order), u (m raw uniforms in [1,2)); sel[i] = chosen slot.
 * Restates resampling (pf_generic_soa.cu:415-453, MTGP branch). */
void orc_resample_ref(const float* w, const float* u, int m, int32_t* sel);

/* Canonical FP64 inclusive scan used by the systematic resampler: each
 * group of `ept` consecutive weights is summed sequentially, the group totals
 * are scanned with a Kogge-Stone scan inside 32-group warps, and the warp
 * totals with a Kogge-Stone scan across warps.  Returns the total. */
double orc_scan_f64(const float* w, int m, int ept, double* cum);

/* Systematic resampling with the canonical FP64 scan: pos_i = (u0 + i) *
 * (total / m), sel[i] = number of slots whose inclusive sum is <= pos_i,
 * clamped to m-1.  u0 in [0,1). */
double orc_resample_systematic(const float* w, int m, int ept, float u0, int32_t* sel);

/* Vose alias table of one sub-filter (FP32), canonical work-list order
 * (ascending slot index where the reference uses atomic_inc/atomic_dec).
 * Restates sum_reduce4 + vose_alias_init + normalisation of
 * resampling_valias (src/partfilt/opencl/resampling-valias.cl:85-195, 262-270). */
/* The alias build's starting probabilities p_i m (p_i = w_i / sum_reduce4(w),
 * or 1/m when the sum is not positive; resampling-valias.cl:117, 262-270). */
void orc_vose_scaled(const float* w, int m, float* scaled);
void orc_vose_build(const float* w, int m, float* prob, uint32_t* alias);
/* One draw (vose_alias_generate_next, resampling-valias.cl:198-202); ux, uy in [0,1). */
uint32_t orc_vose_draw(const float* prob, const uint32_t* alias, int m, float ux, float uy);

/* ---------------- exchange routing ---------------- */
#define ORC_EXCH_NONE 0
#define ORC_EXCH_RING 1
#define ORC_EXCH_TORUS 2
#define ORC_EXCH_ALL2ALL 3
/* 2D torus dimensions: dx = 2^floor(log2 sqrt N), dy = N / dx
 * (src/partfilt/cuda/pf_generic.cu:682-683). */
void orc_torus_dims(int N, int* dx, int* dy);
/* For every slot (b*m + s) the global slot it takes its particle from after
 * the exchange (identity for slots not replaced).  top_keys[b*t + j] is the
 * key of sub-filter b's sorted slot j (only used by ALL2ALL).
 * ring: pf_generic_soa.cu:400-413; torus: pf_generic.cu:352-393 with
 * receiver slots m-1-j-k*t; all-to-all: pf_generic2_all2all.cu:294-331,
 * 404-419, 1007. */
void orc_exchange_sources(int mode, int N, int m, int t, const float* top_keys, int32_t* src);

/* ---------------- models ---------------- */
#define ORC_MODEL_UNICYCLE 0
#define ORC_MODEL_DHARM 1
#define ORC_MODEL_REFARM 2
#define ORC_MODEL_BEACON 3
#define ORC_MODEL_CAMARM 4

typedef struct {
    int model;
    int num_state;   /* floats per particle */
    int num_noise;   /* standard normals per particle per step */
    /* unicycle */
    double dt, sq[3], sigma_r, sigma_b;
    int num_landmarks;
    double lm[8][2];
    /* DH arm */
    double sigma_qd, sigma_p, sigma_a;
    double a[6], alpha[6], d[6];
    /* beacon (range-only unicycle): velocity / turn-rate / heading noise std,
     * beacon positions; sigma_r is the range std */
    double bnoise[3];
    int num_beacons;
    double bc[16][3];
    /* camera arm: focal lengths, principal point, distortion kc1..kc4 */
    double fc[2], cc[2], kc[4];
} orc_model;

/* control / measurement as flat float arrays:
 *   unicycle: control {v, omega}; measurement {range[L], bearing[L]}
 *   dharm:    control {} ;        measurement {px,py,pz,yaw,pitch,roll}
 *   refarm:   control {angles[5]}; measurement {angles[5], x, y}
 *   beacon:   control {v, omega}; measurement {range[L]}
 *   camarm:   control {angles[5]}; measurement {angles[5], pixel x, pixel y} */

/* Propagate one particle in place (state has num_state floats, noise has
 * num_noise normals) and return its log-likelihood.  Double precision. */
double orc_model_step(const orc_model* mdl, float* state, const float* noise,
                      const float* control, const float* meas);

/* ---------------- whole filter ---------------- */
#define ORC_RES_REF 0        /* reference multinomial, FP32 Blelloch */
#define ORC_RES_SYSTEMATIC 1 /* systematic, FP64 canonical scan */
#define ORC_RES_VOSE 2       /* Vose alias */

#define ORC_RNG_REFLAYOUT 0  /* G streams in the reference block layout */
#define ORC_RNG_SUBFILTER 1  /* one stream per sub-filter */

typedef struct {
    orc_model mdl;
    int m, N, t, exchange, resampler, rng, G, ept, log_weights;
    float freq;
    uint32_t seed, mask;
    int64_t T;
    float* state;     /* num_state * T, SoA */
    float* tmp;       /* num_state * T, sorted */
    float* tkey;      /* T sorted keys */
    uint32_t* mtgp;   /* streams * 351 */
    int streams;
    float* rbuf;      /* random buffer (reference layout) */
    int64_t rtotal;
    float ess_frac;   /* > 0: a sub-filter resamples only while (sum w)^2 / sum w^2 < ess_frac * m
                         (the reference's ADAPTIVE_RESAMPLING test, resampling-valias.cl:273-284,
                         with its threshold thr = 1 / (ess_frac * m)); 0 after init */
    int soff;         /* ORC_RNG_SUBFILTER: sub-filter b draws the stream of a whole filter's
                         sub-filter soff + b (orc_filter_set_stream_offset); 0 after init */
} orc_filter;

typedef struct {
    double mean[16];     /* weighted mean state (circular mean for angles) */
    double log_norm;     /* log of the global normalisation sum */
    float best_key;      /* global winner key */
    int32_t best_sub;    /* global winner sub-filter (first max) */
    float best[16];      /* winner particle state */
} orc_estimate;

int orc_filter_init(orc_filter* f, const orc_model* mdl, int m, int N, int t, int exchange,
                    int resampler, int rng, int G, int ept, int log_weights, float freq,
                    uint32_t seed, uint32_t mask, const float* init_state);
void orc_filter_free(orc_filter* f);
/* One full step: RNG, propagate + weight, sort, winner, estimate, exchange,
 * resample.  Optional outputs (may be NULL): sel (T selected slot indices,
 * -1 for sub-filters that skipped resampling). threads <= 0: all cores. */
int orc_filter_step(orc_filter* f, const float* control, const float* meas,
                    orc_estimate* est, int32_t* sel, int threads);
/* The two halves of orc_filter_step: orc_filter_sample runs steps RNG,
 * propagate + weight, sort, winner and estimate (state propagated in place,
 * tmp / tkey the sorted copy); orc_filter_resample runs the exchange and the
 * resampling from tmp / tkey with this step's uniforms into state.  A test
 * may replace tmp / tkey in between (e.g. with a device's own sorted copy) to
 * check exchange routing and resampling given identical weights. */
/* ORC_RNG_SUBFILTER: re-seed so that sub-filter b draws stream off + b
 * (parameter set (off + b) mod 200, seed + off + b + 1), the streams of rows
 * of a larger filter that starts at sub-filter off.  Returns -1 for the
 * reference layout. */
int orc_filter_set_stream_offset(orc_filter* f, int off);
int orc_filter_sample(orc_filter* f, const float* control, const float* meas,
                      orc_estimate* est, int threads);
int orc_filter_resample(orc_filter* f, int32_t* sel, int threads);

/* exp of a max-subtracted log-weight (x <= 0) from correctly rounded FP32
 * operations only, bit-identical to the engine's resampling weights. */
float orc_expneg(float x);

/* Number of uniforms one sub-filter stream consumes per step in
 * ORC_RNG_SUBFILTER mode. */
int64_t orc_stream_draws(int num_noise, int m, int resampler);

#ifdef __cplusplus
}
#endif
#endif
