/*
 * pf_driver.c -- reference-compatible host driver (C): the robot-arm and
 * unicycle trace readers, the reference's estimate errors and the driver
 * loops, on top of the engine's C ABI.
 *
 * Restates src/partfilt/cuda/pf_generic_soa.cu:686-1302 (driver loop),
 * src/models/robotarm/cuda/pf_model_soa.cuh:276-316 (read_trace,
 * estimate_error) and src/models/unicycle/particle_filter.cu:596-1160 (the
 * unicycle program's loop, trace format and error).  Errors are returned as
 * pf_status; nothing exits.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "esthera_b200.h"

pf_status pf_read_trace_line(void* file, pf_model_id model, pf_step_input* out, float* actual_out)
{
    FILE* fp = (FILE*)file;
    if (!fp || !out || !actual_out) return PF_ERR_INVALID;
    if (model == PF_MODEL_BEACON) {
        /* "ranges[10] v omega dt x y theta" (particle_filter.cu:756-772) */
        pf_step_input in;
        float a[3];
        memset(&in, 0, sizeof(in));
        for (int i = 0; i < 10; ++i)
            if (fscanf(fp, "%f", &in.meas[i]) != 1) return PF_ERR_IO;
        if (fscanf(fp, "%f %f %f %f %f %f", &in.control[0], &in.control[1], &in.dt, &a[0], &a[1], &a[2]) != 6)
            return PF_ERR_IO;
        *out = in;
        memcpy(actual_out, a, sizeof(a));
        return PF_OK;
    }
    if (model != PF_MODEL_REFARM && model != PF_MODEL_CAMARM) return PF_ERR_UNSUPPORTED;
    pf_step_input in;
    float actual[9];
    memset(&in, 0, sizeof(in));
    float mx, my, dt, ax, ay;
    if (fscanf(fp, "%f %f", &mx, &my) != 2) return PF_ERR_IO;
    for (int i = 0; i < 5; ++i)
        if (fscanf(fp, "%f", &in.meas[i]) != 1) return PF_ERR_IO;
    for (int i = 0; i < 5; ++i)
        if (fscanf(fp, "%f", &in.control[i]) != 1) return PF_ERR_IO;
    if (fscanf(fp, "%f %f %f", &dt, &ax, &ay) != 3) return PF_ERR_IO;
    for (int i = 0; i < 5; ++i)
        if (fscanf(fp, "%f", &actual[i]) != 1) return PF_ERR_IO;
    in.meas[5] = mx;
    in.meas[6] = my;
    in.dt = dt;
    actual[5] = ax;
    actual[6] = ay;
    actual[7] = 0.0f;
    actual[8] = 0.0f;
    *out = in;
    memcpy(actual_out, actual, sizeof(actual));
    return PF_OK;
}

float pf_refarm_estimate_error(const float* est, const float* act)
{
    float e = 0.0f;
    e += (est[5] - act[5]) * (est[5] - act[5]) * 0.1f;
    e += (est[6] - act[6]) * (est[6] - act[6]) * 0.1f;
    for (int i = 0; i < 5; ++i) e += (est[i] - act[i]) * (est[i] - act[i]) * 0.1f;
    return e;
}

float pf_beacon_estimate_error(const float* est, const float* act)
{
    const float dx = est[0] - act[0], dy = est[1] - act[1];
    return sqrtf(dx * dx + dy * dy);
}

pf_status pf_particle_filter(int32_t num_particles, int32_t num_blocks, int32_t num_transfer,
                             float resampling_freq, const char* input_file, float* mean_error)
{
    if (!input_file) return PF_ERR_INVALID;
    FILE* fp = fopen(input_file, "r");
    if (!fp) return PF_ERR_IO;
    pf_config cfg;
    pf_config_default(&cfg);
    cfg.particles_per_subfilter = num_particles;
    cfg.num_subfilters = num_blocks;
    cfg.num_transfer = num_transfer;
    cfg.exchange = num_transfer > 0 ? PF_EXCHANGE_RING : PF_EXCHANGE_NONE;
    cfg.resampler = PF_RESAMPLE_REFERENCE;
    cfg.resampling_freq = resampling_freq;
    cfg.rng = PF_RNG_REFLAYOUT;
    cfg.mtgp_streams = 120;
    cfg.log_weights = 0;
    cfg.pipeline = PF_PIPELINE_PHASED;
    pf_refarm_params p;
    memset(&p, 0, sizeof(p));
    p.dt = 1.0f;
    for (int i = 0; i < 5; ++i) p.init_state[i] = 0.75f * 3.14159265358979323846f;
    p.init_state[5] = 7.0f;
    pf_filter* f = NULL;
    pf_status s = pf_create(&cfg, PF_MODEL_REFARM, &p, sizeof(p), &f);
    if (s != PF_OK) {
        fclose(fp);
        return s;
    }
    pf_step_input in;
    float actual[PF_MAX_STATE];
    pf_estimate est;
    double err = 0.0;
    int n = 0;
    while (pf_read_trace_line(fp, PF_MODEL_REFARM, &in, actual) == PF_OK) {
        s = pf_step(f, &in, &est);
        if (s != PF_OK) break;
        err += pf_refarm_estimate_error(est.best, actual);
        ++n;
    }
    fclose(fp);
    pf_destroy(f);
    if (s != PF_OK) return s;
    if (mean_error) *mean_error = n > 0 ? (float)(err / n) : 0.0f;
    return PF_OK;
}

/* The unicycle program's loop: every particle starts at the default pose, each
 * trace line is one step, the error of a step is the position distance of the
 * best particle of the best sub-filter (particle_filter.cu:1031-1045), and the
 * mean over the steps is returned.  The reference program's resampling kernel
 * writes each particle back to its own slot instead of the selected one
 * (particle_filter.cu:503), so its selection has no effect; here the
 * sub-filters resample every step with the reference's multinomial rule. */
pf_status pf_beacon_particle_filter(int32_t num_particles, int32_t num_blocks, int32_t num_transfer,
                                    const char* input_file, float* mean_error)
{
    if (!input_file) return PF_ERR_INVALID;
    FILE* fp = fopen(input_file, "r");
    if (!fp) return PF_ERR_IO;
    pf_config cfg;
    pf_config_default(&cfg);
    cfg.particles_per_subfilter = num_particles;
    cfg.num_subfilters = num_blocks;
    cfg.num_transfer = num_transfer;
    cfg.exchange = num_transfer > 0 ? PF_EXCHANGE_RING : PF_EXCHANGE_NONE;
    cfg.resampler = PF_RESAMPLE_REFERENCE;
    cfg.resampling_freq = 1.0f;
    cfg.pipeline = PF_PIPELINE_SPLIT;
    pf_beacon_params p;
    pf_beacon_default_params(&p);
    pf_filter* f = NULL;
    pf_status s = pf_create(&cfg, PF_MODEL_BEACON, &p, sizeof(p), &f);
    if (s != PF_OK) {
        fclose(fp);
        return s;
    }
    pf_step_input in;
    float actual[PF_MAX_STATE];
    pf_estimate est;
    double err = 0.0;
    int n = 0;
    while (pf_read_trace_line(fp, PF_MODEL_BEACON, &in, actual) == PF_OK) {
        s = pf_step(f, &in, &est);
        if (s != PF_OK) break;
        err += pf_beacon_estimate_error(est.best, actual);
        ++n;
    }
    fclose(fp);
    pf_destroy(f);
    if (s != PF_OK) return s;
    if (mean_error) *mean_error = n > 0 ? (float)(err / n) : 0.0f;
    return PF_OK;
}
