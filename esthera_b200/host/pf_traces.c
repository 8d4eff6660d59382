/*
 * pf_traces.c -- seeded synthetic ground truth and measurements for the
 * unicycle, Denavit-Hartenberg arm and beacon (range-only unicycle) models
 * (host C).
 *
 * No public dataset is involved: every trace is generated from a seed.  The
 * random source is SplitMix64 (Steele, Lea, Flood 2014) with Box-Muller
 * normals in double precision; it is independent of the filter's MTGP32
 * streams.
 */
#include <math.h>
#include <string.h>

#include "esthera_b200.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct {
    uint64_t s;
} sm64_t;

static uint64_t sm64_next(sm64_t* r)
{
    uint64_t z = (r->s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static double sm64_unif(sm64_t* r) { return (double)(sm64_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static double sm64_gauss(sm64_t* r)
{
    double u1 = 1.0 - sm64_unif(r), u2 = sm64_unif(r);
    return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

static double wrap(double a) { return a - 2.0 * M_PI * floor((a + M_PI) / (2.0 * M_PI)); }

pf_status pf_unicycle_default_params(uint32_t seed, int32_t num_landmarks, pf_unicycle_params* p)
{
    if (!p || num_landmarks < 1 || num_landmarks > 8) return PF_ERR_INVALID;
    memset(p, 0, sizeof(*p));
    p->dt = 0.1f;
    p->sigma_q[0] = 0.05f;
    p->sigma_q[1] = 0.05f;
    p->sigma_q[2] = 0.01f;
    p->sigma_range = 0.2f;
    p->sigma_bearing = 0.05f;
    p->num_landmarks = num_landmarks;
    sm64_t r = {0x4c414e444d41524bULL ^ ((uint64_t)seed << 20)};
    for (int j = 0; j < num_landmarks; ++j) {
        p->landmarks[j][0] = (float)(-10.0 + 20.0 * sm64_unif(&r));
        p->landmarks[j][1] = (float)(-10.0 + 20.0 * sm64_unif(&r));
    }
    return PF_OK;
}

pf_status pf_dharm_default_params(uint32_t seed, pf_dharm_params* p)
{
    if (!p) return PF_ERR_INVALID;
    memset(p, 0, sizeof(*p));
    p->dt = 0.01f;
    p->sigma_qd = 0.01f;
    p->sigma_pos = 0.005f;
    p->sigma_ang = 0.02f;
    sm64_t r = {0x4448415241524d53ULL ^ ((uint64_t)seed << 20)};
    static const double alphas[3] = {0.0, M_PI / 2, -M_PI / 2};
    for (int i = 0; i < 6; ++i) {
        p->a[i] = (float)(0.2 + 0.4 * sm64_unif(&r));
        int k = (int)(3.0 * sm64_unif(&r));
        p->alpha[i] = (float)alphas[k > 2 ? 2 : k];
        p->d[i] = 0.0f;
    }
    for (int i = 0; i < 6; ++i) {
        p->init_state[i] = (float)(-M_PI / 2 + M_PI * sm64_unif(&r));
        p->init_state[6 + i] = (float)(-0.5 + sm64_unif(&r));
    }
    return PF_OK;
}

/* The reference unicycle program's constants: the fixed beacon positions and
 * noise levels of src/models/unicycle/particle_filter.cu:60-76, the start pose
 * of :708-716, dt = 1 (its trace generator, generate_input.py:31-36), and
 * sigma_range = sqrt(1/2), which makes the log weight -sum e^2 as in its
 * importance_weight (:340-359). */
pf_status pf_beacon_default_params(pf_beacon_params* p)
{
    static const float bx[10] = {12, 12, 13, 14, 16, 16, 18, 20, 20, 20};
    static const float by[10] = {12, 37, 25, 18, 12, 37, 30, 12, 25, 37};
    if (!p) return PF_ERR_INVALID;
    memset(p, 0, sizeof(*p));
    p->dt = 1.0f;
    p->noise[0] = 0.5f;
    p->noise[1] = 0.1f;
    p->noise[2] = 0.01f;
    p->sigma_range = (float)sqrt(0.5);
    p->num_beacons = 10;
    for (int j = 0; j < 10; ++j) {
        p->beacons[j][0] = bx[j];
        p->beacons[j][1] = by[j];
        p->beacons[j][2] = 3.0f;
    }
    p->init_state[0] = 20.0f;
    p->init_state[1] = 40.0f;
    p->init_state[2] = (float)(-M_PI / 2);
    return PF_OK;
}

/* The reference pinhole camera's calibration
 * (src/models/robotarm/cuda/pf_model_soa_packed_code.cuh:33-42) and the
 * robot-arm start state (angles 3/4 pi, x = 7). */
pf_status pf_camarm_default_params(pf_camarm_params* p)
{
    if (!p) return PF_ERR_INVALID;
    memset(p, 0, sizeof(*p));
    p->dt = 1.0f;
    for (int i = 0; i < 5; ++i) p->init_state[i] = (float)(0.75 * M_PI);
    p->init_state[5] = 7.0f;
    p->fc[0] = 408.65831f;
    p->fc[1] = 409.69059f;
    p->cc[0] = 166.32611f;
    p->cc[1] = 108.93539f;
    p->kc[0] = -0.21561f;
    p->kc[1] = 1.60704f;
    p->kc[2] = -0.01291f;
    p->kc[3] = 0.00007f;
    return PF_OK;
}

/* Forward kinematics of the standard DH chain: position p[3] and ZYX yaw/pitch/roll. */
static void dh_fk(const pf_dharm_params* P, const double* q, double* out6)
{
    double R[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, p[3] = {0, 0, 0};
    for (int i = 0; i < 6; ++i) {
        double ct = cos(q[i]), st = sin(q[i]), ca = cos(P->alpha[i]), sa = sin(P->alpha[i]);
        double Ra[3][3] = {{ct, -st * ca, st * sa}, {st, ct * ca, -ct * sa}, {0, sa, ca}};
        double pa[3] = {P->a[i] * ct, P->a[i] * st, P->d[i]};
        double Rn[3][3], pn[3];
        for (int r = 0; r < 3; ++r) {
            for (int k = 0; k < 3; ++k) Rn[r][k] = R[r][0] * Ra[0][k] + R[r][1] * Ra[1][k] + R[r][2] * Ra[2][k];
            pn[r] = R[r][0] * pa[0] + R[r][1] * pa[1] + R[r][2] * pa[2] + p[r];
        }
        memcpy(R, Rn, sizeof(R));
        memcpy(p, pn, sizeof(p));
    }
    out6[0] = p[0];
    out6[1] = p[1];
    out6[2] = p[2];
    out6[3] = atan2(R[1][0], R[0][0]);
    out6[4] = atan2(-R[2][0], sqrt(R[2][1] * R[2][1] + R[2][2] * R[2][2]));
    out6[5] = atan2(R[2][1], R[2][2]);
}

pf_status pf_make_trace(pf_model_id model, const void* params, uint32_t seed, int32_t steps,
                        pf_step_input* inputs, float* truth)
{
    if (!params || steps < 0 || (steps > 0 && (!inputs || !truth))) return PF_ERR_INVALID;
    sm64_t r = {0x5452414345534544ULL ^ ((uint64_t)seed << 24) ^ (uint64_t)model};
    memset(inputs, 0, sizeof(pf_step_input) * (size_t)steps);
    if (model == PF_MODEL_UNICYCLE) {
        const pf_unicycle_params* P = (const pf_unicycle_params*)params;
        const int L = P->num_landmarks;
        if (L < 1 || L > 8) return PF_ERR_INVALID;
        double x = P->init_state[0], y = P->init_state[1], th = P->init_state[2];
        const double dt = P->dt;
        for (int k = 0; k < steps; ++k) {
            const double t = k * dt, v = 1.0, w = 0.3 * sin(0.05 * t);
            const double wd = w * dt;
            double A, B;
            if (fabs(wd) < 1e-4) {
                A = v * dt * (1.0 - wd * wd / 6.0);
                B = v * dt * (wd / 2.0);
            } else {
                A = v * sin(wd) / w;
                B = v * (1.0 - cos(wd)) / w;
            }
            const double c = cos(th), s = sin(th);
            x = x + A * c - B * s + P->sigma_q[0] * sm64_gauss(&r);
            y = y + A * s + B * c + P->sigma_q[1] * sm64_gauss(&r);
            th = wrap(th + wd + P->sigma_q[2] * sm64_gauss(&r));
            pf_step_input* in = &inputs[k];
            in->dt = (float)dt;
            in->control[0] = (float)v;
            in->control[1] = (float)w;
            for (int j = 0; j < L; ++j) {
                const double dx = P->landmarks[j][0] - x, dy = P->landmarks[j][1] - y;
                in->meas[j] = (float)(sqrt(dx * dx + dy * dy) + P->sigma_range * sm64_gauss(&r));
                in->meas[L + j] = (float)wrap(atan2(dy, dx) - th + P->sigma_bearing * sm64_gauss(&r));
            }
            truth[3 * k + 0] = (float)x;
            truth[3 * k + 1] = (float)y;
            truth[3 * k + 2] = (float)th;
        }
        return PF_OK;
    }
    if (model == PF_MODEL_DHARM) {
        const pf_dharm_params* P = (const pf_dharm_params*)params;
        double q[6], qd[6], z[6];
        for (int i = 0; i < 6; ++i) {
            q[i] = P->init_state[i];
            qd[i] = P->init_state[6 + i];
        }
        for (int k = 0; k < steps; ++k) {
            for (int i = 0; i < 6; ++i) {
                q[i] = wrap(q[i] + qd[i] * P->dt);
                qd[i] = qd[i] + P->sigma_qd * sm64_gauss(&r);
            }
            dh_fk(P, q, z);
            pf_step_input* in = &inputs[k];
            in->dt = P->dt;
            for (int i = 0; i < 3; ++i) in->meas[i] = (float)(z[i] + P->sigma_pos * sm64_gauss(&r));
            for (int i = 3; i < 6; ++i) in->meas[i] = (float)wrap(z[i] + P->sigma_ang * sm64_gauss(&r));
            for (int i = 0; i < 6; ++i) {
                truth[12 * k + i] = (float)q[i];
                truth[12 * k + 6 + i] = (float)qd[i];
            }
        }
        return PF_OK;
    }
    if (model == PF_MODEL_BEACON) {
        /* The reference's unicycle trace generator (generate_input.py:37-56):
         * v = |N(0.3, 0.1)|, omega = N(0, 0.3), an exact arc of length v dt,
         * ranges to the beacons with N(0, sigma_range) noise (the generator's
         * sigma is 1; here the filter's own sigma is used). */
        const pf_beacon_params* P = (const pf_beacon_params*)params;
        const int L = P->num_beacons;
        if (L < 1 || L > 16) return PF_ERR_INVALID;
        double x = P->init_state[0], y = P->init_state[1], th = P->init_state[2];
        const double dt = P->dt;
        for (int k = 0; k < steps; ++k) {
            const double v = fabs(0.3 + 0.1 * sm64_gauss(&r)), w = 0.3 * sm64_gauss(&r);
            const double h = 0.5 * w * dt;
            const double sc = fabs(h) < 1e-8 ? 1.0 : sin(h) / h;
            x += v * dt * sc * cos(th + h);
            y += v * dt * sc * sin(th + h);
            th = wrap(th + w * dt);
            pf_step_input* in = &inputs[k];
            in->dt = (float)dt;
            in->control[0] = (float)v;
            in->control[1] = (float)w;
            for (int j = 0; j < L; ++j) {
                const double dx = x - P->beacons[j][0], dy = y - P->beacons[j][1], dz = P->beacons[j][2];
                in->meas[j] = (float)(sqrt(dx * dx + dy * dy + dz * dz) + P->sigma_range * sm64_gauss(&r));
            }
            truth[3 * k + 0] = (float)x;
            truth[3 * k + 1] = (float)y;
            truth[3 * k + 2] = (float)th;
        }
        return PF_OK;
    }
    return PF_ERR_UNSUPPORTED;
}
