/*
 * pf_oracle.c -- CPU restatement of the Esthera distributed particle-filter
 * step.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path and
 * the timed CPU baseline.  The product never links or calls this file.
 *
 * Citations are to the Esthera source tree (paths relative to its root).
 * Compiled with -ffp-contract=off so FP32/FP64 additions happen exactly in
 * the order written (the sort, scan and alias restatements must be
 * bit-identical to the device code given identical inputs).
 */
#include "pf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The MTGP32-11213 parameter sets, 52 words per set (see
 * esthera_b200/csrc/gen_mtgp_params.py for the layout). */
static const uint32_t MTGP_PARAMS[ORC_MTGP_SETS * 52] = {
#include "../esthera_b200/csrc/mtgp32_params_11213.inc"
};

#define P_POS(s) (MTGP_PARAMS[(s) * 52 + 0])
#define P_SH1(s) (MTGP_PARAMS[(s) * 52 + 1])
#define P_SH2(s) (MTGP_PARAMS[(s) * 52 + 2])
#define P_MASK(s) (MTGP_PARAMS[(s) * 52 + 3])
#define P_TBL(s) (&MTGP_PARAMS[(s) * 52 + 4])
#define P_TMP(s) (&MTGP_PARAMS[(s) * 52 + 20])
#define P_FLT(s) (&MTGP_PARAMS[(s) * 52 + 36])

/* mtgp32_init_state, mtgp32-fast.c:119-137 */
void orc_mtgp_init_state(uint32_t* st, int set, uint32_t seed)
{
    const uint32_t* tbl = P_TBL(set);
    uint32_t hidden = tbl[4] ^ (tbl[8] << 16);
    uint32_t tmp = hidden;
    tmp += tmp >> 16;
    tmp += tmp >> 8;
    uint32_t b = tmp & 0xffu;
    uint32_t fill = b | (b << 8) | (b << 16) | (b << 24);
    for (int i = 0; i < ORC_MTGP_N; ++i) st[i] = fill;
    st[0] = seed;
    st[1] = hidden;
    for (int i = 1; i < ORC_MTGP_N; ++i)
        st[i] ^= UINT32_C(1812433253) * (st[i - 1] ^ (st[i - 1] >> 30)) + (uint32_t)i;
}

/* Output k of a stream whose state words are x_0..x_350:
 *   x_{k+351} = rec(x_k, x_{k+1}, x_{k+pos})        (mtgp32_do_recursion, mtgp32-fast.h:145-155)
 *   out_k     = temper(x_{k+351}, x_{k+pos-1})      (mtgp32_temper[_float], mtgp32-fast.h:188-214) */
void orc_mtgp_generate(uint32_t* st, int set, uint32_t mask, int kind, int64_t n, uint32_t* out)
{
    uint32_t ring[1024];
    const uint32_t pos = P_POS(set), sh1 = P_SH1(set), sh2 = P_SH2(set);
    const uint32_t* tbl = P_TBL(set);
    const uint32_t* ttb = kind ? P_FLT(set) : P_TMP(set);
    if (mask == 0) mask = P_MASK(set);
    for (int i = 0; i < ORC_MTGP_N; ++i) ring[i] = st[i];
    for (int64_t k = 0; k < n; ++k) {
        uint32_t x1 = ring[k & 1023], x2 = ring[(k + 1) & 1023], y = ring[(k + pos) & 1023];
        uint32_t x = (x1 & mask) ^ x2;
        x ^= x << sh1;
        y = x ^ (y >> sh2);
        uint32_t r = y ^ tbl[y & 0x0f];
        ring[(k + ORC_MTGP_N) & 1023] = r;
        uint32_t t = ring[(k + pos - 1) & 1023];
        t ^= t >> 16;
        t ^= t >> 8;
        out[k] = kind ? ((r >> 9) ^ ttb[t & 0x0f]) : (r ^ ttb[t & 0x0f]);
    }
    for (int i = 0; i < ORC_MTGP_N; ++i) st[i] = ring[(n + i) & 1023];
}

void orc_mtgp_generate_blocks(uint32_t* states, int G, uint32_t mask, int kind,
                              int64_t total, uint32_t* out)
{
    int64_t size = total / G;
    for (int g = 0; g < G; ++g)
        orc_mtgp_generate(states + (int64_t)g * ORC_MTGP_N, g % ORC_MTGP_SETS, mask, kind, size,
                          out + (int64_t)g * size);
}

/* boxmuller, pf_generic_soa.cu:481-500 */
void orc_boxmuller(float* data, int64_t n)
{
    for (int64_t i = 0; 2 * i < n; ++i) {
        double u1 = 2.0 - (double)data[2 * i];
        double u2 = 2.0 - (double)data[2 * i + 1];
        double r = sqrt(-2.0 * log(u1));
        double phi = 2.0 * M_PI * u2;
        data[2 * i] = (float)(r * cos(phi));
        data[2 * i + 1] = (float)(r * sin(phi));
    }
}

/* comparator + bitonic_sort, bitonic-sort.cu:11-61 (dir = 0: descending) */
static inline void cmpx(float* w, int32_t* ix, unsigned a, unsigned b, unsigned dir)
{
    if ((unsigned)(w[a] > w[b]) == dir) {
        float tw = w[a]; w[a] = w[b]; w[b] = tw;
        int32_t ti = ix[a]; ix[a] = ix[b]; ix[b] = ti;
    }
}

void orc_bitonic_sort_desc(float* key, int32_t* idx, int m)
{
    const unsigned dir = 0, half = (unsigned)m / 2;
    for (unsigned size = 2; size < (unsigned)m; size <<= 1)
        for (unsigned stride = size / 2; stride > 0; stride >>= 1)
            for (unsigned q = 0; q < half; ++q) {
                unsigned ddd = dir ^ ((q & (size / 2)) != 0);
                unsigned pos = 2 * q - (q & (stride - 1));
                cmpx(key, idx, pos, pos + stride, ddd);
            }
    for (unsigned stride = (unsigned)m / 2; stride > 0; stride >>= 1)
        for (unsigned q = 0; q < half; ++q) {
            unsigned pos = 2 * q - (q & (stride - 1));
            cmpx(key, idx, pos, pos + stride, dir);
        }
}

/* prefix_sum, pf_generic_soa.cu:169-216 */
float orc_blelloch_scan(float* e, int m)
{
    int offset = 1;
    for (int d = m / 2; d > 0; d /= 2) {
        for (int tid = 0; tid < d; ++tid) {
            int ai = offset * (2 * tid + 1) - 1, bi = offset * (2 * tid + 2) - 1;
            e[bi] += e[ai];
        }
        offset *= 2;
    }
    float cum = e[m - 1];
    e[m - 1] = 0;
    for (int d = 1; d < m; d *= 2) {
        offset /= 2;
        for (int tid = 0; tid < d; ++tid) {
            int ai = offset * (2 * tid + 1) - 1, bi = offset * (2 * tid + 2) - 1;
            float t = e[ai];
            e[ai] = e[bi];
            e[bi] += t;
        }
    }
    return cum;
}

/* binary_search, pf_generic_soa.cu:221-240 */
int orc_binary_search(const float* hay, float needle, int size)
{
    int lo = 0, hi = size - 1;
    do {
        int cur = lo + (hi - lo + 1) / 2;
        if (hay[cur] > needle) hi = cur - 1;
        else lo = cur;
    } while (lo < hi);
    return lo;
}

/* resampling, pf_generic_soa.cu:415-453 (MTGP uniforms in [1,2)) */
void orc_resample_ref(const float* w, const float* u, int m, int32_t* sel)
{
    float e[1024];
    memcpy(e, w, sizeof(float) * (size_t)m);
    float cum = orc_blelloch_scan(e, m);
    for (int i = 0; i < m; ++i) {
        float s = (u[i] - 1.0f) * cum;
        sel[i] = orc_binary_search(e, s, m);
    }
}

double orc_scan_f64(const float* w, int m, int ept, double* cum)
{
    int nt = m / ept;
    double tt[1024], inc[1024], ex[1024];
    for (int j = 0; j < nt; ++j) {
        double s = (double)w[j * ept];
        for (int e = 1; e < ept; ++e) s = s + (double)w[j * ept + e];
        tt[j] = s;
    }
    /* Kogge-Stone inside each 32-lane warp */
    for (int j = 0; j < nt; ++j) inc[j] = tt[j];
    for (int d = 1; d < 32; d <<= 1) {
        double nv[1024];
        for (int j = 0; j < nt; ++j) {
            int lane = j & 31;
            nv[j] = (lane >= d) ? inc[j] + inc[j - d] : inc[j];
        }
        memcpy(inc, nv, sizeof(double) * (size_t)nt);
    }
    for (int j = 0; j < nt; ++j) ex[j] = ((j & 31) == 0) ? 0.0 : inc[j - 1];
    /* Kogge-Stone across warp totals */
    int nw = (nt + 31) / 32;
    double wt[32], wi[32];
    for (int w2 = 0; w2 < nw; ++w2) {
        int last = w2 * 32 + 31;
        if (last > nt - 1) last = nt - 1;
        wt[w2] = inc[last];
    }
    for (int w2 = 0; w2 < nw; ++w2) wi[w2] = wt[w2];
    for (int d = 1; d < 32; d <<= 1) {
        double nv[32];
        for (int w2 = 0; w2 < nw; ++w2) nv[w2] = (w2 >= d) ? wi[w2] + wi[w2 - d] : wi[w2];
        memcpy(wi, nv, sizeof(double) * (size_t)nw);
    }
    for (int j = 0; j < nt; ++j) {
        int w2 = j >> 5;
        double base = (w2 == 0 ? 0.0 : wi[w2 - 1]) + ex[j];
        double c = base + (double)w[j * ept];
        cum[j * ept] = c;
        for (int e = 1; e < ept; ++e) {
            c = c + (double)w[j * ept + e];
            cum[j * ept + e] = c;
        }
    }
    return cum[m - 1];
}

double orc_resample_systematic(const float* w, int m, int ept, float u0, int32_t* sel)
{
    double cum[1024];
    double total = orc_scan_f64(w, m, ept, cum);
    double step = total / (double)m;
    for (int i = 0; i < m; ++i) {
        double p = ((double)u0 + (double)i) * step;
        int lo = 0, hi = m;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (cum[mid] <= p) lo = mid + 1;
            else hi = mid;
        }
        sel[i] = lo < m ? lo : m - 1;
    }
    return total;
}

/* sum_reduce4, resampling-valias.cl:85-104 */
static float sum_reduce4(float* arr, int m)
{
    int offset = m;
    while (offset > 2) {
        offset >>= 2;
        for (int l = 0; l < offset; ++l) {
            float x = arr[l + offset] + arr[l + offset + offset] + arr[l + offset + offset + offset];
            arr[l] = arr[l] + x;
        }
    }
    if (offset > 1) arr[0] = arr[0] + arr[1];
    return arr[0];
}

/* resampling_valias normalisation (:262-270) and vose_alias_init's scaling by
 * m (:117): the alias build's starting probabilities */
void orc_vose_scaled(const float* w, int m, float* scaled)
{
    float scratch[1024];
    memcpy(scratch, w, sizeof(float) * (size_t)m);
    float sum = sum_reduce4(scratch, m);
    for (int i = 0; i < m; ++i) {
        float p = w[i];
        if (sum > 0.0f) p = p / sum;
        else p = 1.0f / (float)m;
        scaled[i] = p * (float)m;
    }
}

/* resampling_valias normalisation (:262-270) + vose_alias_init (:111-195) */
void orc_vose_build(const float* w, int m, float* prob, uint32_t* alias)
{
    float scratch[1024];
    uint32_t sl[1024];
    memcpy(scratch, w, sizeof(float) * (size_t)m);
    float sum = sum_reduce4(scratch, m);
    for (int i = 0; i < m; ++i) {
        float p = w[i];
        if (sum > 0.0f) p = p / sum;
        else p = 1.0f / (float)m;
        prob[i] = p * (float)m;
        alias[i] = (uint32_t)i;
    }
    unsigned small_end = 0, large_rend = (unsigned)m - 1;
    for (int i = 0; i < m; ++i) {
        if (prob[i] <= 1.0f) sl[small_end++] = (uint32_t)i;
        else sl[large_rend--] = (uint32_t)i;
    }
    unsigned small_begin = 0;
    for (;;) {
        unsigned se = small_end;
        unsigned a = se - small_begin, b = (unsigned)m - se;
        unsigned nactive = a < b ? a : b;
        if (nactive == 0) break;
        large_rend += nactive;
        uint32_t sidx[1024], lidx[1024];
        float ps[1024], pl[1024];
        for (unsigned k = 0; k < nactive; ++k) {
            sidx[k] = sl[small_begin + k];
            lidx[k] = sl[se + k];
            ps[k] = prob[sidx[k]];
            alias[sidx[k]] = lidx[k];
            pl[k] = prob[lidx[k]];
        }
        for (unsigned k = 0; k < nactive; ++k) {
            float nl = (pl[k] + ps[k]) - 1.0f;
            unsigned old;
            if (nl <= 1.0f) old = small_end++;
            else old = large_rend--;
            sl[old] = lidx[k];
            prob[lidx[k]] = nl;
        }
        small_begin += nactive;
    }
}

uint32_t orc_vose_draw(const float* prob, const uint32_t* alias, int m, float ux, float uy)
{
    uint32_t col = (uint32_t)floorf(ux * (float)m);
    if (col >= (uint32_t)m) col = (uint32_t)m - 1;
    return (uy < prob[col]) ? col : alias[col];
}

void orc_torus_dims(int N, int* dx, int* dy)
{
    int x = 1;
    while ((int64_t)(2 * x) * (2 * x) <= N) x *= 2;
    *dx = x;
    *dy = N / x;
}

typedef struct { float k; int32_t g; int32_t ord; } cand_t;
static int cand_cmp(const void* a, const void* b)
{
    const cand_t* x = (const cand_t*)a;
    const cand_t* y = (const cand_t*)b;
    if (x->k > y->k) return -1;
    if (x->k < y->k) return 1;
    return x->ord - y->ord;
}

void orc_exchange_sources(int mode, int N, int m, int t, const float* top_keys, int32_t* src)
{
    for (int64_t i = 0; i < (int64_t)N * m; ++i) src[i] = (int32_t)i;
    if (mode == ORC_EXCH_NONE || t <= 0) return;
    if (mode == ORC_EXCH_RING) {
        for (int b = 0; b < N; ++b) {
            int from = (b - 1 + N) % N;
            for (int j = 0; j < t; ++j) src[b * m + m - 1 - j] = from * m + j;
        }
    } else if (mode == ORC_EXCH_TORUS) {
        int dx, dy;
        orc_torus_dims(N, &dx, &dy);
        for (int b = 0; b < N; ++b) {
            int x = b % dx, y = b / dx;
            int right = y * dx + (x + 1) % dx;
            int left = y * dx + (x - 1 + dx) % dx;
            int bottom = ((y + 1) % dy) * dx + x;
            int top = ((y - 1 + dy) % dy) * dx + x;
            int from[4] = {right, left, bottom, top};
            for (int k = 0; k < 4; ++k)
                for (int j = 0; j < t; ++j) src[b * m + m - 1 - j - k * t] = from[k] * m + j;
        }
    } else if (mode == ORC_EXCH_ALL2ALL) {
        int nc = N * t;
        cand_t* c = (cand_t*)malloc(sizeof(cand_t) * (size_t)nc);
        for (int b = 0; b < N; ++b)
            for (int j = 0; j < t; ++j) {
                c[b * t + j].k = top_keys[b * t + j];
                c[b * t + j].g = b * m + j;
                c[b * t + j].ord = b * t + j;
            }
        qsort(c, (size_t)nc, sizeof(cand_t), cand_cmp);
        for (int b = 0; b < N; ++b)
            for (int j = 0; j < t; ++j) src[b * m + m - 1 - j] = c[j].g;
        free(c);
    }
}

/* ---------------- models ---------------- */
static double wrap_pi(double a)
{
    return a - 2.0 * M_PI * floor((a + M_PI) / (2.0 * M_PI));
}

/* Unicycle with range/bearing landmarks.  Motion: exact arc of the velocity
 * model (structure of sampling, src/models/unicycle/particle_filter.cu:314-334,
 * rewritten without the division by omega), plus additive Gaussian process
 * noise; likelihood: Gaussian range and wrapped-bearing errors (log domain). */
static double unicycle_step(const orc_model* md, float* s, const float* n, const float* c,
                            const float* z)
{
    double v = c[0], w = c[1], dt = md->dt;
    double wd = w * dt, A, B;
    if (fabs(wd) < 1e-4) {
        A = v * dt * (1.0 - wd * wd / 6.0);
        B = v * dt * (wd / 2.0);
    } else {
        A = v * sin(wd) / w;
        B = v * (1.0 - cos(wd)) / w;
    }
    double x = s[0], y = s[1], th = s[2];
    double ct = cos(th), st = sin(th);
    double nx = x + A * ct - B * st + md->sq[0] * n[0];
    double ny = y + A * st + B * ct + md->sq[1] * n[1];
    double nt = wrap_pi(th + wd + md->sq[2] * n[2]);
    s[0] = (float)nx;
    s[1] = (float)ny;
    s[2] = (float)nt;
    x = s[0]; y = s[1]; th = s[2];
    double acc = 0.0;
    int L = md->num_landmarks;
    for (int j = 0; j < L; ++j) {
        double dx = md->lm[j][0] - x, dy = md->lm[j][1] - y;
        double r = sqrt(dx * dx + dy * dy);
        double er = (z[j] - r) / md->sigma_r;
        double ph = th + z[L + j];
        double eb = atan2(sin(ph) * dx - cos(ph) * dy, cos(ph) * dx + sin(ph) * dy) / md->sigma_b;
        acc += er * er + eb * eb;
    }
    return -0.5 * acc;
}

/* 6-joint serial arm, standard Denavit-Hartenberg chain, constant-velocity
 * joints.  Measurement: end-effector position + ZYX yaw/pitch/roll. */
static double dharm_step(const orc_model* md, float* s, const float* n, const float* c,
                         const float* z)
{
    (void)c;
    double q[6];
    for (int i = 0; i < 6; ++i) {
        double qi = wrap_pi((double)s[i] + (double)s[6 + i] * md->dt);
        s[i] = (float)qi;
        s[6 + i] = (float)((double)s[6 + i] + md->sigma_qd * n[i]);
        q[i] = s[i];
    }
    double R[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, p[3] = {0, 0, 0};
    for (int i = 0; i < 6; ++i) {
        double ct = cos(q[i]), st = sin(q[i]);
        double ca = cos(md->alpha[i]), sa = sin(md->alpha[i]);
        double Ra[3][3] = {{ct, -st * ca, st * sa}, {st, ct * ca, -ct * sa}, {0, sa, ca}};
        double pa[3] = {md->a[i] * ct, md->a[i] * st, md->d[i]};
        double Rn[3][3], pn[3];
        for (int r = 0; r < 3; ++r) {
            for (int k = 0; k < 3; ++k)
                Rn[r][k] = R[r][0] * Ra[0][k] + R[r][1] * Ra[1][k] + R[r][2] * Ra[2][k];
            pn[r] = R[r][0] * pa[0] + R[r][1] * pa[1] + R[r][2] * pa[2] + p[r];
        }
        memcpy(R, Rn, sizeof(R));
        memcpy(p, pn, sizeof(p));
    }
    double yaw = atan2(R[1][0], R[0][0]);
    double pitch = atan2(-R[2][0], sqrt(R[2][1] * R[2][1] + R[2][2] * R[2][2]));
    double roll = atan2(R[2][1], R[2][2]);
    double ang[3] = {yaw, pitch, roll};
    double acc = 0.0;
    for (int k = 0; k < 3; ++k) {
        double e = (z[k] - p[k]) / md->sigma_p;
        acc += e * e;
    }
    for (int k = 0; k < 3; ++k) {
        double d = z[3 + k] - ang[k];
        double e = atan2(sin(d), cos(d)) / md->sigma_a;
        acc += e * e;
    }
    return -0.5 * acc;
}

/* The reference's robot-arm model (sampling_iw, src/models/robotarm/cuda/
 * pf_model_soa.cuh:114-184): 5 joint angles + cart (x, y, vX, vY), planar
 * camera chain, likelihood exp(-sum 0.1 e^2).  Returns log of that weight. */
/* The arm chain shared by the reference's arm and its pinhole-camera variant:
 * propagates the particle in place, returns the angle part of the error
 * value and the cart's camera coordinates in cam[3]. */
static double arm_chain(const orc_model* md, float* s, const float* n, const float* c, const float* z,
                        double* cam)
{
    const double dt = md->dt;
    const double arm[5] = {0, 3, 3, 3, 3};
    double vx = s[7], vy = s[8];
    double x = (double)s[5] + vx * dt + (double)n[5] * 0.2;
    double y = (double)s[6] + vy * dt + (double)n[6] * 0.2;
    s[5] = (float)x;
    s[6] = (float)y;
    s[7] = (float)(vx + (double)n[7] * 2.0);
    s[8] = (float)(vy + (double)n[8] * 2.0);
    x = s[5]; y = s[6];
    double value = 0.0, cx = 0, cy = 0, cz = 0;
    for (int i = 0; i < 5; ++i) {
        double a = (double)s[i] + (double)c[i] * dt + (double)n[i] * 0.2;
        s[i] = (float)a;
        a = s[i];
        double sf = sin(a), cf = cos(a);
        if (i == 0) {
            cx = x * cf + y * sf;
            cy = -x * sf + y * cf;
            cz = 0;
        } else {
            double nb = cy * cf - cz * sf, nc = cy * sf + cz * cf;
            cy = nb;
            cz = nc - arm[i];
        }
        double e = a - z[i];
        value += e * e * 0.1;
    }
    cam[0] = cx;
    cam[1] = cy;
    cam[2] = cz;
    return value;
}

/* The reference's pinhole-camera arm (sampling_iw, src/models/robotarm/cuda/
 * pf_model_soa_packed_code.cuh:61-145): the arm chain, the cart's camera
 * coordinates projected (x/z, y/z), distorted (radial kc1, kc2; tangential
 * kc3, kc4) and mapped to pixels; log of the weight exp(-sum 0.1 e^2). */
static double camarm_step(const orc_model* md, float* s, const float* n, const float* c,
                          const float* z)
{
    double cam[3];
    double value = arm_chain(md, s, n, c, z, cam);
    const double xn = cam[0] / cam[2], yn = cam[1] / cam[2];
    const double r2 = xn * xn + yn * yn;
    const double rad = 1.0 + md->kc[0] * r2 + md->kc[1] * r2 * r2;
    const double xd = rad * xn + 2.0 * md->kc[2] * xn * yn + md->kc[3] * (3.0 * xn * xn + yn * yn);
    const double yd = rad * yn + md->kc[2] * (3.0 * yn * yn + xn * xn) + 2.0 * md->kc[3] * xn * yn;
    const double xp = md->fc[0] * xd + md->cc[0], yp = md->fc[1] * yd + md->cc[1];
    value += (xp - z[5]) * (xp - z[5]) * 0.1;
    value += (yp - z[6]) * (yp - z[6]) * 0.1;
    return -value;
}

static double refarm_step(const orc_model* md, float* s, const float* n, const float* c,
                          const float* z)
{
    double cam[3];
    double value = arm_chain(md, s, n, c, z, cam);
    value += (cam[0] - z[5]) * (cam[0] - z[5]) * 0.1;
    value += (cam[1] - z[6]) * (cam[1] - z[6]) * 0.1;
    return -value;
}

/* The reference's unicycle program (src/models/unicycle/particle_filter.cu:
 * 314-359) in its own difference form: v and omega with additive noise,
 * x += v/omega (sin(th + omega dt) - sin th), y -= v/omega (cos(th + omega dt)
 * - cos th), th += (omega + gamma) dt (wrapped to [-pi, pi) as the engine
 * does), log weight log(1e5) - (L/2) log(2 pi) - sum e^2 / (2 sigma^2) with e
 * the range error to each 3-D beacon (L/2 an integer division). */
static double beacon_step(const orc_model* md, float* s, const float* n, const float* c,
                          const float* z)
{
    const double dt = md->dt;
    const double v = (double)c[0] + md->bnoise[0] * n[0];
    const double w = (double)c[1] + md->bnoise[1] * n[1];
    const double g = md->bnoise[2] * n[2];
    const double th = s[2];
    double nx, ny;
    if (fabs(w * dt) < 1e-9) { /* the arc's straight-line limit */
        nx = s[0] + v * dt * cos(th);
        ny = s[1] + v * dt * sin(th);
    } else {
        nx = s[0] + v / w * (sin(th + w * dt) - sin(th));
        ny = s[1] - v / w * (cos(th + w * dt) - cos(th));
    }
    s[0] = (float)nx;
    s[1] = (float)ny;
    s[2] = (float)wrap_pi(th + w * dt + g * dt);
    const double x = s[0], y = s[1];
    const int L = md->num_beacons;
    double acc = 0.0;
    for (int j = 0; j < L; ++j) {
        const double dx = x - md->bc[j][0], dy = y - md->bc[j][1], dz = md->bc[j][2];
        const double e = sqrt(dx * dx + dy * dy + dz * dz) - z[j];
        acc += e * e;
    }
    return log(1e5) - (double)(L / 2) * log(2.0 * M_PI) - acc / (2.0 * md->sigma_r * md->sigma_r);
}

double orc_model_step(const orc_model* md, float* state, const float* noise, const float* control,
                      const float* meas)
{
    switch (md->model) {
    case ORC_MODEL_UNICYCLE: return unicycle_step(md, state, noise, control, meas);
    case ORC_MODEL_DHARM: return dharm_step(md, state, noise, control, meas);
    case ORC_MODEL_BEACON: return beacon_step(md, state, noise, control, meas);
    case ORC_MODEL_CAMARM: return camarm_step(md, state, noise, control, meas);
    default: return refarm_step(md, state, noise, control, meas);
    }
}

static int is_angle(const orc_model* md, int v)
{
    if (md->model == ORC_MODEL_UNICYCLE || md->model == ORC_MODEL_BEACON) return v == 2;
    if (md->model == ORC_MODEL_DHARM) return v < 6;
    return v < 5;
}

/* ---------------- whole filter ---------------- */
/* exp(x) for max-subtracted log-weights x <= 0 from correctly rounded FP32
 * operations only: n = rint(x log2 e), r = x - n ln2 (Cody-Waite, two fmaf),
 * exp(x) = 2^n P(r) with the project's degree-6 fit of P (the engine's
 * pf_expneg evaluates the same operations in the same order, so both give the
 * same bits; esthera_b200/csrc/fit_exp.py fits and checks the polynomial).
 * x < -87 (and -inf) gives 0; NaN stays NaN. */
float orc_expneg(float x)
{
    const float n = rintf(x * 1.442695022e+00f);
    float r = fmaf(n, -0.693145751953125f, x);
    r = fmaf(n, -1.428606765e-06f, r);
    float p = 1.384175848e-03f;
    p = fmaf(p, r, 8.375782520e-03f);
    p = fmaf(p, r, 4.166811332e-02f);
    p = fmaf(p, r, 1.666641235e-01f);
    p = fmaf(p, r, 4.999999404e-01f);
    p = fmaf(p, r, 1.000000000e+00f);
    p = fmaf(p, r, 1.0f);
    if (x != x) return x;
    if (!(x >= -87.0f)) return 0.0f;
    const int ni = (int)n;
    if (ni < -126) return 0.0f;
    union {
        uint32_t u;
        float f;
    } sc;
    sc.u = (uint32_t)(ni + 127) << 23;
    return p * sc.f;
}

int64_t orc_stream_draws(int num_noise, int m, int resampler)
{
    int64_t nb = 2 * (((int64_t)num_noise * m + 1) / 2);
    int64_t ru = resampler == ORC_RES_REF ? m : (resampler == ORC_RES_VOSE ? 2 * m : 1);
    return nb + 1 + ru;
}

int orc_filter_init(orc_filter* f, const orc_model* mdl, int m, int N, int t, int exchange,
                    int resampler, int rng, int G, int ept, int log_weights, float freq,
                    uint32_t seed, uint32_t mask, const float* init_state)
{
    memset(f, 0, sizeof(*f));
    f->mdl = *mdl;
    f->m = m; f->N = N; f->t = t; f->exchange = exchange; f->resampler = resampler;
    f->rng = rng; f->G = G; f->ept = ept; f->log_weights = log_weights; f->freq = freq;
    f->seed = seed; f->mask = mask;
    f->T = (int64_t)m * N;
    int S = mdl->num_state;
    f->state = (float*)malloc(sizeof(float) * (size_t)(S * f->T));
    f->tmp = (float*)malloc(sizeof(float) * (size_t)(S * f->T));
    f->tkey = (float*)malloc(sizeof(float) * (size_t)f->T);
    for (int v = 0; v < S; ++v)
        for (int64_t i = 0; i < f->T; ++i) f->state[v * f->T + i] = init_state[v];
    f->streams = rng == ORC_RNG_REFLAYOUT ? G : N;
    f->mtgp = (uint32_t*)malloc(sizeof(uint32_t) * ORC_MTGP_N * (size_t)f->streams);
    for (int g = 0; g < f->streams; ++g)
        orc_mtgp_init_state(f->mtgp + (int64_t)g * ORC_MTGP_N, g % ORC_MTGP_SETS, seed + (uint32_t)g + 1u);
    if (rng == ORC_RNG_REFLAYOUT) {
        int64_t nn = (int64_t)mdl->num_noise * f->T;
        int64_t nu = resampler == ORC_RES_VOSE ? (int64_t)(2 * m + 1) * N : (int64_t)(m + 1) * N;
        int64_t unit = 768LL * G;
        f->rtotal = ((nn + nu + unit - 1) / unit) * unit;
    } else {
        f->rtotal = orc_stream_draws(mdl->num_noise, m, resampler) * N;
    }
    f->rbuf = (float*)malloc(sizeof(float) * (size_t)f->rtotal);
    return 0;
}

int orc_filter_set_stream_offset(orc_filter* f, int off)
{
    if (f->rng != ORC_RNG_SUBFILTER || off < 0) return -1;
    f->soff = off;
    for (int b = 0; b < f->N; ++b)
        orc_mtgp_init_state(f->mtgp + (int64_t)b * ORC_MTGP_N, (off + b) % ORC_MTGP_SETS,
                            f->seed + (uint32_t)(off + b) + 1u);
    return 0;
}

void orc_filter_free(orc_filter* f)
{
    free(f->state); free(f->tmp); free(f->tkey); free(f->mtgp); free(f->rbuf);
    memset(f, 0, sizeof(*f));
}

int orc_filter_step(orc_filter* f, const float* control, const float* meas, orc_estimate* est,
                    int32_t* sel_out, int threads)
{
    int r = orc_filter_sample(f, control, meas, est, threads);
    return r ? r : orc_filter_resample(f, sel_out, threads);
}

int orc_filter_sample(orc_filter* f, const float* control, const float* meas, orc_estimate* est, int threads)
{
    const int m = f->m, N = f->N, S = f->mdl.num_state, K = f->mdl.num_noise;
    const int64_t T = f->T;
    const int64_t draws = orc_stream_draws(K, m, f->resampler);
    const int64_t nb = 2 * (((int64_t)K * m + 1) / 2);
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
    /* 1. random numbers */
    if (f->rng == ORC_RNG_REFLAYOUT) {
        int64_t size = f->rtotal / f->G;
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int g = 0; g < f->G; ++g)
            orc_mtgp_generate(f->mtgp + (int64_t)g * ORC_MTGP_N, g % ORC_MTGP_SETS, f->mask, 1, size,
                              (uint32_t*)f->rbuf + (int64_t)g * size);
        orc_boxmuller(f->rbuf, (int64_t)K * T);
    } else {
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int b = 0; b < N; ++b) {
            float* buf = f->rbuf + (int64_t)b * draws;
            orc_mtgp_generate(f->mtgp + (int64_t)b * ORC_MTGP_N, (f->soff + b) % ORC_MTGP_SETS, f->mask, 1, draws,
                              (uint32_t*)buf);
            orc_boxmuller(buf, nb);
        }
    }
    /* 2. propagate + weight, sort, per-sub-filter partial estimates */
    double* part = (double*)calloc((size_t)N * 40, sizeof(double));
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int b = 0; b < N; ++b) {
        float key[1024];
        int32_t ix[1024];
        float st[16], nz[16];
        for (int i = 0; i < m; ++i) {
            int64_t idx = (int64_t)b * m + i;
            for (int v = 0; v < S; ++v) st[v] = f->state[v * T + idx];
            for (int v = 0; v < K; ++v)
                nz[v] = f->rng == ORC_RNG_REFLAYOUT ? f->rbuf[v * T + idx]
                                                    : f->rbuf[(int64_t)b * draws + (int64_t)v * m + i];
            double ll = orc_model_step(&f->mdl, st, nz, control, meas);
            for (int v = 0; v < S; ++v) f->state[v * T + idx] = st[v];
            key[i] = f->log_weights ? (float)ll : (float)exp(ll);
            ix[i] = i;
        }
        orc_bitonic_sort_desc(key, ix, m);
        for (int p = 0; p < m; ++p) {
            int64_t d = (int64_t)b * m + p;
            f->tkey[d] = key[p];
            for (int v = 0; v < S; ++v) f->tmp[v * T + d] = f->state[v * T + (int64_t)b * m + ix[p]];
        }
        double lmax = f->log_weights ? (double)key[0] : 0.0;
        double* pp = part + (size_t)b * 40;
        pp[0] = lmax;
        for (int p = 0; p < m; ++p) {
            double w = f->log_weights ? exp((double)key[p] - lmax) : (double)key[p];
            pp[1] += w;
            for (int v = 0; v < S; ++v) {
                double xv = f->tmp[v * T + (int64_t)b * m + p];
                if (is_angle(&f->mdl, v)) {
                    pp[2 + v] += w * sin(xv);
                    pp[20 + v] += w * cos(xv);
                } else {
                    pp[2 + v] += w * xv;
                }
            }
        }
    }
    /* 3. winner (first max, thrust::max_element semantics) + estimate */
    if (est) {
        int best = 0;
        for (int b = 1; b < N; ++b)
            if (f->tkey[(int64_t)b * m] > f->tkey[(int64_t)best * m]) best = b;
        est->best_sub = best;
        est->best_key = f->tkey[(int64_t)best * m];
        for (int v = 0; v < S; ++v) est->best[v] = f->tmp[v * T + (int64_t)best * m];
        double gmax = -INFINITY;
        for (int b = 0; b < N; ++b)
            if (part[b * 40] > gmax) gmax = part[b * 40];
        double Ssum = 0, acc[16] = {0}, acc2[16] = {0};
        for (int b = 0; b < N; ++b) {
            double sc = f->log_weights ? exp(part[b * 40] - gmax) : 1.0;
            Ssum += sc * part[b * 40 + 1];
            for (int v = 0; v < S; ++v) {
                acc[v] += sc * part[b * 40 + 2 + v];
                acc2[v] += sc * part[b * 40 + 20 + v];
            }
        }
        for (int v = 0; v < S; ++v)
            est->mean[v] = is_angle(&f->mdl, v) ? atan2(acc[v], acc2[v]) : acc[v] / Ssum;
        est->log_norm = (f->log_weights ? gmax : 0.0) + log(Ssum);
    }
    free(part);
    return 0;
}

int orc_filter_resample(orc_filter* f, int32_t* sel_out, int threads)
{
    const int m = f->m, N = f->N, S = f->mdl.num_state, K = f->mdl.num_noise;
    const int64_t T = f->T;
    const int64_t draws = orc_stream_draws(K, m, f->resampler);
    const int64_t nb = 2 * (((int64_t)K * m + 1) / 2);
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
    /* 4. exchange routing */
    int32_t* src = (int32_t*)malloc(sizeof(int32_t) * (size_t)T);
    float* topk = NULL;
    if (f->exchange == ORC_EXCH_ALL2ALL && f->t > 0) {
        topk = (float*)malloc(sizeof(float) * (size_t)N * f->t);
        for (int b = 0; b < N; ++b)
            for (int j = 0; j < f->t; ++j) topk[b * f->t + j] = f->tkey[(int64_t)b * m + j];
    }
    orc_exchange_sources(f->exchange, N, m, f->t, topk, src);
    free(topk);
    /* 5. resampling */
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int b = 0; b < N; ++b) {
        float w[1024], uu[1024], prob[1024];
        uint32_t al[1024];
        int32_t sel[1024];
        const int64_t base = (int64_t)b * m;
        const float* U = f->rng == ORC_RNG_REFLAYOUT ? f->rbuf + (int64_t)K * T : NULL;
        const float* sb = f->rng == ORC_RNG_SUBFILTER ? f->rbuf + (int64_t)b * draws + nb : NULL;
        float dec = (U ? U[T + b] : sb[0]) - 1.0f;
        if (dec > f->freq) {
            if (sel_out)
                for (int i = 0; i < m; ++i) sel_out[base + i] = -1;
            continue;
        }
        float mx = -INFINITY;
        for (int s = 0; s < m; ++s) {
            w[s] = f->tkey[src[base + s]];
            if (w[s] > mx) mx = w[s];
        }
        if (f->log_weights)
            for (int s = 0; s < m; ++s) w[s] = orc_expneg(w[s] - mx);
        if (f->ess_frac > 0.0f) {
            /* effective sample size in FP64; all-zero weights count as uniform */
            double s1 = 0.0, s2 = 0.0;
            for (int s = 0; s < m; ++s) {
                s1 += (double)w[s];
                s2 += (double)w[s] * (double)w[s];
            }
            if (!(s2 > 0.0) || s1 * s1 >= (double)f->ess_frac * (double)m * s2) {
                if (sel_out)
                    for (int i = 0; i < m; ++i) sel_out[base + i] = -1;
                continue;
            }
        }
        if (f->resampler == ORC_RES_REF) {
            for (int i = 0; i < m; ++i) uu[i] = U ? U[base + i] : sb[1 + i];
            orc_resample_ref(w, uu, m, sel);
        } else if (f->resampler == ORC_RES_SYSTEMATIC) {
            float u0 = (U ? U[base] : sb[1]) - 1.0f;
            orc_resample_systematic(w, m, f->ept, u0, sel);
        } else {
            orc_vose_build(w, m, prob, al);
            for (int i = 0; i < m; ++i) {
                float ux = (U ? U[2 * (base + i)] : sb[1 + 2 * i]) - 1.0f;
                float uy = (U ? U[2 * (base + i) + 1] : sb[2 + 2 * i]) - 1.0f;
                sel[i] = (int32_t)orc_vose_draw(prob, al, m, ux, uy);
            }
        }
        for (int i = 0; i < m; ++i) {
            int64_t from = src[base + sel[i]];
            for (int v = 0; v < S; ++v) f->state[v * T + base + i] = f->tmp[v * T + from];
            if (sel_out) sel_out[base + i] = sel[i];
        }
    }
    free(src);
    return 0;
}
