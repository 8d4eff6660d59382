// pf_step.cuh -- the single-kernel filter step: one warp per sub-filter.
//
// Step s of a filter is ONE launch.  Warp w owns sub-filter b and runs, with
// warp-level synchronisation only:
//   G  its MTGP32 stream -> this step's uniforms (normals via Box-Muller into
//      shared memory; the resampling draws go to global memory for step s+1)
//   R  the resampling of step s-1, deferred to here: the sorted particles of
//      step s-1 (and the neighbours' top-t for the exchange) are read from the
//      other half of the double-buffered sorted state, weighted, resampled
//      (systematic / reference multinomial / Vose) and gathered into shared
//      memory -- or, on the first step and for sub-filters that skipped
//      resampling, the propagated state is read from `state`
//   P  propagate + log-weight, E = m/32 particles per lane
//   S  bitonic sort of the m keys (E per lane: register and shuffle stages)
//   W  sorted keys and particles of step s -> this step's half of the buffer,
//      winner, FP64 estimate partials
//   E  the last warp of each group of 32 sub-filters combines the group, the
//      last group writes the estimate (fixed order, deterministic).
// The arithmetic of every phase is the one of the split/phased kernels
// (same device functions), so the pipelines agree; the particles a caller
// reads after step s are produced by k_resample_only (phase R alone).
#pragma once

#include "pf_kernels.cuh"

namespace pfdev {

// Extra per-filter state of the single-kernel pipeline.
struct StepState {
    float* tmp2;        // second half of the sorted-state double buffer (S*T)
    float* tkey2;       // second half of the sorted-key double buffer (T)
    int32_t* steps;     // persistent step count (buffer parity), never reset by runs
    int32_t* need_init; // 1: `state` holds the particles (first step / after set / restore)
    int32_t* grp_ctr;   // ceil(N/32) group tickets
};

constexpr int kWarpsPerCta = 2;  // sub-filters per CTA (one warp each)

// Shared-memory rows of one warp: lane r owns "row" r = slots E*r .. E*r+E-1.
// prow(i): position of slot i in an unpadded S x M state array whose float4
// chunks are XOR-swizzled per row, so that both float4 row accesses (8 lanes
// per phase) and the strided pattern i = lane + 32 e hit distinct banks.
template <int E>
__device__ __forceinline__ int prow(int i)
{
    if constexpr (E >= 8) {
        constexpr int RPB = 32 / E, NC = E / 4;
        const int r = i / E, c = i % E;
        const int sw = (r / RPB) & (NC - 1);
        return r * E + ((((c >> 2) ^ sw) << 2) | (c & 3));
    } else {
        return i;
    }
}
// First float of float4 chunk q of row r in the swizzled layout.
template <int E>
__device__ __forceinline__ int pchunk(int r, int q)
{
    if constexpr (E >= 8) {
        constexpr int RPB = 32 / E, NC = E / 4;
        return r * E + ((q ^ ((r / RPB) & (NC - 1))) << 2);
    } else {
        return r * E + 4 * q;
    }
}

template <int E>
struct LaneRows {
    static constexpr int F = E + 4;  // padded float rows of the key transpose
    static constexpr int D = E + 1;  // odd double stride: 16-lane 64-bit accesses hit distinct bank pairs
};

// MTGP32 state ring of 768 words (3 rounds of 256): x_j at ring[j mod 768].
struct MtgpRing {
    uint32_t ring[768];
    uint32_t tbl[16];
    uint32_t ttb[16];
    uint32_t pos, sh1, sh2, mask;
};

template <class Mdl, int M, int RES>
struct StepSmem {
    static constexpr int E = M / 32;
    static constexpr int S = Mdl::S, K = Mdl::K;
    static constexpr int NBM = 2 * ((K * M + 1) / 2);
    template <class A, class B>
    static constexpr size_t mx(A a, B b) { return (size_t)a > (size_t)b ? (size_t)a : (size_t)b; }
    static constexpr size_t r16(size_t x) { return (x + 15) / 16 * 16; }
    // A: MTGP ring (phase G) / padded key transpose (phases S, W)
    static constexpr size_t kA = r16(mx(sizeof(MtgpRing), (size_t)32 * LaneRows<E>::F * 4));
    // N: the resampler's arrays (phase R, before G) / normals (G, P)
    static constexpr size_t kRes = RES == PF_RESAMPLE_SYSTEMATIC ? (size_t)32 * LaneRows<E>::D * 8
                                 : (RES == PF_RESAMPLE_REFERENCE ? (size_t)M * 4 : (size_t)M * 12);
    static constexpr size_t kN = r16(mx((size_t)NBM * 4, kRes));
    // B: particle state, S x M swizzled rows
    static constexpr size_t kB = (size_t)S * M * 4;
    static constexpr size_t kConsts = r16(sizeof(typename Mdl::Consts));
    static constexpr size_t kPerWarp = kA + kN + kB + kConsts;
};

__device__ __forceinline__ int r768(int x) { return x >= 768 ? x - 768 : x; }

__device__ __forceinline__ void mtgp_load_ring(MtgpRing& s, const uint32_t* __restrict__ gstate, int set,
                                               uint32_t mask, int lane)
{
    for (int i = lane; i < kMtgpN; i += 32) s.ring[i] = gstate[i];
    const uint32_t* P = g_mtgp_params + set * 52;
    if (lane < 16) {
        s.tbl[lane] = P[4 + lane];
        s.ttb[lane] = P[36 + lane];
    }
    if (lane == 0) {
        s.pos = P[0];
        s.sh1 = P[1];
        s.sh2 = P[2];
        s.mask = mask ? mask : P[3];
    }
    __syncwarp();
}

// mtgp_generate for one warp on the 768-word ring: 8 lanes of the 256-wide
// round per thread; every ring index stays below 2*768 before the wrap.
template <class Emit>
__device__ __forceinline__ void mtgp_generate_ring(MtgpRing& s, int n, int lane, Emit emit)
{
    const int pos = (int)s.pos;
    const uint32_t sh1 = s.sh1, sh2 = s.sh2, mask = s.mask;
    int bm = 0;  // base mod 768
    for (int base = 0; base < n; base += kMtgpLanes) {
#pragma unroll
        for (int r = 0; r < kMtgpLanes / 32; ++r) {
            const int l = lane + 32 * r;
            const int j = bm + l;
            const uint32_t x1 = s.ring[r768(j)], x2 = s.ring[r768(j + 1)];
            uint32_t y = s.ring[r768(j + pos)];
            uint32_t t = s.ring[r768(j + pos - 1)];
            uint32_t x = (x1 & mask) ^ x2;
            x ^= x << sh1;
            y = x ^ (y >> sh2);
            const uint32_t rr = y ^ s.tbl[y & 0x0f];
            s.ring[r768(j + kMtgpN)] = rr;
            t ^= t >> 16;
            t ^= t >> 8;
            if (base + l < n) emit(base + l, (rr >> 9) ^ s.ttb[t & 0x0f]);
        }
        bm = bm == 512 ? 0 : bm + 256;
        __syncwarp();
    }
}

__device__ __forceinline__ void mtgp_store_ring(const MtgpRing& s, uint32_t* __restrict__ gstate, int n, int lane)
{
    for (int i = lane; i < kMtgpN; i += 32) gstate[i] = s.ring[(n + i) % 768];
}

// ---------------------------------------------------------------------------
// The reference's descending bitonic network (bitonic-sort.cu:28-61, dir = 0,
// equal keys swap) for one warp holding E consecutive keys per lane -- the same
// comparisons as bitonic_sort_desc, with the stage loops kept as runtime loops
// so the kernel stays small enough for the instruction cache; only the
// per-key work of one stage is unrolled.
// ---------------------------------------------------------------------------
template <int E>
__device__ __forceinline__ void cswap(float (&k)[E], int (&ix)[E], int a, int b, bool ddd)
{
    const float ka = k[a], kb = k[b];
    if ((ka > kb) == ddd) {
        k[a] = kb;
        k[b] = ka;
        const int t = ix[a];
        ix[a] = ix[b];
        ix[b] = t;
    }
}

// Strides E/2 .. 1 inside the lane with one direction for all pairs.
template <int E>
__device__ __forceinline__ void reg_merge(float (&k)[E], int (&ix)[E], bool ddd)
{
#pragma unroll
    for (int stride = E / 2; stride > 0; stride >>= 1)
#pragma unroll
        for (int e = 0; e < E; ++e)
            if ((e & stride) == 0) cswap<E>(k, ix, e, e + stride, ddd);
}

template <int M, int E>
__device__ __forceinline__ void bitonic_warp_desc(float (&k)[E], int (&ix)[E], int lane)
{
    // sizes 2 .. E/2: both keys of every pair in the lane, direction bit of e
#pragma unroll
    for (int size = 2; size < E; size <<= 1)
#pragma unroll
        for (int stride = size / 2; stride > 0; stride >>= 1)
#pragma unroll
            for (int e = 0; e < E; ++e)
                if ((e & stride) == 0) cswap<E>(k, ix, e, e + stride, (e & size) != 0);
    // size E: direction = bit log2(E) of E*lane + e = lane bit 0
    if constexpr (E > 1) reg_merge<E>(k, ix, (lane & 1) != 0);
    // sizes 2E .. M: shuffle stages for strides >= E, then the in-lane merge;
    // the direction (E*lane & size) is the same for all keys of the lane
#pragma unroll 1
    for (int size = 2 * E; size <= M; size <<= 1) {
        const bool ddd = ((E * lane) & size) != 0;
#pragma unroll 1
        for (int stride = size >> 1; stride >= E; stride >>= 1) {
            const int lm = stride / E;
            const bool upper = (lane & lm) != 0;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const float ok = __shfl_xor_sync(kFull, k[e], lm);
                const int oi = __shfl_xor_sync(kFull, ix[e], lm);
                const float lo = upper ? ok : k[e];
                const float hi = upper ? k[e] : ok;
                if ((lo > hi) == ddd) {
                    k[e] = ok;
                    ix[e] = oi;
                }
            }
        }
        if constexpr (E > 1) reg_merge<E>(k, ix, ddd);
    }
}

// ---------------------------------------------------------------------------
// Phase R: resample sub-filter b of step s-1 into the swizzled state rows B.
// src_* are the sorted arrays of step s-1; U the draws of step s-1 (decision
// first); W is the resampler's scratch (the normals region, idle before G).
// Output slot i = E*lane + e (E consecutive outputs per lane) receives its
// particle at prow(i); sel_out (optional) records the chosen slot.
// ---------------------------------------------------------------------------
template <int S, int M, int RES>
__device__ __forceinline__ void phase_resample(const FilterDesc& D, int b, const float* __restrict__ src_tmp,
                                               const float* __restrict__ src_key, const float* __restrict__ U,
                                               float* B, unsigned char* W, int lane, int32_t* sel_out)
{
    constexpr int E = M / 32;
    constexpr int RD = LaneRows<E>::D;
    const int64_t T = D.T;
    const int64_t base = (int64_t)b * M;
    float w[E];
#pragma unroll
    for (int q = 0; q < E; q += 4) {
        const float4 v = *reinterpret_cast<const float4*>(src_key + base + E * lane + q);
        w[q] = v.x;
        w[q + 1] = v.y;
        w[q + 2] = v.z;
        w[q + 3] = v.w;
    }
#pragma unroll
    for (int v = 0; v < S; ++v)
#pragma unroll
        for (int q = 0; q < E / 4; ++q)
            *reinterpret_cast<float4*>(B + v * M + pchunk<E>(lane, q)) =
                *reinterpret_cast<const float4*>(src_tmp + v * T + base + E * lane + 4 * q);
    // exchange: the last nx slots take the neighbours' top-t (read out of place)
    const int nx = exchange_count(D);
    __syncwarp();
    for (int x = lane; x < nx; x += 32) {
        const int64_t g = exchange_source(D, b, x);
        const int s = M - 1 - x;
#pragma unroll
        for (int v = 0; v < S; ++v) B[v * M + prow<E>(s)] = src_tmp[v * T + g];
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int x = M - 1 - (E * lane + e);
        if (x < nx) w[e] = src_key[exchange_source(D, b, x)];
    }
    __syncwarp();
    if (D.log_weights) {
        float mx = w[0];
#pragma unroll
        for (int e = 1; e < E; ++e) mx = fmaxf(mx, w[e]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
#pragma unroll
        for (int e = 0; e < E; ++e) w[e] = __expf(w[e] - mx);
    }
    int sel[E];
    if constexpr (RES == PF_RESAMPLE_SYSTEMATIC) {
        // canonical FP64 scan (groups of E per lane, Kogge-Stone over the 32 lanes)
        double* cum = reinterpret_cast<double*>(W);
        double tt = (double)w[0];
#pragma unroll
        for (int e = 1; e < E; ++e) tt = tt + (double)w[e];
        double inc = tt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double o = __shfl_up_sync(kFull, inc, d);
            if (lane >= d) inc = inc + o;
        }
        double ex = __shfl_up_sync(kFull, inc, 1);
        if (lane == 0) ex = 0.0;
        double c = (0.0 + ex) + (double)w[0];
        cum[lane * RD] = c;
#pragma unroll
        for (int e = 1; e < E; ++e) {
            c = c + (double)w[e];
            cum[lane * RD + e] = c;
        }
        const double total = __shfl_sync(kFull, c, 31);  // cum[M-1], as the oracle defines it
        __syncwarp();
        const float u0 = U[1] - 1.0f;
        const double step = total / (double)M;
        // outputs E*lane + e are consecutive: gallop from the previous answer, then bisect
        int a = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double pos = ((double)u0 + (double)(E * lane + e)) * step;
            int bnd = M, d = 1;
            while (true) {
                const int t = a + d - 1;
                if (t >= M) break;
                if (cum[(t / E) * RD + (t % E)] > pos) {
                    bnd = t;
                    break;
                }
                a = t + 1;
                d <<= 1;
            }
            while (a < bnd) {
                const int mid = (a + bnd) >> 1;
                if (cum[(mid / E) * RD + (mid % E)] <= pos) a = mid + 1;
                else bnd = mid;
            }
            sel[e] = a < M ? a : M - 1;
        }
    } else if constexpr (RES == PF_RESAMPLE_REFERENCE) {
        // FP32 Blelloch tree exactly as prefix_sum (pf_generic_soa.cu:169-216), then
        // binary_search per output
        float* ex = reinterpret_cast<float*>(W);
#pragma unroll
        for (int e = 0; e < E; ++e) ex[E * lane + e] = w[e];
        int offset = 1;
        for (int d = M / 2; d > 0; d /= 2) {
            __syncwarp();
            for (int q = lane; q < d; q += 32) {
                const int ai = offset * (2 * q + 1) - 1, bi = offset * (2 * q + 2) - 1;
                ex[bi] += ex[ai];
            }
            offset *= 2;
        }
        __syncwarp();
        const float tot = ex[M - 1];
        __syncwarp();
        if (lane == 0) ex[M - 1] = 0.0f;
        for (int d = 1; d < M; d *= 2) {
            offset /= 2;
            __syncwarp();
            for (int q = lane; q < d; q += 32) {
                const int ai = offset * (2 * q + 1) - 1, bi = offset * (2 * q + 2) - 1;
                const float t = ex[ai];
                ex[ai] = ex[bi];
                ex[bi] += t;
            }
        }
        __syncwarp();
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int i = E * lane + e;
            sel[e] = ref_binary_search(ex, (U[1 + i] - 1.0f) * tot, M);
        }
    } else {
        // Vose alias table (resampling-valias.cl:85-195), one warp, work lists in
        // ascending slot order
        float* prob = reinterpret_cast<float*>(W);
        unsigned* alias = reinterpret_cast<unsigned*>(prob + M);
        unsigned* sl = alias + M;
        float* scr = reinterpret_cast<float*>(sl);
#pragma unroll
        for (int e = 0; e < E; ++e) scr[E * lane + e] = w[e];
        int off = M;
        while (off > 2) {
            off >>= 2;
            __syncwarp();
            for (int l = lane; l < off; l += 32) {
                const float x = scr[l + off] + scr[l + off + off] + scr[l + off + off + off];
                scr[l] = scr[l] + x;
            }
        }
        __syncwarp();
        if (off > 1 && lane == 0) scr[0] = scr[0] + scr[1];
        __syncwarp();
        const float sum = scr[0];
        __syncwarp();
        int my_small = 0;
        bool fl[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int i = E * lane + e;
            float p = w[e];
            if (sum > 0.0f) p = p / sum;
            else p = 1.0f / (float)M;
            const float pr = p * (float)M;
            prob[i] = pr;
            alias[i] = (unsigned)i;
            fl[e] = pr <= 1.0f;
            my_small += fl[e] ? 1 : 0;
        }
        int incs = my_small;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(kFull, incs, d);
            if (lane >= d) incs += o;
        }
        const int nsmall = __shfl_sync(kFull, incs, 31);
        int s_i = incs - my_small, l_i = E * lane - (incs - my_small);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int i = E * lane + e;
            if (fl[e]) sl[s_i++] = (unsigned)i;
            else sl[M - 1 - (l_i++)] = (unsigned)i;
        }
        __syncwarp();
        unsigned small_end = (unsigned)nsmall, large_rend = small_end - 1u, small_begin = 0;
        for (int round = 0; round < M; ++round) {
            const unsigned se = small_end;
            const unsigned aa = se - small_begin, bb = (unsigned)M - se;
            const unsigned nactive = aa < bb ? aa : bb;
            if (nactive == 0) break;
            large_rend += nactive;
            constexpr int R = (M / 2 + 31) / 32;
            unsigned lidx[R];
            float pS[R], pL[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const unsigned kk = (unsigned)lane + 32u * r;
                if (kk < nactive) {
                    const unsigned sidx = sl[small_begin + kk];
                    lidx[r] = sl[se + kk];
                    pS[r] = prob[sidx];
                    alias[sidx] = lidx[r];
                    pL[r] = prob[lidx[r]];
                }
            }
            __syncwarp();
            unsigned s_base = 0, l_base = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const unsigned kk = (unsigned)lane + 32u * r;
                const bool act = kk < nactive;
                float nl = 0.0f;
                bool small = false;
                if (act) {
                    nl = (pL[r] + pS[r]) - 1.0f;
                    small = nl <= 1.0f;
                }
                const unsigned bs = __ballot_sync(kFull, act && small);
                const unsigned bl = __ballot_sync(kFull, act && !small);
                const unsigned below = (1u << lane) - 1u;
                if (act) {
                    const unsigned dst = small ? small_end + s_base + (unsigned)__popc(bs & below)
                                               : large_rend - l_base - (unsigned)__popc(bl & below);
                    sl[dst] = lidx[r];
                    prob[lidx[r]] = nl;
                }
                s_base += (unsigned)__popc(bs);
                l_base += (unsigned)__popc(bl);
            }
            small_end += s_base;
            large_rend -= l_base;
            small_begin += nactive;
            __syncwarp();
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int i = E * lane + e;
            sel[e] = (int)vose_draw<M>(prob, alias, U[1 + 2 * i] - 1.0f, U[2 + 2 * i] - 1.0f);
        }
    }
    __syncwarp();
    // gather in place, one variable at a time (all reads of a variable before its writes)
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float g[E];
#pragma unroll
        for (int e = 0; e < E; ++e) g[e] = B[v * M + prow<E>(sel[e])];
        __syncwarp();
#pragma unroll
        for (int q = 0; q < E / 4; ++q)
            *reinterpret_cast<float4*>(B + v * M + pchunk<E>(lane, q)) =
                make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
        __syncwarp();
    }
    if (sel_out) {
#pragma unroll
        for (int e = 0; e < E; ++e) sel_out[base + E * lane + e] = sel[e];
    }
}

// The propagated particles of sub-filter b from `state` (original order) into B.
template <int S, int M>
__device__ __forceinline__ void load_state_rows(const FilterDesc& D, int b, float* B, int lane)
{
    constexpr int E = M / 32;
    const int64_t base = (int64_t)b * M;
#pragma unroll
    for (int v = 0; v < S; ++v)
#pragma unroll
        for (int q = 0; q < E / 4; ++q)
            *reinterpret_cast<float4*>(B + v * M + pchunk<E>(lane, q)) =
                *reinterpret_cast<const float4*>(D.state + v * D.T + base + E * lane + 4 * q);
    __syncwarp();
}

// Group + final estimate by the last warps to finish (two-level ticket).
template <int S>
__device__ __forceinline__ void estimate_last_done(const FilterDesc& D, const StepState& X, int b,
                                                   const InputRef& in, int32_t* step_ctr, int lane)
{
    __syncwarp();
    __threadfence();
    const int g = b >> 5, ng = (D.N + 31) >> 5;
    const int gsize = (g == ng - 1) ? D.N - 32 * g : 32;
    int last = 0;
    if (lane == 0) last = atomicAdd(&X.grp_ctr[g], 1) == gsize - 1;
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    constexpr int NVMAX = 2 + 2 * S;
    const int NV = 2 + S + D.na;
    const int sb = 32 * g + lane;
    const bool valid = sb < D.N;
    const double* pp = D.part + (int64_t)(valid ? sb : 32 * g) * kPartStride;
    double gl = valid ? __ldcg(pp) : -INFINITY;
    float wk = valid ? __ldcg(D.winner + sb) : -INFINITY;
    int wi = valid ? sb : 0x7fffffff;
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
    const double sc = valid ? (D.log_weights ? exp(__ldcg(pp) - gl) : 1.0) : 0.0;
    double* go = D.gpart + (int64_t)g * kPartStride;
#pragma unroll
    for (int j = 1; j < NVMAX; ++j) {
        if (j < NV) {
            double v = valid ? sc * __ldcg(pp + j) : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
            if (lane == 0) go[j] = v;
        }
    }
    if (lane == 0) {
        go[0] = D.log_weights ? gl : 0.0;
        go[NV] = (double)wk;
        go[NV + 1] = (double)wi;
        X.grp_ctr[g] = 0;
    }
    // second level: the same combination as estimate_groups
    __syncwarp();
    __threadfence();
    last = 0;
    if (lane == 0) last = atomicAdd(D.est_ctr, 1) == ng - 1;
    last = __shfl_sync(kFull, last, 0);
    if (!last) return;
    __threadfence();
    double gm = -INFINITY;
    float bk = -INFINITY;
    int bi = 0x7fffffff;
    for (int q = lane; q < ng; q += 32) {
        const double* gq = D.gpart + (int64_t)q * kPartStride;
        gm = fmax(gm, __ldcg(gq));
        const float k = (float)__ldcg(gq + NV);
        const int i = (int)__ldcg(gq + NV + 1);
        if (k > bk || (k == bk && i < bi)) {
            bk = k;
            bi = i;
        }
    }
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
    double acc[NVMAX];
#pragma unroll
    for (int j = 0; j < NVMAX; ++j) acc[j] = 0.0;
    for (int q = lane; q < ng; q += 32) {
        const double* gq = D.gpart + (int64_t)q * kPartStride;
        const double sq = D.log_weights ? exp(__ldcg(gq) - gm) : 1.0;
#pragma unroll
        for (int j = 1; j < NVMAX; ++j)
            if (j < NV) acc[j] += sq * __ldcg(gq + j);
    }
#pragma unroll
    for (int j = 1; j < NVMAX; ++j)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(kFull, acc[j], o);
    if (lane == 0) {
        const int best = (bi >= 0 && bi < D.N) ? bi : 0;
        const double lg = D.log_weights ? gm : 0.0;
        const int64_t idx = step_index(in);
        pf_estimate& Eo = D.est[idx];
        const double W = acc[1];
        const int par = (*X.steps) & 1;
        const float* cur_tmp = par ? X.tmp2 : D.tmp;
        int a = 0;
        for (int v = 0; v < PF_MAX_STATE; ++v) Eo.mean[v] = 0.0;
#pragma unroll
        for (int v = 0; v < S; ++v) {
            if ((D.angle_mask >> v) & 1u) {
                Eo.mean[v] = atan2(acc[2 + v], acc[2 + S + a]);
                ++a;
            } else {
                Eo.mean[v] = acc[2 + v] / W;
            }
        }
        Eo.log_norm = lg + log(W);
        for (int v = 0; v < PF_MAX_STATE; ++v)
            Eo.best[v] = v < S ? __ldcg(cur_tmp + v * D.T + (int64_t)best * D.M) : 0.0f;
        Eo.best_key = bk;
        Eo.best_subfilter = best;
        Eo.step = in.ctr ? *in.ctr + 1 : 0;
        Eo.flags = (isfinite(lg) && isfinite(W) && W > 0.0) ? 0 : 1;
        *D.est_ctr = 0;
        *X.need_init = 0;
        __threadfence();
        *X.steps += 1;
        if (step_ctr) *step_ctr += 1;
    }
}

// ---------------------------------------------------------------------------
// The step kernel: kWarpsPerCta sub-filters per CTA, one per warp.
// ---------------------------------------------------------------------------
template <class Mdl, int M, int RES>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_step(const FilterDesc* __restrict__ descs, StepState X,
                                                           const int2* __restrict__ cta_map, InputRef in,
                                                           int32_t* step_ctr)
{
    constexpr int E = M / 32, S = Mdl::S, K = Mdl::K;
    constexpr int RF = LaneRows<E>::F;
    using SM = StepSmem<Mdl, M, RES>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int gw = blockIdx.x * kWarpsPerCta + wp;
    const FilterDesc& D = descs[0];
    if (gw >= D.N) return;
    const int b = gw;
    unsigned char* base_p = smem + (size_t)wp * SM::kPerWarp;
    MtgpRing* ms = reinterpret_cast<MtgpRing*>(base_p);
    float* kb = reinterpret_cast<float*>(base_p);
    unsigned char* Wn = base_p + SM::kA;
    float* nz = reinterpret_cast<float*>(Wn);
    float* B = reinterpret_cast<float*>(base_p + SM::kA + SM::kN);
    typename Mdl::Consts& cst = *reinterpret_cast<typename Mdl::Consts*>(base_p + SM::kA + SM::kN + SM::kB);
    const int64_t T = D.T;
    const int64_t sbase = (int64_t)b * M;
    const int par = (*X.steps) & 1;
    const int init = *X.need_init;
    float* cur_tmp = par ? X.tmp2 : D.tmp;
    float* cur_key = par ? X.tkey2 : D.tkey;
    const float* prev_tmp = par ? D.tmp : X.tmp2;
    const float* prev_key = par ? D.tkey : X.tkey2;
    float* ru = D.ru + (int64_t)b * D.ru_stride;
    // the previous step's resampling draws (in `ru`) are consumed before phase G
    // overwrites them with this step's: R runs first
    const float dec_prev = ru[0] - 1.0f;
    if (lane == 0) Mdl::prepare(cst, *input_of(in, 0), D.mp);
    __syncwarp();
    // ---- R
    if (init || dec_prev > D.freq) {
        load_state_rows<S, M>(D, b, B, lane);
        if (D.sel && !init) {
#pragma unroll
            for (int e = 0; e < E; ++e) D.sel[sbase + E * lane + e] = -1;
        }
    } else {
        phase_resample<S, M, RES>(D, b, prev_tmp, prev_key, ru, B, Wn, lane, D.sel);
    }
    __syncwarp();
    // ---- G: this step's uniforms
    {
        uint32_t* gst = D.mtgp + (int64_t)b * kMtgpN;
        mtgp_load_ring(*ms, gst, (D.stream_base + b) % kMtgpSets, D.mask, lane);
        const int nbm = D.nbm;
        mtgp_generate_ring(*ms, D.draws, lane, [&](int k, uint32_t o) {
            if (k < nbm) nz[k] = __uint_as_float(o);
            else ru[k - nbm] = __uint_as_float(o);
        });
        mtgp_store_ring(*ms, gst, D.draws, lane);
        for (int q = lane; q < nbm / 2; q += 32) {
            float z1, z2;
            box_muller(nz[2 * q], nz[2 * q + 1], z1, z2);
            nz[2 * q] = z1;
            nz[2 * q + 1] = z2;
        }
        __syncwarp();
    }
    // ---- P: propagate + weight, particle i = lane + 32 e; keys go to the (now
    //      free) A region in padded lane rows, ready for the transpose
#pragma unroll 1
    for (int e = 0; e < E; ++e) {
        const int i = lane + 32 * e;
        float st[S], n[K], sn[Mdl::NA], cs[Mdl::NA];
#pragma unroll
        for (int v = 0; v < S; ++v) st[v] = B[v * M + prow<E>(i)];
#pragma unroll
        for (int v = 0; v < K; ++v) n[v] = nz[v * M + i];
        const float ll = Mdl::step(cst, st, n, sn, cs);
        kb[(i / E) * RF + (i % E)] = D.log_weights ? ll : __expf(ll);
#pragma unroll
        for (int v = 0; v < S; ++v) B[v * M + prow<E>(i)] = st[v];
        if (D.inplace) {
#pragma unroll
            for (int v = 0; v < S; ++v) D.state[v * T + sbase + i] = st[v];
        }
    }
    __syncwarp();
    // ---- S: keys in layout A (E consecutive slots per lane), sort
    float k[E];
    int ix[E];
#pragma unroll
    for (int q = 0; q < E; q += 4) {
        const float4 v = *reinterpret_cast<const float4*>(kb + lane * RF + q);
        k[q] = v.x;
        k[q + 1] = v.y;
        k[q + 2] = v.z;
        k[q + 3] = v.w;
    }
#pragma unroll
    for (int e = 0; e < E; ++e) ix[e] = E * lane + e;
    bitonic_warp_desc<M, E>(k, ix, lane);
    // ---- W: sorted keys and particles -> this step's half of the buffer
#pragma unroll
    for (int q = 0; q < E; q += 4)
        *reinterpret_cast<float4*>(cur_key + sbase + E * lane + q) = make_float4(k[q], k[q + 1], k[q + 2], k[q + 3]);
#pragma unroll
    for (int v = 0; v < S; ++v) {
        float o[E];
#pragma unroll
        for (int e = 0; e < E; ++e) o[e] = B[v * M + prow<E>(ix[e])];
#pragma unroll
        for (int q = 0; q < E; q += 4)
            *reinterpret_cast<float4*>(cur_tmp + v * T + sbase + E * lane + q) =
                make_float4(o[q], o[q + 1], o[q + 2], o[q + 3]);
    }
    const float lmax = __shfl_sync(kFull, k[0], 0);
    if (lane == 0) D.winner[b] = k[0];
    // estimate partials in the particle order of phase P
    {
        constexpr int NA = Mdl::NA, NV = 1 + S + NA;
        double acc[NV];
#pragma unroll
        for (int j = 0; j < NV; ++j) acc[j] = 0.0;
        const float lm = D.log_weights ? lmax : 0.0f;
#pragma unroll 1
        for (int e = 0; e < E; ++e) {
            const int i = lane + 32 * e;
            const float ok = kb[(i / E) * RF + (i % E)];
            const double w = D.log_weights ? (double)__expf(ok - lm) : (double)ok;
            acc[0] += w;
            int a = 0;
#pragma unroll
            for (int v = 0; v < S; ++v) {
                const float x = B[v * M + prow<E>(i)];
                if (is_angle_var<Mdl>(v)) {
                    float sn, cs;
                    __sincosf(x, &sn, &cs);
                    acc[1 + v] += w * (double)sn;
                    acc[1 + S + a] += w * (double)cs;
                    ++a;
                } else {
                    acc[1 + v] += w * (double)x;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NV; ++j)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(kFull, acc[j], o);
        if (lane == 0) {
            double* out = D.part + (int64_t)b * kPartStride;
            out[0] = (double)lm;
#pragma unroll
            for (int j = 0; j < NV; ++j) out[1 + j] = acc[j];
        }
    }
    // ---- E
    estimate_last_done<S>(D, X, b, in, step_ctr, lane);
}

// Phase R alone: the particles after the last step's resampling into `state`
// (sel optionally recorded).  Reads the half of the buffer written last.
template <class Mdl, int M, int RES>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_resample_only(const FilterDesc* __restrict__ descs,
                                                                    StepState X)
{
    constexpr int E = M / 32, S = Mdl::S;
    using SM = StepSmem<Mdl, M, RES>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int b = blockIdx.x * kWarpsPerCta + wp;
    const FilterDesc& D = descs[0];
    if (b >= D.N) return;
    if (*X.need_init) return;  // `state` already holds the particles
    unsigned char* base_p = smem + (size_t)wp * SM::kPerWarp;
    unsigned char* Wn = base_p + SM::kA;
    float* B = reinterpret_cast<float*>(base_p + SM::kA + SM::kN);
    const int par = ((*X.steps) & 1) ^ 1;  // half written by the last step
    const float* t_tmp = par ? X.tmp2 : D.tmp;
    const float* t_key = par ? X.tkey2 : D.tkey;
    const float* ru = D.ru + (int64_t)b * D.ru_stride;
    const int64_t sbase = (int64_t)b * M;
    if (ru[0] - 1.0f > D.freq) {
        if (D.sel) {
#pragma unroll
            for (int e = 0; e < E; ++e) D.sel[sbase + E * lane + e] = -1;
        }
        return;  // skipped: `state` holds the propagated particles (written in place)
    }
    phase_resample<S, M, RES>(D, b, t_tmp, t_key, ru, B, Wn, lane, D.sel);
#pragma unroll
    for (int v = 0; v < S; ++v)
#pragma unroll
        for (int q = 0; q < E / 4; ++q)
            *reinterpret_cast<float4*>(D.state + v * D.T + sbase + E * lane + 4 * q) =
                *reinterpret_cast<const float4*>(B + v * M + pchunk<E>(lane, q));
}

}  // namespace pfdev
