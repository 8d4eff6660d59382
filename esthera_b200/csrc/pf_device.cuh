// pf_device.cuh -- device building blocks of the particle-filter step (sm_100a).
//
// Each block restates one routine of the Esthera step with B200-first data
// movement: SoA particle state read as float2/float4 per thread, a
// sub-filter staged in shared memory, warp shuffles for the short sort
// strides and the scans, one MTGP32 stream per CTA generating straight into
// shared memory.  Citations are to the Esthera source tree.
#pragma once
#include <type_traits>

#include <cstdint>
#include <cuda_runtime.h>

#include "esthera_b200.h"

namespace pfdev {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvTwoPi = 0.15915494309189533577f;
constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// MTGP32-11213 (mtgp32-cuda.cu:82-128, 259-306; mtgp32-fast.h:145-214)
// ---------------------------------------------------------------------------
constexpr int kMtgpN = 351;        // state words
constexpr int kMtgpSets = 200;     // parameter sets
constexpr int kMtgpLanes = 256;    // outputs per recursion round (N - max(pos) > 256)
constexpr int kMtgpRing = 1024;    // shared ring; x_j lives at ring[j & 1023]

// The 200 parameter sets, 52 words each (layout in gen_mtgp_params.py).  One
// copy per translation unit; only 41.6 KB and read once per CTA into smem.
static __device__ const uint32_t g_mtgp_params[kMtgpSets * 52] = {
#include "mtgp32_params_11213.inc"
};

struct MtgpSmem {
    uint32_t ring[kMtgpRing];
    uint32_t tbl[16];
    uint32_t ttb[16];  // flt_tmp_tbl (float output) or tmp_tbl (uint32 output)
    uint32_t pos, sh1, sh2, mask;
};

// Stream state words x_0..x_350 -> ring[0..350]; parameter set tables -> smem.
__device__ __forceinline__ void mtgp_load(MtgpSmem& s, const uint32_t* __restrict__ gstate, int set,
                                          uint32_t mask, bool float_out)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < kMtgpN; i += nt) s.ring[i] = gstate[i];
    const uint32_t* P = g_mtgp_params + set * 52;
    for (int i = tid; i < 16; i += nt) {
        s.tbl[i] = P[4 + i];
        s.ttb[i] = float_out ? P[36 + i] : P[20 + i];
    }
    if (tid == 0) {
        s.pos = P[0];
        s.sh1 = P[1];
        s.sh2 = P[2];
        s.mask = mask ? mask : P[3];
    }
    __syncthreads();
}

// mtgp_load with the global reads of the stream words issued first (into
// registers, NT threads) and `work()` run while they are in flight -- the
// sampling kernels compute the step's model constants there.  Same result as
// mtgp_load; ends with a barrier.
template <int NT, class Work>
__device__ __forceinline__ void mtgp_load_overlap(MtgpSmem& s, const uint32_t* __restrict__ gstate, int set,
                                                  uint32_t mask, Work work)
{
    constexpr int R = (kMtgpN + NT - 1) / NT;
    const int tid = threadIdx.x;
    uint32_t w[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = tid + r * NT;
        w[r] = i < kMtgpN ? __ldcs(gstate + i) : 0u;
    }
    const uint32_t* P = g_mtgp_params + set * 52;
    const uint32_t tb = tid < 16 ? P[4 + tid] : 0u, tt = tid < 16 ? P[36 + tid] : 0u;
    work();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = tid + r * NT;
        if (i < kMtgpN) s.ring[i] = w[r];
    }
    if (tid < 16) {
        s.tbl[tid] = tb;
        s.ttb[tid] = tt;
    }
    if (tid == 0) {
        s.pos = P[0];
        s.sh1 = P[1];
        s.sh2 = P[2];
        s.mask = mask ? mask : P[3];
    }
    __syncthreads();
}

// Generate n outputs of the stream held in s.ring, in rounds of 256:
// output k: x_{k+351} = rec(x_k, x_{k+1}, x_{k+pos}); out_k = temper(x_{k+351}, x_{k+pos-1}).
// Within a round every read index is < base+351 <= every write index, so
// the 256 lanes are independent; one barrier separates rounds.  emit(k, word)
// is called for k < n.  Ends with a barrier.
template <class Emit>
__device__ __forceinline__ void mtgp_generate(MtgpSmem& s, int n, bool float_out, Emit emit)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const uint32_t pos = s.pos, sh1 = s.sh1, sh2 = s.sh2, mask = s.mask;
    for (int base = 0; base < n; base += kMtgpLanes) {
        for (int l = tid; l < kMtgpLanes; l += nt) {
            const int k = base + l;
            const uint32_t x1 = s.ring[k & 1023], x2 = s.ring[(k + 1) & 1023];
            uint32_t y = s.ring[(k + pos) & 1023];
            uint32_t t = s.ring[(k + pos - 1) & 1023];
            uint32_t x = (x1 & mask) ^ x2;
            x ^= x << sh1;
            y = x ^ (y >> sh2);
            const uint32_t r = y ^ s.tbl[y & 0x0f];
            s.ring[(k + kMtgpN) & 1023] = r;
            t ^= t >> 16;
            t ^= t >> 8;
            const uint32_t o = float_out ? ((r >> 9) ^ s.ttb[t & 0x0f]) : (r ^ s.ttb[t & 0x0f]);
            if (k < n) emit(k, o);
        }
        __syncthreads();
    }
}

// State after n outputs: x_n .. x_{n+350}.
__device__ __forceinline__ void mtgp_store(const MtgpSmem& s, uint32_t* __restrict__ gstate, int n)
{
    for (int i = threadIdx.x; i < kMtgpN; i += blockDim.x) gstate[i] = s.ring[(n + i) & 1023];
}

// ---------------------------------------------------------------------------
// Box-Muller on MTGP floats in [1,2) (boxmuller, pf_generic_soa.cu:481-500):
// u1 = 2-x, u2 = 2-y in (0,1]; z = sqrt(-2 ln u1) (cos 2 pi u2, sin 2 pi u2).
// The angle is evaluated as 2 pi (u2 - 1/2) in (-pi, pi], where the SFU
// sine/cosine are accurate to ~4e-7 absolute, and the signs flipped back
// (cos(a + pi) = -cos a); the radius uses the SFU reciprocal square root.
// ln u1 keeps the full-precision logf: near u1 = 1 the result is tiny and an
// approximate logarithm would lose all its relative precision.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void box_muller(float x, float y, float& z1, float& z2)
{
    const float u1 = 2.0f - x, u2 = 2.0f - y;
    const float t = -2.0f * logf(u1);
    const float r = t > 0.0f ? t * rsqrtf(t) : 0.0f;
    float s, c;
    __sincosf(kTwoPi * (u2 - 0.5f), &s, &c);
    z1 = -r * c;
    z2 = -r * s;
}

// mtgp_generate for float output with the first nbm words (nbm even) turned
// into normals by Box-Muller on the fly: each thread produces the adjacent
// words (k, k+1) of a round, so the pair's recursion inputs come in 64-bit
// shared loads and the normals go out as one 64-bit store to nz[k], nz[k+1]
// (the same values as mtgp_generate followed by box_muller on nz[2q], nz[2q+1]).
// Words k >= nbm (k < n) go to emit(k, word).  Ends with a barrier.
// RAW: the first nbm words are stored as they are (floats in [1,2)) and the
// caller applies box_muller to each pair (nz[2q], nz[2q+1]) when it reads
// them; the same normals, with the Box-Muller chains taken out of the
// barrier-separated rounds.
template <bool RAW = false, class Emit>
__device__ __forceinline__ void mtgp_generate_bm(MtgpSmem& s, int n, int nbm, float* __restrict__ nz, Emit emit)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const uint32_t pos = s.pos, sh1 = s.sh1, sh2 = s.sh2, mask = s.mask;
    const uint32_t* ring = s.ring;
    auto ld2 = [&](int i) { return *reinterpret_cast<const uint2*>(ring + (i & 1023)); };  // i even
    for (int base = 0; base < n; base += kMtgpLanes) {
        for (int l2 = tid; l2 < kMtgpLanes / 2; l2 += nt) {
            const int k = base + 2 * l2;  // even
            // past the requested words (the last round): nothing this pair
            // writes is read again -- the state kept is x_n .. x_{n+350}, the
            // last of which pair (n-2, n-1) writes
            if (k >= n) continue;
            const uint2 x01 = ld2(k), x23 = ld2(k + 2);
            uint32_t t0, y0, y1;
            if ((pos & 1u) == 0) {
                const uint2 yy = ld2(k + (int)pos);
                y0 = yy.x;
                y1 = yy.y;
                t0 = ld2(k + (int)pos - 2).y;
            } else {
                const uint2 ty = ld2(k + (int)pos - 1), y2 = ld2(k + (int)pos + 1);
                t0 = ty.x;
                y0 = ty.y;
                y1 = y2.x;
            }
            const uint32_t t1 = y0;
            uint32_t xa = (x01.x & mask) ^ x01.y;
            xa ^= xa << sh1;
            uint32_t ya = xa ^ (y0 >> sh2);
            const uint32_t r0 = ya ^ s.tbl[ya & 0x0f];
            uint32_t xb = (x01.y & mask) ^ x23.x;
            xb ^= xb << sh1;
            uint32_t yb = xb ^ (y1 >> sh2);
            const uint32_t r1 = yb ^ s.tbl[yb & 0x0f];
            s.ring[(k + kMtgpN) & 1023] = r0;
            s.ring[(k + kMtgpN + 1) & 1023] = r1;
            uint32_t ta = t0;
            ta ^= ta >> 16;
            ta ^= ta >> 8;
            uint32_t tb = t1;
            tb ^= tb >> 16;
            tb ^= tb >> 8;
            const uint32_t o0 = (r0 >> 9) ^ s.ttb[ta & 0x0f];
            const uint32_t o1 = (r1 >> 9) ^ s.ttb[tb & 0x0f];
            if (k < nbm) {
                if constexpr (RAW) {
                    *reinterpret_cast<uint2*>(nz + k) = make_uint2(o0, o1);
                } else {
                    float z1, z2;
                    box_muller(__uint_as_float(o0), __uint_as_float(o1), z1, z2);
                    *reinterpret_cast<float2*>(nz + k) = make_float2(z1, z2);
                }
            } else {
                if (k < n) emit(k, o0);
                if (k + 1 < n) emit(k + 1, o1);
            }
        }
        __syncthreads();
    }
}

// atan2 from an odd polynomial for atan on [0, 1] -- degree 15 in a, i.e. 8
// coefficients in a^2, fitted for this project by least squares on 4000
// Chebyshev nodes refined with Lawson iterations towards the minimax fit
// (max error 1.4e-7 in FP32 Horner) -- plus octant reduction with one fast
// division.  Max absolute error about 3e-7 rad.  fit_atan2.py (beside this
// file) regenerates the fit and checks both bounds against FP64 atan2.
__device__ __forceinline__ float pf_atan2(float y, float x)
{
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    const float a = mx > 0.0f ? __fdividef(mn, mx) : 0.0f;
    const float s = a * a;
    float p = -4.054567008e-03f;
    p = fmaf(p, s, 2.186295757e-02f);
    p = fmaf(p, s, -5.591232720e-02f);
    p = fmaf(p, s, 9.642197449e-02f);
    p = fmaf(p, s, -1.390862965e-01f);
    p = fmaf(p, s, 1.994656569e-01f);
    p = fmaf(p, s, -3.332986079e-01f);
    p = fmaf(p, s, 9.999993356e-01f);
    float r = a * p;
    if (ay > ax) r = 1.57079632679489662f - r;
    if (x < 0.0f) r = kPi - r;
    return copysignf(r, y);
}

// exp(x) for the resampling's max-subtracted log-weights x <= 0, from
// correctly rounded FP32 operations only (no SFU approximation), so that the
// oracle's restatement (orc_expneg) gives the same bits and resampling is
// bit-identical given identical log-weights: n = rint(x log2 e), r = x - n ln2
// (Cody-Waite split, two fmaf), exp(x) = 2^n P(r), P of degree 6 fitted for
// this project (least squares + Lawson iterations on [-ln2/2, ln2/2],
// relative error 2.3e-9; fit_exp.py beside this file regenerates and checks
// it: at most 2 ulp on [-87, 0]).  x < -87 (and -inf) gives 0, NaN stays NaN.
__device__ __forceinline__ float pf_expneg(float x)
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
    const int ni = (int)n;
    const bool ok = x >= -87.0f && ni >= -126;
    const float scale = __int_as_float((ok ? ni + 127 : 0) << 23);
    return x != x ? x : (ok ? p * scale : 0.0f);
}

// sqrt(d2) for d2 >= 0 through the SFU reciprocal square root (0 -> 0).
__device__ __forceinline__ float pf_sqrt(float d2) { return d2 * rsqrtf(fmaxf(d2, 1e-30f)); }

// ---------------------------------------------------------------------------
// Descending bitonic key+index sort of M keys, E consecutive keys per thread
// (thread t holds positions E*t .. E*t+E-1).  The comparator network is the
// reference's (bitonic-sort.cu:28-61 with dir = 0): for every (size, stride)
// the pair (p, p+stride) with p & stride == 0 swaps iff
// (key[p] > key[p+stride]) == ((p & size) != 0), so equal keys swap.
// Strides below E are register pairs, strides below 32E are warp shuffles,
// longer strides go through shared memory (sk/si hold M entries).  `tid` is
// the thread's rank within the sub-filter (the lane when a warp owns one).
// TP = 2: two adjacent lanes hold the same E keys (two threads per particle);
// the pair runs the network together (lane masks doubled) and only the
// `writer` lane stores to shared memory.
// ---------------------------------------------------------------------------
template <int M, int E, int TP = 1>
__device__ __forceinline__ void bitonic_sort_desc(float (&k)[E], int (&ix)[E], float* sk, int* si,
                                                  int tid = threadIdx.x, bool writer = true)
{
#pragma unroll
    for (int size = 2; size <= M; size <<= 1) {
#pragma unroll
        for (int stride = size / 2; stride > 0; stride >>= 1) {
            if (stride < E) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    if ((e & stride) == 0) {
                        const int p = E * tid + e;
                        const bool ddd = (p & size) != 0;
                        const float a = k[e], b = k[e + stride];
                        if ((a > b) == ddd) {
                            k[e] = b;
                            k[e + stride] = a;
                            const int t = ix[e];
                            ix[e] = ix[e + stride];
                            ix[e + stride] = t;
                        }
                    }
                }
            } else if (stride < (32 / TP) * E) {
                const int lm = stride / E;
                const bool upper = (tid & lm) != 0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const float ok = __shfl_xor_sync(kFull, k[e], lm * TP);
                    const int oi = __shfl_xor_sync(kFull, ix[e], lm * TP);
                    const int p = E * tid + e;
                    const bool ddd = (p & size) != 0;
                    const float lo = upper ? ok : k[e];
                    const float hi = upper ? k[e] : ok;
                    if ((lo > hi) == ddd) {
                        k[e] = ok;
                        ix[e] = oi;
                    }
                }
            } else {
                __syncthreads();
                if (writer) {
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        sk[E * tid + e] = k[e];
                        si[E * tid + e] = ix[e];
                    }
                }
                __syncthreads();
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int p = E * tid + e;
                    const int q = p ^ stride;
                    const float ok = sk[q];
                    const int oi = si[q];
                    const bool ddd = (p & size) != 0;
                    const bool upper = (p & stride) != 0;
                    const float lo = upper ? ok : k[e];
                    const float hi = upper ? k[e] : ok;
                    if ((lo > hi) == ddd) {
                        k[e] = ok;
                        ix[e] = oi;
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The same descending sort when ties are rare (small-state models, whose keys
// are continuous functions of freshly perturbed states).  With distinct keys
// the sorted permutation is unique, so any correct sort gives the network's
// result; this one runs the network on the keys alone (a shuffle and a min /
// max per element and stage instead of two shuffles and four selects), then
// recovers the permutation: each thread finds the sorted position of each of
// its keys by a binary search over the sorted keys in shared memory and
// writes its index there.  If any two keys compare equal (ties, +0 / -0,
// repeated -inf) or a key is NaN, the whole CTA (every thread takes the same
// branch) sorts the original (key, index) pairs with bitonic_sort_desc, which
// keeps the reference network's tie order.  Same contract as
// bitonic_sort_desc for a CTA owning one sub-filter (tid = threadIdx.x);
// returns true when the CTA fell back to the full network.  TP as for
// bitonic_sort_desc (the pair's lanes hold the same keys).
// ---------------------------------------------------------------------------
template <int M, int E, int TP = 1>
__device__ __forceinline__ bool rank_sort_desc(float (&k)[E], int (&ix)[E], float* sk, int* si)
{
    const int tid = threadIdx.x / TP;
    const bool writer = threadIdx.x % TP == 0;
    float v[E];
    bool nan = false;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        v[e] = k[e];
        nan |= k[e] != k[e];
    }
    // the keys alone through a bitonic network in its mirrored form: the first
    // stage of each merge pairs p with p ^ (size - 1), the later ones p with
    // p ^ stride, and every comparator leaves the larger key at the lower
    // position (no direction bit per block)
#pragma unroll
    for (int size = 2; size <= M; size <<= 1) {
#pragma unroll
        for (int stride = size / 2; stride > 0; stride >>= 1) {
            const bool first = stride == size / 2;
            if (stride < E) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int pe = first ? (e ^ (size - 1)) : (e ^ stride);
                    if (e < pe) {
                        const float hi = fmaxf(v[e], v[pe]), lo = fminf(v[e], v[pe]);
                        v[e] = hi;
                        v[pe] = lo;
                    }
                }
            } else if (stride < (32 / TP) * E) {
                // partner thread tid ^ lm (first stage: tid ^ (size / E - 1),
                // element E - 1 - e); the lower thread of the pair keeps the maxima
                const int lm = first ? size / E - 1 : stride / E;
                const bool keep_max = (tid & (stride / E)) == 0;
                float o[E];
#pragma unroll
                for (int e = 0; e < E; ++e) o[e] = __shfl_xor_sync(kFull, v[first ? E - 1 - e : e], lm * TP);
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = keep_max ? fmaxf(v[e], o[e]) : fminf(v[e], o[e]);
            } else {
                __syncthreads();
                if (writer) {
#pragma unroll
                    for (int e = 0; e < E; ++e) sk[E * tid + e] = v[e];
                }
                __syncthreads();
                const bool keep_max = ((E * tid) & stride) == 0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int p = E * tid + e;
                    const float o = sk[first ? p ^ (size - 1) : p ^ stride];
                    v[e] = keep_max ? fmaxf(v[e], o) : fminf(v[e], o);
                }
            }
        }
    }
    __syncthreads();
    if (writer) {
#pragma unroll
        for (int e = 0; e < E; ++e) sk[E * tid + e] = v[e];
    }
    __syncthreads();
    bool tie = nan;
#pragma unroll
    for (int e = 0; e + 1 < E; ++e) tie |= v[e] == v[e + 1];
    if (E * tid + E < M) tie |= v[E - 1] == sk[E * tid + E];
    if (__syncthreads_or(tie)) {
        bitonic_sort_desc<M, E, TP>(k, ix, sk, si, tid, writer);
        return true;
    }
    // sorted position of each original key = the number of keys above it
#pragma unroll
    for (int e = 0; e < E; ++e) {
        int pos = 0;
#pragma unroll
        for (int step = M / 2; step > 0; step >>= 1)
            if (sk[pos + step - 1] > k[e]) pos += step;
        if (writer) si[pos] = E * tid + e;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; ++e) {
        k[e] = v[e];
        ix[e] = si[E * tid + e];
    }
    return false;
}

// ---------------------------------------------------------------------------
// Block reductions / scans.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float block_max(float v, float* red)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    float r = red[0];
    for (int i = 1; i < nw; ++i) r = fmaxf(r, red[i]);
    return r;
}

// Canonical FP64 inclusive scan (the oracle's orc_scan_f64): each thread sums
// its E weights sequentially, lanes combine with a Kogge-Stone scan, warp
// totals with a second Kogge-Stone scan; cum[e] receives the inclusive sum
// through particle E*tid + e (kept in registers).  *prev receives the
// inclusive sum through particle E*tid - 1 as the previous thread computed it
// (-inf for thread 0).  Returns the total.  red needs 2 * 32 doubles; two
// barriers: every warp forms the prefix of the warp totals itself (the same
// additions in the same order as one warp scanning them), and the last
// thread of each warp publishes its last sum for the first thread of the
// next.
template <int M, int E>
__device__ __forceinline__ double scan_f64(const float (&w)[E], double (&cum)[E], double* red, double* prev)
{
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    constexpr int NW = (M / E + 31) / 32;
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
    if (lane == 31) red[wp] = inc;
    __syncthreads();
    double v = lane < NW ? red[lane] : 0.0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double o = __shfl_up_sync(kFull, v, d);
        if (lane >= d) v = v + o;
    }
    const double wpre = __shfl_sync(kFull, v, wp > 0 ? wp - 1 : 0);  // inclusive prefix of the warps before
    const double base = (wp == 0 ? 0.0 : wpre) + ex;
    double c = base + (double)w[0];
    cum[0] = c;
#pragma unroll
    for (int e = 1; e < E; ++e) {
        c = c + (double)w[e];
        cum[e] = c;
    }
    double p = __shfl_up_sync(kFull, cum[E - 1], 1);
    if (lane == 31) red[32 + wp] = cum[E - 1];
    __syncthreads();
    if (lane == 0) p = wp == 0 ? -INFINITY : red[32 + wp - 1];
    *prev = p;
    return red[32 + NW - 1];
}

// Number of cum[] entries <= x (upper bound), clamped to M-1.
template <int M>
__device__ __forceinline__ int upper_count(const double* cum, double x)
{
    int lo = 0, hi = M;
#pragma unroll
    for (int it = 0; it < 11; ++it) {
        if (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cum[mid] <= x) lo = mid + 1;
            else hi = mid;
        }
    }
    return lo < M ? lo : M - 1;
}

// Systematic selection from the inclusive sums (scan_f64: this thread's cum[e]
// and the previous thread's last sum `prev`) by interval boundaries: input j
// is selected by the outputs i with cum[j-1] <= pos(i) < cum[j],
// pos(i) = (u0 + i) * step (cum[-1] = -inf; the last input also takes every
// output with pos(i) >= cum[M-1]).  Each thread finds, for its E inputs
// j = E*tid+e, the first output at or above cum[j-1] (an estimate from t /
// step, corrected with the exact pos(i) comparisons), writes its inputs' runs
// of outputs to sidx[0..M), and reads back its own E outputs.  pos(i) and the
// comparisons are those of upper_count(cum, pos(i)), so every output selects
// the same input (pos is non-decreasing in i).  Synchronises the CTA.
template <int M, int E>
__device__ __forceinline__ void systematic_select(const double (&cum)[E], double prev, float u0f, double step,
                                                  int* sidx, int (&sel)[E])
{
    const int tid = threadIdx.x;
    const double u0 = (double)u0f;
    const double inv = step > 0.0 ? 1.0 / step : 0.0;
    auto pos = [&](int i) { return (u0 + (double)i) * step; };
    auto first_at_or_above = [&](double t) {  // first i in [0, M] with pos(i) >= t
        const double est = ceil(t * inv - u0);
        int i = est >= 0.0 ? (est <= (double)M ? (int)est : M) : 0;
        while (i > 0 && pos(i - 1) >= t) --i;
        while (i < M && pos(i) < t) ++i;
        return i;
    };
    const int j0 = E * tid;
    int lo = j0 == 0 ? 0 : first_at_or_above(prev);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int j = j0 + e;
        const int hi = j == M - 1 ? M : first_at_or_above(cum[e]);
        for (int i = lo; i < hi; ++i) sidx[i] = j;
        lo = hi > lo ? hi : lo;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; ++e) sel[e] = sidx[E * tid + e];
}

// FP32 Blelloch exclusive scan of M values in place (prefix_sum,
// pf_generic_soa.cu:169-216); same tree, pairs shared out over the block.
template <int M>
__device__ __forceinline__ float blelloch_scan(float* e)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    int offset = 1;
    for (int d = M / 2; d > 0; d /= 2) {
        __syncthreads();
        for (int q = tid; q < d; q += nt) {
            const int ai = offset * (2 * q + 1) - 1, bi = offset * (2 * q + 2) - 1;
            e[bi] += e[ai];
        }
        offset *= 2;
    }
    __syncthreads();
    const float cum = e[M - 1];
    __syncthreads();
    if (tid == 0) e[M - 1] = 0.0f;
    for (int d = 1; d < M; d *= 2) {
        offset /= 2;
        __syncthreads();
        for (int q = tid; q < d; q += nt) {
            const int ai = offset * (2 * q + 1) - 1, bi = offset * (2 * q + 2) - 1;
            const float t = e[ai];
            e[ai] = e[bi];
            e[bi] += t;
        }
    }
    __syncthreads();
    return cum;
}

// binary_search, pf_generic_soa.cu:221-240: last i with hay[i] <= needle.
__device__ __forceinline__ int ref_binary_search(const float* hay, float needle, int size)
{
    int lo = 0, hi = size - 1;
    do {
        const int cur = lo + (hi - lo + 1) / 2;
        if (hay[cur] > needle) hi = cur - 1;
        else lo = cur;
    } while (lo < hi);
    return lo;
}

// Block-wide exclusive count of `flag` in ascending rank order where rank =
// tid + nt*round; returns this thread's exclusive count, *total the sum.
// red needs 33 ints.  Contains barriers: every thread must call.
__device__ __forceinline__ int block_excl_count(bool flag, int* red, int* total)
{
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5, nw = blockDim.x >> 5;
    const unsigned b = __ballot_sync(kFull, flag);
    const int in_warp = __popc(b & ((1u << lane) - 1u));
    __syncthreads();
    if (lane == 0) red[wp] = __popc(b);
    __syncthreads();
    int before = 0, tot = 0;
    for (int i = 0; i < nw; ++i) {
        const int c = red[i];
        if (i < wp) before += c;
        tot += c;
    }
    *total = tot;
    return before + in_warp;
}

// Vose alias table of M weights (resampling-valias.cl:85-195 + 262-270) in
// FP32 with the reference's arithmetic: sum_reduce4 order, p = w/sum (or
// 1/M), prob = p*M, small iff prob <= 1, pairing prob_L = (prob_L + prob_S) - 1.
// Work lists are filled in ascending slot order where the reference uses
// atomic_inc / atomic_dec (the oracle does the same).  Shared: prob[M],
// alias[M], sl[M], scratch[M] floats, red[33].
template <int M, int E>
__device__ void vose_build(const float (&w)[E], float* prob, unsigned* alias, unsigned* sl,
                           float* scratch, int* red)
{
    const int tid = threadIdx.x, nt = blockDim.x;
#pragma unroll
    for (int e = 0; e < E; ++e) scratch[E * tid + e] = w[e];
    __syncthreads();
    // sum_reduce4
    int offset = M;
    while (offset > 2) {
        offset >>= 2;
        for (int l = tid; l < offset; l += nt) {
            const float x = scratch[l + offset] + scratch[l + offset + offset] + scratch[l + offset + offset + offset];
            scratch[l] = scratch[l] + x;
        }
        __syncthreads();
    }
    if (offset > 1) {
        if (tid == 0) scratch[0] = scratch[0] + scratch[1];
        __syncthreads();
    }
    const float sum = scratch[0];
    // normalise, scale, initial split (small ascending from 0, large descending from M-1)
    int ns_before = 0;
    for (int e = 0; e < E; ++e) {
        const int i = E * tid + e;
        float p = w[e];
        if (sum > 0.0f) p = p / sum;
        else p = 1.0f / (float)M;
        prob[i] = p * (float)M;
        alias[i] = (unsigned)i;
    }
    // ascending i = E*tid + e: count smalls of lower threads, then within thread
    int my_small = 0;
    bool fl[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        fl[e] = prob[E * tid + e] <= 1.0f;
        my_small += fl[e] ? 1 : 0;
    }
    {
        // exclusive scan of my_small over threads (ascending tid)
        const int lane = tid & 31, wp = tid >> 5, nw = nt >> 5;
        int inc = my_small;
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(kFull, inc, d);
            if (lane >= d) inc += o;
        }
        __syncthreads();
        if (lane == 31) red[wp] = inc;
        __syncthreads();
        int wbase = 0, tot = 0;
        for (int i = 0; i < nw; ++i) {
            if (i < wp) wbase += red[i];
            tot += red[i];
        }
        ns_before = wbase + inc - my_small;
        int nl_before = E * tid - ns_before;
        int s_i = ns_before, l_i = nl_before;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int i = E * tid + e;
            if (fl[e]) sl[s_i++] = (unsigned)i;
            else sl[M - 1 - (l_i++)] = (unsigned)i;
        }
        __syncthreads();
        if (tid == 0) red[32] = tot;
        __syncthreads();
    }
    unsigned small_end = (unsigned)red[32];
    unsigned large_rend = small_end - 1u;  // = M-1 - n_large
    unsigned small_begin = 0;
    __syncthreads();
    // Pairing rounds; each retires >= 1 small entry, so <= M rounds.  Round:
    // the first `nactive` smalls take the `nactive` larges at the bottom of the
    // large list as aliases, the larges' reduced probabilities are appended to
    // the small list (ascending) or pushed back on the large list, in pair
    // order.  Rounds of at most 32 pairs (the common case once the few large
    // weights are being used up) run in warp 0 alone, without CTA barriers.
    const int lane = tid & 31;
    for (int round = 0; round < M;) {
        const unsigned se = small_end;
        const unsigned a = se - small_begin, b = (unsigned)M - se;
        const unsigned nactive = a < b ? a : b;
        if (nactive == 0) break;
        if (nactive <= 32) {
            if (tid < 32) {
                unsigned sb = small_begin, sen = small_end, lr = large_rend;
                int rr = round;
                for (; rr < M; ++rr) {
                    const unsigned aa = sen - sb, bb = (unsigned)M - sen;
                    const unsigned na = aa < bb ? aa : bb;
                    if (na == 0 || na > 32) break;
                    if (bb == 1) {
                        // One large entry left: every further round pairs it with the
                        // next small one until its probability drops to <= 1 (it then
                        // joins the small list and the pairing ends) or the smalls run
                        // out.  Lane 0 runs those rounds back to back: the same pairs,
                        // arithmetic and list updates as one round at a time.
                        if (lane == 0) {
                            const unsigned L = sl[sen];
                            float pl = prob[L];
                            bool to_small = false;
                            while (sb < sen && rr < M) {
                                unsigned sm[4];
                                float ps[4];
                                const unsigned left = sen - sb;
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    sm[q] = (unsigned)q < left ? sl[sb + q] : 0u;
                                    ps[q] = (unsigned)q < left ? prob[sm[q]] : 0.0f;
                                }
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    if (!to_small && (unsigned)q < left && rr < M) {
                                        alias[sm[q]] = L;
                                        pl = (pl + ps[q]) - 1.0f;
                                        ++sb;
                                        ++rr;
                                        to_small = pl <= 1.0f;
                                    }
                                }
                                if (to_small) break;
                            }
                            prob[L] = pl;
                            if (to_small) {
                                ++sen;  // sl[sen] already holds L: it becomes the last small entry
                                ++lr;
                            }
                        }
                        sb = __shfl_sync(kFull, sb, 0);
                        sen = __shfl_sync(kFull, sen, 0);
                        lr = __shfl_sync(kFull, lr, 0);
                        rr = __shfl_sync(kFull, rr, 0);
                        __syncwarp();
                        break;
                    }
                    lr += na;
                    const bool act = (unsigned)lane < na;
                    unsigned li = 0;
                    float nl = 0.0f;
                    bool small = false;
                    if (act) {
                        const unsigned si2 = sl[sb + lane];
                        li = sl[sen + lane];
                        alias[si2] = li;
                        nl = (prob[li] + prob[si2]) - 1.0f;
                        small = nl <= 1.0f;
                    }
                    __syncwarp();  // every read of this round's list entries precedes the writes
                    const unsigned bs = __ballot_sync(kFull, act && small);
                    const unsigned bl = __ballot_sync(kFull, act && !small);
                    const unsigned below = (1u << lane) - 1u;
                    if (act) {
                        const unsigned dst = small ? sen + (unsigned)__popc(bs & below)
                                                   : lr - (unsigned)__popc(bl & below);
                        sl[dst] = li;
                        prob[li] = nl;
                    }
                    sen += (unsigned)__popc(bs);
                    lr -= (unsigned)__popc(bl);
                    sb += na;
                    __syncwarp();
                }
                if (lane == 0) {
                    red[0] = (int)sb;
                    red[1] = (int)sen;
                    red[2] = (int)lr;
                    red[3] = rr;
                }
            }
            __syncthreads();
            small_begin = (unsigned)red[0];
            small_end = (unsigned)red[1];
            large_rend = (unsigned)red[2];
            round = red[3];
            __syncthreads();
            continue;
        }
        ++round;
        large_rend += nactive;
        constexpr int R = (M / 2 + 31) / 32 + 1;  // upper bound on items per thread
        unsigned lidx[R];
        float pS[R], pL[R];
        int nitems = 0;
        for (unsigned kk = tid, r = 0; kk < nactive && r < (unsigned)R; kk += nt, ++r) {
            const unsigned sidx = sl[small_begin + kk];
            lidx[r] = sl[se + kk];
            pS[r] = prob[sidx];
            alias[sidx] = lidx[r];
            pL[r] = prob[lidx[r]];
            nitems = (int)r + 1;
        }
        __syncthreads();
        unsigned s_base = 0, l_base = 0;
        const int rounds = (int)((nactive + nt - 1) / nt);
        for (int r = 0; r < rounds; ++r) {
            const unsigned kk = (unsigned)tid + (unsigned)r * nt;
            const bool act = kk < nactive;
            float nl = 0.0f;
            bool small = false;
            if (act && r < nitems) {
                nl = (pL[r] + pS[r]) - 1.0f;
                small = nl <= 1.0f;
            }
            int tot_s;
            const int rank_s = block_excl_count(act && small, red, &tot_s);
            int tot_l;
            const int rank_l = block_excl_count(act && !small, red, &tot_l);
            if (act) {
                const unsigned dst = small ? small_end + s_base + (unsigned)rank_s
                                           : large_rend - l_base - (unsigned)rank_l;
                sl[dst] = lidx[r];
                prob[lidx[r]] = nl;
            }
            s_base += (unsigned)tot_s;
            l_base += (unsigned)tot_l;
        }
        small_end += s_base;
        large_rend -= l_base;
        small_begin += nactive;
        __syncthreads();
    }
}

// vose_alias_generate_next (resampling-valias.cl:198-202).
template <int M>
__device__ __forceinline__ unsigned vose_draw(const float* prob, const unsigned* alias, float ux, float uy)
{
    unsigned col = (unsigned)floorf(ux * (float)M);
    if (col >= (unsigned)M) col = M - 1;
    return (uy < prob[col]) ? col : alias[col];
}

// ---------------------------------------------------------------------------
// Models.  Each provides S (state floats), K (normals per particle), NA
// (angular state variables, reported as sin/cos for circular means),
// prepare() (per-step constants, called by the 32 lanes of one warp: each
// lane fills its own fields, the transcendental ones one per lane so the
// FP64 chains run side by side instead of one after another) and step() (one particle:
// propagate in place, return the FP32 log-likelihood, and sin/cos of the
// angular variables of the new state).
// ---------------------------------------------------------------------------
constexpr int kMaxModelParamBytes = 256;  // a registered model's parameter struct fits here
union ModelParams {
    pf_unicycle_params uni;
    pf_dharm_params arm;
    pf_refarm_params ref;
    pf_beacon_params bcn;
    pf_camarm_params cam;
    unsigned char raw[kMaxModelParamBytes];  // any other registered model's parameters (esthera_b200_model.cuh)
};

__device__ __forceinline__ float wrap_pi(float a) { return fmaf(-kTwoPi, floorf((a + kPi) * kInvTwoPi), a); }

struct Unicycle {
    static constexpr int S = 3, K = 3, NA = 1, C = 2, Z = 16;
    __host__ __device__ static constexpr int angle_var(int) { return 2; }
    struct Consts {
        float A, B, wd, sq0, sq1, sq2, isr, isb;
        int L;
        float lx[8], ly[8], rm[8], cb[8], sb[8];
    };
    // Exact-arc velocity model: x' = x + A cos th - B sin th, y' = y + A sin th + B cos th
    // with A = v sin(w dt)/w, B = v (1 - cos(w dt))/w (straight-line limit as w -> 0),
    // evaluated in FP32 through the half angle h = w dt / 2: sin(w dt) = 2 sin h cos h,
    // 1 - cos(w dt) = 2 sin^2 h (no cancellation for small w dt).
    // lane 8: motion constants; lanes 0..7: landmark `lane`
    __device__ static void prepare(Consts& c, const pf_step_input& in, const ModelParams& mp, int lane)
    {
        const pf_unicycle_params& p = mp.uni;
        const int L = p.num_landmarks < 1 ? 1 : (p.num_landmarks > 8 ? 8 : p.num_landmarks);
        if (lane == 8) {
            const float dt = in.dt > 0.0f ? in.dt : p.dt;
            const float v = in.control[0], w = in.control[1];
            const float wd = w * dt;
            float A, B;
            if (fabsf(wd) < 1e-4f) {
                A = v * dt * (1.0f - wd * wd / 6.0f);
                B = v * dt * (wd * 0.5f);
            } else {
                float sh, ch;
                sincosf(0.5f * wd, &sh, &ch);
                A = v * (2.0f * sh * ch) / w;
                B = v * (2.0f * sh * sh) / w;
            }
            c.A = A;
            c.B = B;
            c.wd = wd;
            c.sq0 = p.sigma_q[0];
            c.sq1 = p.sigma_q[1];
            c.sq2 = p.sigma_q[2];
            c.isr = 1.0f / p.sigma_range;
            c.isb = 1.0f / p.sigma_bearing;
            c.L = L;
        } else if (lane < 8) {
            const int j = lane;
            c.lx[j] = p.landmarks[j][0];
            c.ly[j] = p.landmarks[j][1];
            c.rm[j] = j < L ? in.meas[j] : 0.0f;
            sincosf(j < L ? in.meas[L + j] : 0.0f, &c.sb[j], &c.cb[j]);
        }
    }
    __device__ static __forceinline__ float step(const Consts& c, float* s, const float* n, float* sn,
                                                 float* cs)
    {
        float st, ct;
        __sincosf(s[2], &st, &ct);
        const float nx = fmaf(c.sq0, n[0], fmaf(c.A, ct, fmaf(-c.B, st, s[0])));
        const float ny = fmaf(c.sq1, n[1], fmaf(c.A, st, fmaf(c.B, ct, s[1])));
        const float nt = wrap_pi(fmaf(c.sq2, n[2], s[2] + c.wd));
        s[0] = nx;
        s[1] = ny;
        s[2] = nt;
        float s2, c2;
        __sincosf(nt, &s2, &c2);
        sn[0] = s2;
        cs[0] = c2;
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (j < c.L) {
                const float dx = c.lx[j] - nx, dy = c.ly[j] - ny;
                const float r = pf_sqrt(fmaf(dx, dx, dy * dy));
                const float er = (c.rm[j] - r) * c.isr;
                const float cp = fmaf(c2, c.cb[j], -(s2 * c.sb[j]));
                const float sp = fmaf(s2, c.cb[j], c2 * c.sb[j]);
                const float eb = pf_atan2(fmaf(sp, dx, -(cp * dy)), fmaf(cp, dx, sp * dy)) * c.isb;
                acc = fmaf(er, er, acc);
                acc = fmaf(eb, eb, acc);
            }
        }
        return -0.5f * acc;
    }
    // Two threads per particle (lane pair h = 0, 1): both lanes propagate the
    // particle (identical arithmetic), each sums the landmarks j = h, h + 2,
    // ..., and the pair adds the two sums in lane order.
    __device__ static __forceinline__ float step_pair(const Consts& c, float* s, const float* n, int h, float* sn,
                                                      float* cs)
    {
        float st, ct;
        __sincosf(s[2], &st, &ct);
        const float nx = fmaf(c.sq0, n[0], fmaf(c.A, ct, fmaf(-c.B, st, s[0])));
        const float ny = fmaf(c.sq1, n[1], fmaf(c.A, st, fmaf(c.B, ct, s[1])));
        const float nt = wrap_pi(fmaf(c.sq2, n[2], s[2] + c.wd));
        s[0] = nx;
        s[1] = ny;
        s[2] = nt;
        float s2, c2;
        __sincosf(nt, &s2, &c2);
        sn[0] = s2;
        cs[0] = c2;
        float acc = 0.0f;
#pragma unroll 1
        for (int j = h; j < c.L; j += 2) {
            const float dx = c.lx[j] - nx, dy = c.ly[j] - ny;
            const float r = pf_sqrt(fmaf(dx, dx, dy * dy));
            const float er = (c.rm[j] - r) * c.isr;
            const float cp = fmaf(c2, c.cb[j], -(s2 * c.sb[j]));
            const float sp = fmaf(s2, c.cb[j], c2 * c.sb[j]);
            const float eb = pf_atan2(fmaf(sp, dx, -(cp * dy)), fmaf(cp, dx, sp * dy)) * c.isb;
            acc = fmaf(er, er, acc);
            acc = fmaf(eb, eb, acc);
        }
        const float o = __shfl_xor_sync(kFull, acc, 1);
        return -0.5f * (h ? o + acc : acc + o);
    }
    // E particles at once: the same per-particle arithmetic as step() in the
    // same order (bit-identical results), with the landmark loop outside the
    // particle loop so each landmark's constants are read once per thread and
    // the E likelihood chains interleave.  noise(e, v) gives particle e's v-th
    // normal.
    template <int E, class Noise>
    __device__ static __forceinline__ void step_batch(const Consts& c, float (&s)[E][S], Noise noise,
                                                      float (&sn)[E][NA], float (&cs)[E][NA], float (&ll)[E])
    {
        float s2[E], c2[E], acc[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            float st, ct;
            __sincosf(s[e][2], &st, &ct);
            const float nx = fmaf(c.sq0, noise(e, 0), fmaf(c.A, ct, fmaf(-c.B, st, s[e][0])));
            const float ny = fmaf(c.sq1, noise(e, 1), fmaf(c.A, st, fmaf(c.B, ct, s[e][1])));
            const float nt = wrap_pi(fmaf(c.sq2, noise(e, 2), s[e][2] + c.wd));
            s[e][0] = nx;
            s[e][1] = ny;
            s[e][2] = nt;
            __sincosf(nt, &s2[e], &c2[e]);
            sn[e][0] = s2[e];
            cs[e][0] = c2[e];
            acc[e] = 0.0f;
        }
        const int L = c.L;
        const float isr = c.isr, isb = c.isb;
#pragma unroll 1
        for (int j = 0; j < L; ++j) {
            const float lx = c.lx[j], ly = c.ly[j], rm = c.rm[j], cb = c.cb[j], sb = c.sb[j];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const float dx = lx - s[e][0], dy = ly - s[e][1];
                const float r = pf_sqrt(fmaf(dx, dx, dy * dy));
                const float er = (rm - r) * isr;
                const float cp = fmaf(c2[e], cb, -(s2[e] * sb));
                const float sp = fmaf(s2[e], cb, c2[e] * sb);
                const float eb = pf_atan2(fmaf(sp, dx, -(cp * dy)), fmaf(cp, dx, sp * dy)) * isb;
                acc[e] = fmaf(er, er, acc[e]);
                acc[e] = fmaf(eb, eb, acc[e]);
            }
        }
#pragma unroll
        for (int e = 0; e < E; ++e) ll[e] = -0.5f * acc[e];
    }
};

struct DhArm {
    static constexpr int S = 12, K = 6, NA = 6, C = 0, Z = 6;
    __host__ __device__ static constexpr int angle_var(int a) { return a; }
    struct Consts {
        float dt, sqd, isp, isa;
        float a[6], d[6], ca[6], sa[6], z[6];
    };
    // lane 6: scalars; lanes 0..5: joint `lane`
    __device__ static void prepare(Consts& c, const pf_step_input& in, const ModelParams& mp, int lane)
    {
        const pf_dharm_params& p = mp.arm;
        if (lane == 6) {
            c.dt = in.dt > 0.0f ? in.dt : p.dt;
            c.sqd = p.sigma_qd;
            c.isp = 1.0f / p.sigma_pos;
            c.isa = 1.0f / p.sigma_ang;
        } else if (lane < 6) {
            const int i = lane;
            c.a[i] = p.a[i];
            c.d[i] = p.d[i];
            sincosf(p.alpha[i], &c.sa[i], &c.ca[i]);
            c.z[i] = in.meas[i];
        }
    }
    __device__ static __forceinline__ float step(const Consts& c, float* s, const float* n, float* sn,
                                                 float* cs)
    {
        float R00 = 1, R01 = 0, R02 = 0, R10 = 0, R11 = 1, R12 = 0, R20 = 0, R21 = 0, R22 = 1;
        float p0 = 0, p1 = 0, p2 = 0;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const float q = wrap_pi(fmaf(s[6 + i], c.dt, s[i]));
            s[i] = q;
            s[6 + i] = fmaf(c.sqd, n[i], s[6 + i]);
            float sq, cq;
            __sincosf(q, &sq, &cq);
            sn[i] = sq;
            cs[i] = cq;
            // A_i = [[c, -s ca, s sa, a c], [s, c ca, -c sa, a s], [0, sa, ca, d]]
            const float a00 = cq, a01 = -(sq * c.ca[i]), a02 = sq * c.sa[i];
            const float a10 = sq, a11 = cq * c.ca[i], a12 = -(cq * c.sa[i]);
            const float a21 = c.sa[i], a22 = c.ca[i];
            const float t0 = c.a[i] * cq, t1 = c.a[i] * sq, t2 = c.d[i];
            const float n00 = fmaf(R01, a10, R00 * a00), n01 = fmaf(R02, a21, fmaf(R01, a11, R00 * a01)),
                        n02 = fmaf(R02, a22, fmaf(R01, a12, R00 * a02));
            const float n10 = fmaf(R11, a10, R10 * a00), n11 = fmaf(R12, a21, fmaf(R11, a11, R10 * a01)),
                        n12 = fmaf(R12, a22, fmaf(R11, a12, R10 * a02));
            const float n20 = fmaf(R21, a10, R20 * a00), n21 = fmaf(R22, a21, fmaf(R21, a11, R20 * a01)),
                        n22 = fmaf(R22, a22, fmaf(R21, a12, R20 * a02));
            p0 = fmaf(R02, t2, fmaf(R01, t1, fmaf(R00, t0, p0)));
            p1 = fmaf(R12, t2, fmaf(R11, t1, fmaf(R10, t0, p1)));
            p2 = fmaf(R22, t2, fmaf(R21, t1, fmaf(R20, t0, p2)));
            R00 = n00; R01 = n01; R02 = n02;
            R10 = n10; R11 = n11; R12 = n12;
            R20 = n20; R21 = n21; R22 = n22;
        }
        const float yaw = pf_atan2(R10, R00);
        const float pitch = pf_atan2(-R20, pf_sqrt(fmaf(R21, R21, R22 * R22)));
        const float roll = pf_atan2(R21, R22);
        const float e0 = (c.z[0] - p0) * c.isp, e1 = (c.z[1] - p1) * c.isp, e2 = (c.z[2] - p2) * c.isp;
        float d3 = c.z[3] - yaw, d4 = c.z[4] - pitch, d5 = c.z[5] - roll;
        d3 = fmaf(-kTwoPi, rintf(d3 * kInvTwoPi), d3) * c.isa;
        d4 = fmaf(-kTwoPi, rintf(d4 * kInvTwoPi), d4) * c.isa;
        d5 = fmaf(-kTwoPi, rintf(d5 * kInvTwoPi), d5) * c.isa;
        float acc = e0 * e0;
        acc = fmaf(e1, e1, acc);
        acc = fmaf(e2, e2, acc);
        acc = fmaf(d3, d3, acc);
        acc = fmaf(d4, d4, acc);
        acc = fmaf(d5, d5, acc);
        return -0.5f * acc;
    }
    // Two threads per particle (lane pair h = 0, 1): both lanes advance all
    // joints (identical arithmetic); lane h chains the transforms of joints
    // 3h .. 3h+2 from the identity, the pair swaps chains and joint sines, and
    // both form the whole chain T = T_0 T_1 (position p_0 + R_0 p_1); lane 0
    // weighs the position and yaw, lane 1 pitch and roll, and the pair adds
    // the two sums in lane order.
    __device__ static __forceinline__ float step_pair(const Consts& c, float* s, const float* n, int h, float* sn,
                                                      float* cs)
    {
        float q[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            q[i] = wrap_pi(fmaf(s[6 + i], c.dt, s[i]));
            s[i] = q[i];
            s[6 + i] = fmaf(c.sqd, n[i], s[6 + i]);
        }
        float R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, p[3] = {0, 0, 0};
        float msn[3], mcs[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int i = 3 * h + k;
            const float qi = h ? q[3 + k] : q[k];
            float sq, cq;
            __sincosf(qi, &sq, &cq);
            msn[k] = sq;
            mcs[k] = cq;
            const float ca = c.ca[i], sa = c.sa[i];
            const float a00 = cq, a01 = -(sq * ca), a02 = sq * sa;
            const float a10 = sq, a11 = cq * ca, a12 = -(cq * sa);
            const float a21 = sa, a22 = ca;
            const float t0 = c.a[i] * cq, t1 = c.a[i] * sq, t2 = c.d[i];
            float N[9];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                N[3 * r + 0] = fmaf(R[3 * r + 1], a10, R[3 * r + 0] * a00);
                N[3 * r + 1] = fmaf(R[3 * r + 2], a21, fmaf(R[3 * r + 1], a11, R[3 * r + 0] * a01));
                N[3 * r + 2] = fmaf(R[3 * r + 2], a22, fmaf(R[3 * r + 1], a12, R[3 * r + 0] * a02));
                p[r] = fmaf(R[3 * r + 2], t2, fmaf(R[3 * r + 1], t1, fmaf(R[3 * r + 0], t0, p[r])));
            }
#pragma unroll
            for (int j = 0; j < 9; ++j) R[j] = N[j];
        }
        float Ro[9], po[3];
#pragma unroll
        for (int j = 0; j < 9; ++j) Ro[j] = __shfl_xor_sync(kFull, R[j], 1);
#pragma unroll
        for (int j = 0; j < 3; ++j) po[j] = __shfl_xor_sync(kFull, p[j], 1);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float os = __shfl_xor_sync(kFull, msn[k], 1), oc = __shfl_xor_sync(kFull, mcs[k], 1);
            sn[k] = h ? os : msn[k];
            cs[k] = h ? oc : mcs[k];
            sn[3 + k] = h ? msn[k] : os;
            cs[3 + k] = h ? mcs[k] : oc;
        }
        const float* A = h ? Ro : R;  // joints 0..2
        const float* B = h ? R : Ro;  // joints 3..5
        const float* pa = h ? po : p;
        const float* pb = h ? p : po;
        float W[9], P[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int col = 0; col < 3; ++col)
                W[3 * r + col] = fmaf(A[3 * r + 2], B[6 + col], fmaf(A[3 * r + 1], B[3 + col], A[3 * r] * B[col]));
            P[r] = fmaf(A[3 * r + 2], pb[2], fmaf(A[3 * r + 1], pb[1], fmaf(A[3 * r], pb[0], pa[r])));
        }
        float acc;
        if (h == 0) {
            const float yaw = pf_atan2(W[3], W[0]);
            const float e0 = (c.z[0] - P[0]) * c.isp, e1 = (c.z[1] - P[1]) * c.isp, e2 = (c.z[2] - P[2]) * c.isp;
            float d3 = c.z[3] - yaw;
            d3 = fmaf(-kTwoPi, rintf(d3 * kInvTwoPi), d3) * c.isa;
            acc = e0 * e0;
            acc = fmaf(e1, e1, acc);
            acc = fmaf(e2, e2, acc);
            acc = fmaf(d3, d3, acc);
        } else {
            const float pitch = pf_atan2(-W[6], pf_sqrt(fmaf(W[7], W[7], W[8] * W[8])));
            const float roll = pf_atan2(W[7], W[8]);
            float d4 = c.z[4] - pitch, d5 = c.z[5] - roll;
            d4 = fmaf(-kTwoPi, rintf(d4 * kInvTwoPi), d4) * c.isa;
            d5 = fmaf(-kTwoPi, rintf(d5 * kInvTwoPi), d5) * c.isa;
            acc = d4 * d4;
            acc = fmaf(d5, d5, acc);
        }
        const float o = __shfl_xor_sync(kFull, acc, 1);
        return -0.5f * (h ? o + acc : acc + o);
    }
};

// The reference's camera robot arm: the planar chain of sampling_iw
// (src/models/robotarm/cuda/pf_model_soa.cuh:114-184): state angles[5], x, y,
// vX, vY; normals in the same variable order.  Propagates the particle in
// place, returns the angle part of the error value (sum 0.1 e^2) and the
// camera coordinates (cx, cy, cz) of the cart in the last link's frame.
struct ArmConsts {
    float dt;
    float cdt[5];
    float z[7];
};

__device__ static void arm_prepare(ArmConsts& c, const pf_step_input& in, float dt_default)
{
    c.dt = in.dt > 0.0f ? in.dt : dt_default;
    for (int i = 0; i < 5; ++i) c.cdt[i] = in.control[i] * c.dt;
    for (int i = 0; i < 7; ++i) c.z[i] = in.meas[i];
}

__device__ __forceinline__ float arm_chain(const ArmConsts& c, float* s, const float* n, float* sn, float* cs,
                                           float& cx, float& cy, float& cz)
{
    const float arm[5] = {0.0f, 3.0f, 3.0f, 3.0f, 3.0f};
    const float vX = s[7], vY = s[8];
    const float x = fmaf(n[5], 0.2f, fmaf(vX, c.dt, s[5]));
    const float y = fmaf(n[6], 0.2f, fmaf(vY, c.dt, s[6]));
    s[5] = x;
    s[6] = y;
    s[7] = fmaf(n[7], 2.0f, vX);
    s[8] = fmaf(n[8], 2.0f, vY);
    float value = 0.0f;
    cx = 0.0f;
    cy = 0.0f;
    cz = 0.0f;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const float ang = fmaf(n[i], 0.2f, s[i] + c.cdt[i]);
        s[i] = ang;
        float sf, cf;
        __sincosf(ang, &sf, &cf);
        sn[i] = sf;
        cs[i] = cf;
        if (i == 0) {
            cx = fmaf(x, cf, y * sf);
            cy = fmaf(-x, sf, y * cf);
            cz = 0.0f;
        } else {
            const float nb = fmaf(cy, cf, -(cz * sf)), nc = fmaf(cy, sf, cz * cf);
            cy = nb;
            cz = nc - arm[i];
        }
        const float e = ang - c.z[i];
        value = fmaf(e * e, 0.1f, value);
    }
    return value;
}

// The reference's camera arm (sampling_iw, pf_model_soa.cuh:114-184): the cart
// position in the camera frame is measured directly; log weight =
// -(sum 0.1 e^2) (the reference returns its exp).
struct RefArm {
    static constexpr int S = 9, K = 9, NA = 5, C = 5, Z = 7;
    __host__ __device__ static constexpr int angle_var(int a) { return a; }
    using Consts = ArmConsts;
    __device__ static void prepare(Consts& c, const pf_step_input& in, const ModelParams& mp, int lane)
    {
        if (lane == 0) arm_prepare(c, in, mp.ref.dt);
    }
    __device__ static __forceinline__ float step(const Consts& c, float* s, const float* n, float* sn,
                                                 float* cs)
    {
        float cx, cy, cz;
        float value = arm_chain(c, s, n, sn, cs, cx, cy, cz);
        value = fmaf((cx - c.z[5]) * (cx - c.z[5]), 0.1f, value);
        value = fmaf((cy - c.z[6]) * (cy - c.z[6]), 0.1f, value);
        return -value;
    }
};

// The reference's pinhole-camera variant of the arm (sampling_iw,
// src/models/robotarm/cuda/pf_model_soa_packed_code.cuh:61-145): the same
// chain, then the cart's camera coordinates are projected, x_n = cx / cz,
// y_n = cy / cz, distorted (radial kc1, kc2; tangential kc3, kc4) and mapped
// to pixels (xp = fc_x xd + cc_x, yp = fc_y yd + cc_y); the measured x, y
// are pixels.  Log weight = -(sum 0.1 e^2).
struct CamArm {
    static constexpr int S = 9, K = 9, NA = 5, C = 5, Z = 7;
    __host__ __device__ static constexpr int angle_var(int a) { return a; }
    struct Consts {
        ArmConsts a;
        float fx, fy, ux, uy, k1, k2, k3, k4;
    };
    __device__ static void prepare(Consts& c, const pf_step_input& in, const ModelParams& mp, int lane)
    {
        if (lane != 0) return;
        const pf_camarm_params& p = mp.cam;
        arm_prepare(c.a, in, p.dt);
        c.fx = p.fc[0];
        c.fy = p.fc[1];
        c.ux = p.cc[0];
        c.uy = p.cc[1];
        c.k1 = p.kc[0];
        c.k2 = p.kc[1];
        c.k3 = p.kc[2];
        c.k4 = p.kc[3];
    }
    __device__ static __forceinline__ float step(const Consts& c, float* s, const float* n, float* sn,
                                                 float* cs)
    {
        float cx, cy, cz;
        float value = arm_chain(c.a, s, n, sn, cs, cx, cy, cz);
        const float xn = cx / cz, yn = cy / cz;
        const float xx = xn * xn, yy = yn * yn, xy = xn * yn;
        const float r2 = xx + yy;
        const float dxx = fmaf(2.0f * c.k3, xy, c.k4 * fmaf(3.0f, xx, yy));
        const float dxy = fmaf(c.k3, fmaf(3.0f, yy, xx), 2.0f * c.k4 * xy);
        const float rad = fmaf(c.k2 * r2, r2, fmaf(c.k1, r2, 1.0f));
        const float xp = fmaf(c.fx, fmaf(rad, xn, dxx), c.ux);
        const float yp = fmaf(c.fy, fmaf(rad, yn, dxy), c.uy);
        value = fmaf((xp - c.a.z[5]) * (xp - c.a.z[5]), 0.1f, value);
        value = fmaf((yp - c.a.z[6]) * (yp - c.a.z[6]), 0.1f, value);
        return -value;
    }
};

// The reference's unicycle program (src/models/unicycle/particle_filter.cu:
// 314-359): noisy velocity and turn rate, arc motion, heading noise gamma,
// weight from the ranges to fixed 3-D beacons.  The arc is evaluated through
//   sin(th + a) - sin th =  2 sin(a/2) cos(th + a/2)
//   cos(th + a) - cos th = -2 sin(a/2) sin(th + a/2),   a = omega dt
// (the same motion, without the cancellation of the difference form when
// a is small, and finite as omega -> 0).  The heading is wrapped to [-pi, pi)
// (the ranges do not depend on it).  Log weight: lnorm - h sum_i e_i^2 with
// h = 1 / (2 sigma_range^2) (1 for the reference's exp(-sum e^2)) and
// lnorm = log(1e5) - (L/2) log(2 pi), the reference's normalisation.
struct Beacon {
    static constexpr int S = 3, K = 3, NA = 1, C = 2, Z = 16;
    __host__ __device__ static constexpr int angle_var(int) { return 2; }
    struct Consts {
        float dt, hdt, v, w, nv, nw, ng, h, lnorm;
        int L;
        float bx[16], by[16], bz2[16], z[16];
    };
    // lane 16: scalars; lanes 0..15: beacon `lane`
    __device__ static void prepare(Consts& c, const pf_step_input& in, const ModelParams& mp, int lane)
    {
        const pf_beacon_params& p = mp.bcn;
        const int L = p.num_beacons < 1 ? 1 : (p.num_beacons > 16 ? 16 : p.num_beacons);
        if (lane == 16) {
            const float dt = in.dt > 0.0f ? in.dt : p.dt;
            c.dt = dt;
            c.hdt = 0.5f * dt;
            c.v = in.control[0];
            c.w = in.control[1];
            c.nv = p.noise[0];
            c.nw = p.noise[1];
            c.ng = p.noise[2];
            c.h = (float)(0.5 / ((double)p.sigma_range * (double)p.sigma_range));
            // log(1e5) - (L/2) log(2 pi), the logarithms as FP64 constants
            c.lnorm = (float)(11.512925464970229 - (double)(L / 2) * 1.8378770664093453);
            c.L = L;
        } else if (lane < 16) {
            const int j = lane;
            c.bx[j] = p.beacons[j][0];
            c.by[j] = p.beacons[j][1];
            c.bz2[j] = p.beacons[j][2] * p.beacons[j][2];
            c.z[j] = j < L ? in.meas[j] : 0.0f;
        }
    }
    // sin(u) / u: the series to u^4 below |u| = 2^-6 (remainder under u^6/5040,
    // below 3e-15), the library sine above it.
    __device__ static __forceinline__ float sinc(float u)
    {
        const float u2 = u * u;
        if (fabsf(u) < 0.015625f) return fmaf(u2, fmaf(u2, 1.0f / 120.0f, -1.0f / 6.0f), 1.0f);
        return sinf(u) / u;
    }
    __device__ static __forceinline__ float step(const Consts& c, float* s, const float* n, float* sn,
                                                 float* cs)
    {
        const float v = fmaf(c.nv, n[0], c.v);
        const float w = fmaf(c.nw, n[1], c.w);
        const float g = c.ng * n[2];
        const float ha = w * c.hdt;  // a / 2
        const float k = v * c.dt * sinc(ha);  // v / w * 2 sin(a/2)
        float sm, cm;
        __sincosf(s[2] + ha, &sm, &cm);
        const float nx = fmaf(k, cm, s[0]);
        const float ny = fmaf(k, sm, s[1]);
        const float nt = wrap_pi(fmaf(g, c.dt, fmaf(w, c.dt, s[2])));
        s[0] = nx;
        s[1] = ny;
        s[2] = nt;
        float s2, c2;
        __sincosf(nt, &s2, &c2);
        sn[0] = s2;
        cs[0] = c2;
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            if (j < c.L) {
                const float dx = nx - c.bx[j], dy = ny - c.by[j];
                const float e = pf_sqrt(fmaf(dx, dx, fmaf(dy, dy, c.bz2[j]))) - c.z[j];
                acc = fmaf(e, e, acc);
            }
        }
        return fmaf(-c.h, acc, c.lnorm);
    }
    // Two threads per particle (lane pair h = 0, 1): both lanes propagate the
    // particle (identical arithmetic), each sums the beacons j = h, h + 2, ...,
    // and the pair adds the two sums in lane order.
    __device__ static __forceinline__ float step_pair(const Consts& c, float* s, const float* n, int h, float* sn,
                                                      float* cs)
    {
        const float v = fmaf(c.nv, n[0], c.v);
        const float w = fmaf(c.nw, n[1], c.w);
        const float g = c.ng * n[2];
        const float ha = w * c.hdt;
        const float k = v * c.dt * sinc(ha);
        float sm, cm;
        __sincosf(s[2] + ha, &sm, &cm);
        const float nx = fmaf(k, cm, s[0]);
        const float ny = fmaf(k, sm, s[1]);
        const float nt = wrap_pi(fmaf(g, c.dt, fmaf(w, c.dt, s[2])));
        s[0] = nx;
        s[1] = ny;
        s[2] = nt;
        __sincosf(nt, &sn[0], &cs[0]);
        float acc = 0.0f;
#pragma unroll 1
        for (int j = h; j < c.L; j += 2) {
            const float dx = nx - c.bx[j], dy = ny - c.by[j];
            const float e = pf_sqrt(fmaf(dx, dx, fmaf(dy, dy, c.bz2[j]))) - c.z[j];
            acc = fmaf(e, e, acc);
        }
        const float o = __shfl_xor_sync(kFull, acc, 1);
        return fmaf(-c.h, h ? o + acc : acc + o, c.lnorm);
    }
    // E particles at once: step()'s per-particle arithmetic in the same order
    // (bit-identical results), the beacon loop outside the particle loop so
    // each beacon's constants are read once per thread and the E range
    // chains interleave.  noise(e, v) gives particle e's v-th normal.
    template <int E, class Noise>
    __device__ static __forceinline__ void step_batch(const Consts& c, float (&s)[E][S], Noise noise,
                                                      float (&sn)[E][NA], float (&cs)[E][NA], float (&ll)[E])
    {
        float acc[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float v = fmaf(c.nv, noise(e, 0), c.v);
            const float w = fmaf(c.nw, noise(e, 1), c.w);
            const float g = c.ng * noise(e, 2);
            const float ha = w * c.hdt;
            const float k = v * c.dt * sinc(ha);
            float sm, cm;
            __sincosf(s[e][2] + ha, &sm, &cm);
            const float nx = fmaf(k, cm, s[e][0]);
            const float ny = fmaf(k, sm, s[e][1]);
            const float nt = wrap_pi(fmaf(g, c.dt, fmaf(w, c.dt, s[e][2])));
            s[e][0] = nx;
            s[e][1] = ny;
            s[e][2] = nt;
            __sincosf(nt, &sn[e][0], &cs[e][0]);
            acc[e] = 0.0f;
        }
        const int L = c.L;
#pragma unroll 1
        for (int j = 0; j < L; ++j) {
            const float bx = c.bx[j], by = c.by[j], bz2 = c.bz2[j], z = c.z[j];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const float dx = s[e][0] - bx, dy = s[e][1] - by;
                const float r = pf_sqrt(fmaf(dx, dx, fmaf(dy, dy, bz2))) - z;
                acc[e] = fmaf(r, r, acc[e]);
            }
        }
#pragma unroll
        for (int e = 0; e < E; ++e) ll[e] = fmaf(-c.h, acc[e], c.lnorm);
    }
};

template <class Mdl>
__host__ __device__ constexpr bool is_angle_var(int v)
{
    for (int i = 0; i < Mdl::NA; ++i)
        if (Mdl::angle_var(i) == v) return true;
    return false;
}


// E particles of a model at once: Mdl::step_batch when the model has one,
// otherwise step() particle by particle.  noise(e, v): particle e's v-th normal.
template <class Mdl, class = void>
struct HasStepBatch : std::false_type {};
template <class Mdl>
struct HasStepBatch<Mdl, std::void_t<decltype(&Mdl::template step_batch<1, float (*)(int, int)>)>> : std::true_type {};

template <class Mdl, int E, class Noise>
__device__ __forceinline__ void model_step_batch(const typename Mdl::Consts& c, float (&s)[E][Mdl::S], Noise noise,
                                                 float (&sn)[E][Mdl::NA > 0 ? Mdl::NA : 1],
                                                 float (&cs)[E][Mdl::NA > 0 ? Mdl::NA : 1], float (&ll)[E])
{
    if constexpr (HasStepBatch<Mdl>::value) {
        Mdl::template step_batch<E>(c, s, noise, sn, cs, ll);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            float n[Mdl::K];
#pragma unroll
            for (int v = 0; v < Mdl::K; ++v) n[v] = noise(e, v);
            ll[e] = Mdl::step(c, s[e], n, sn[e], cs[e]);
        }
    }
}

// Two threads per particle (TP = 2, lane pair h = lane & 1, both lanes
// holding the same E particles): models with step_pair split each particle's
// work between the pair; others run model_step_batch on both lanes, which
// compute identical results.
template <class Mdl, class = void>
struct HasStepPair : std::false_type {};
template <class Mdl>
struct HasStepPair<Mdl, std::void_t<decltype(&Mdl::step_pair)>> : std::true_type {};

template <class Mdl, int E, int TP, class Noise>
__device__ __forceinline__ void model_step_tp(const typename Mdl::Consts& c, float (&s)[E][Mdl::S], Noise noise,
                                              int h, float (&sn)[E][Mdl::NA > 0 ? Mdl::NA : 1],
                                              float (&cs)[E][Mdl::NA > 0 ? Mdl::NA : 1], float (&ll)[E])
{
    if constexpr (TP == 2 && HasStepPair<Mdl>::value) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            float n[Mdl::K];
#pragma unroll
            for (int v = 0; v < Mdl::K; ++v) n[v] = noise(e, v);
            ll[e] = Mdl::step_pair(c, s[e], n, h, sn[e], cs[e]);
        }
    } else {
        model_step_batch<Mdl, E>(c, s, noise, sn, cs, ll);
    }
}

// Models whose weights are continuous functions of a state that every step
// perturbs in every variable the weight depends on: two particles share a key
// only by coincidence, so their sub-filters sort with rank_sort_desc.  The
// DH arm is not one (a resampled duplicate's joint angles advance with the
// velocity of the previous step, before its noise, so duplicates keep equal
// keys), nor, conservatively, are the reference's arms.
template <class Mdl>
struct RareTies : std::false_type {};
template <>
struct RareTies<Unicycle> : std::true_type {};
template <>
struct RareTies<Beacon> : std::true_type {};

// The sampling kernels' sort of one sub-filter per CTA (see rank_sort_desc).
template <class Mdl, int M, int E, int TP = 1>
__device__ __forceinline__ void sort_subfilter(float (&k)[E], int (&ix)[E], float* sk, int* si)
{
    if constexpr (RareTies<Mdl>::value) {
        rank_sort_desc<M, E, TP>(k, ix, sk, si);
    } else {
        bitonic_sort_desc<M, E, TP>(k, ix, sk, si, threadIdx.x / TP, threadIdx.x % TP == 0);
    }
}

}  // namespace pfdev
