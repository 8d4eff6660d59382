// Model-independent launchers: RNG in the reference layout, Box-Muller,
// all-to-all merge, and the kernel-level test entry points.
#include "pf_launch.cuh"

namespace pfdev {

// Slot sources of every sub-filter (identity where no particle arrives).
__global__ void k_exchange_sources(const FilterDesc* __restrict__ d, int32_t* __restrict__ src)
{
    const FilterDesc& D = *d;
    const int b = blockIdx.x;
    const int nx = exchange_count(D);
    for (int s = threadIdx.x; s < D.M; s += blockDim.x) {
        const int x = D.M - 1 - s;
        src[(int64_t)b * D.M + s] = (int32_t)(x < nx ? exchange_source(D, b, x) : (int64_t)b * D.M + s);
    }
}

// All-to-all: the t best of all sub-filters' sorted top-t lists, ties to the
// lower (sub-filter, rank) -- a stable descending sort of the candidates, as
// thrust::sort_by_key(greater) gives (pf_generic2_all2all.cu:1007).
__global__ void k_a2a_merge(const FilterDesc* __restrict__ descs)
{
    const FilterDesc& D = descs[blockIdx.x];
    constexpr int R = 8;  // sub-filters per thread (N <= 8 * blockDim)
    __shared__ float sk[32];
    __shared__ int so[32];
    __shared__ int s_win;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wp = tid >> 5;
    int head[R];
#pragma unroll
    for (int r = 0; r < R; ++r) head[r] = 0;
    for (int j = 0; j < D.t; ++j) {
        float bk = -INFINITY;
        int bo = 0x7fffffff;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int sb = tid + r * nt;
            if (sb < D.N && head[r] < D.t) {
                const float kk = D.tkey[(int64_t)sb * D.M + head[r]];
                const int ord = sb * D.t + head[r];
                if (kk > bk || (kk == bk && ord < bo)) {
                    bk = kk;
                    bo = ord;
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float ok = __shfl_xor_sync(kFull, bk, o);
            const int oo = __shfl_xor_sync(kFull, bo, o);
            if (ok > bk || (ok == bk && oo < bo)) {
                bk = ok;
                bo = oo;
            }
        }
        if (lane == 0) {
            sk[wp] = bk;
            so[wp] = bo;
        }
        __syncthreads();
        if (tid == 0) {
            float k2 = sk[0];
            int o2 = so[0];
            for (int w = 1; w < nt / 32; ++w)
                if (sk[w] > k2 || (sk[w] == k2 && so[w] < o2)) {
                    k2 = sk[w];
                    o2 = so[w];
                }
            if (o2 == 0x7fffffff) o2 = j < D.t ? j : 0;  // only NaN keys left: take sub-filter 0's slot
            s_win = o2;
            const int sbw = o2 / D.t, rank = o2 - sbw * D.t;
            D.a2a[j] = sbw * D.M + rank;
        }
        __syncthreads();
        const int win = s_win;
        const int sbw = win / D.t;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (tid + r * nt == sbw) head[r]++;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// RNG in the reference block layout.
// ---------------------------------------------------------------------------
// Stream g (parameter set g % 200) writes out[g*size + i] (mtgp32_single_kernel).
__global__ void __launch_bounds__(256) k_mtgp_blocks(uint32_t* __restrict__ states, uint32_t* __restrict__ out,
                                                     int64_t size, uint32_t mask, int float_out, int set_base)
{
    __shared__ MtgpSmem ms;
    const int g = blockIdx.x;
    uint32_t* gst = states + (int64_t)g * kMtgpN;
    mtgp_load(ms, gst, (set_base + g) % kMtgpSets, mask, float_out != 0);
    uint32_t* o = out + (int64_t)g * size;
    // size may exceed INT_MAX only in absurd configurations; the host bounds it.
    mtgp_generate(ms, (int)size, float_out != 0, [&](int k, uint32_t w) { o[k] = w; });
    mtgp_store(ms, gst, (int)size);
}

// In-place Box-Muller over pairs (2i, 2i+1) with 2i < n.
__global__ void k_boxmuller(float* __restrict__ data, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * i < n) {
        float2 v = reinterpret_cast<float2*>(data)[i];
        float z1, z2;
        box_muller(v.x, v.y, z1, z2);
        reinterpret_cast<float2*>(data)[i] = make_float2(z1, z2);
    }
}

// All-to-all winners of the half written by the last step (k_a2a_merge on a
// double-buffered key array).
__global__ void k_a2a_merge_step(const FilterDesc* __restrict__ descs, StepState X)
{
    __shared__ FilterDesc Dl;
    if (threadIdx.x == 0) {
        Dl = descs[0];
        if (((*X.steps) & 1) ^ 1) Dl.tkey = X.tkey2;
    }
    __syncthreads();
    const FilterDesc& D = Dl;
    constexpr int R = 8;
    __shared__ float sk[32];
    __shared__ int so[32];
    __shared__ int s_win;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wp = tid >> 5;
    int head[R];
#pragma unroll
    for (int r = 0; r < R; ++r) head[r] = 0;
    for (int j = 0; j < D.t; ++j) {
        float bk = -INFINITY;
        int bo = 0x7fffffff;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int sb = tid + r * nt;
            if (sb < D.N && head[r] < D.t) {
                const float kk = D.tkey[(int64_t)sb * D.M + head[r]];
                const int ord = sb * D.t + head[r];
                if (kk > bk || (kk == bk && ord < bo)) {
                    bk = kk;
                    bo = ord;
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float ok = __shfl_xor_sync(kFull, bk, o);
            const int oo = __shfl_xor_sync(kFull, bo, o);
            if (ok > bk || (ok == bk && oo < bo)) {
                bk = ok;
                bo = oo;
            }
        }
        if (lane == 0) {
            sk[wp] = bk;
            so[wp] = bo;
        }
        __syncthreads();
        if (tid == 0) {
            float k2 = sk[0];
            int o2 = so[0];
            for (int w = 1; w < nt / 32; ++w)
                if (sk[w] > k2 || (sk[w] == k2 && so[w] < o2)) {
                    k2 = sk[w];
                    o2 = so[w];
                }
            if (o2 == 0x7fffffff) o2 = j < D.t ? j : 0;
            s_win = o2;
            const int sbw = o2 / D.t, rank = o2 - sbw * D.t;
            D.a2a[j] = sbw * D.M + rank;
        }
        __syncthreads();
        const int sbw = s_win / D.t;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (tid + r * nt == sbw) head[r]++;
        __syncthreads();
    }
}


cudaError_t launch_test_sort(int M, int E, int nsub, float* keys, int32_t* idx, int rank, int32_t* fallbacks,
                             cudaStream_t st)
{
#define PF_TS(m, e)                                                                  \
    if (M == m && E == e) {                                                          \
        if (rank) k_test_sort<m, e, true><<<nsub, m / e, 0, st>>>(keys, idx, fallbacks); \
        else k_test_sort<m, e, false><<<nsub, m / e, 0, st>>>(keys, idx, fallbacks);    \
        return cudaGetLastError();                                                   \
    }
    PF_ME_LIST(PF_TS)
#undef PF_TS
    return cudaErrorInvalidValue;
}

template <int RES>
static cudaError_t test_resample_res(int M, int E, int nsub, const float* w, const float* u, int32_t* sel,
                                     float* prob, uint32_t* alias, cudaStream_t st)
{
#define PF_TR(m, e)                                                                          \
    if (M == m && E == e) {                                                                  \
        constexpr size_t sm = RES == PF_RESAMPLE_SYSTEMATIC ? (size_t)m * 12                 \
                            : (RES == PF_RESAMPLE_REFERENCE ? (size_t)m * 4 : (size_t)m * 16); \
        k_test_resample<m, e, RES><<<nsub, m / e, sm, st>>>(w, u, sel, prob, alias);         \
        return cudaGetLastError();                                                           \
    }
    PF_ME_LIST(PF_TR)
#undef PF_TR
    return cudaErrorInvalidValue;
}

cudaError_t launch_test_resample(int res, int M, int E, int nsub, const float* w, const float* u, int32_t* sel,
                                 float* prob, uint32_t* alias, cudaStream_t st)
{
    if (res == PF_RESAMPLE_SYSTEMATIC)
        return test_resample_res<PF_RESAMPLE_SYSTEMATIC>(M, E, nsub, w, u, sel, prob, alias, st);
    if (res == PF_RESAMPLE_REFERENCE)
        return test_resample_res<PF_RESAMPLE_REFERENCE>(M, E, nsub, w, u, sel, prob, alias, st);
    return test_resample_res<PF_RESAMPLE_VOSE>(M, E, nsub, w, u, sel, prob, alias, st);
}

cudaError_t launch_mtgp_blocks(int G, uint32_t* states, uint32_t* out, int64_t size, uint32_t mask, int float_out,
                               int set_base, cudaStream_t st)
{
    k_mtgp_blocks<<<G, 256, 0, st>>>(states, out, size, mask, float_out, set_base);
    return cudaGetLastError();
}

// MTGP32 stream initialisation (mtgp32_init_state, mtgp32-fast.c:119-137), one
// thread per stream: stream i gets parameter set (g0 + i) mod 200 and seed
// seed + g0 + i + 1 -- the words the host-side initialisation writes.
__global__ void k_mtgp_init(uint32_t* __restrict__ states, int n, int g0, uint32_t seed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int g = g0 + i;
    const uint32_t* tbl = g_mtgp_params + (g % kMtgpSets) * 52 + 4;
    const uint32_t hidden = tbl[4] ^ (tbl[8] << 16);
    uint32_t t = hidden;
    t += t >> 16;
    t += t >> 8;
    const uint32_t b = t & 0xffu;
    const uint32_t fill = b | (b << 8) | (b << 16) | (b << 24);
    uint32_t* st = states + (int64_t)i * kMtgpN;
    uint32_t prev = seed + (uint32_t)g + 1u;
    st[0] = prev;
    // word 0 is the seed; word k >= 1 is (k == 1 ? hidden : fill) xor'ed with
    // 1812433253 * (w ^ (w >> 30)) + k of its predecessor w
    for (int k = 1; k < kMtgpN; ++k) {
        const uint32_t w = (k == 1 ? hidden : fill) ^ (1812433253u * (prev ^ (prev >> 30)) + (uint32_t)k);
        st[k] = w;
        prev = w;
    }
}

cudaError_t launch_mtgp_init(uint32_t* states, int n, int g0, uint32_t seed, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_mtgp_init<<<(n + 127) / 128, 128, 0, st>>>(states, n, g0, seed);
    return cudaGetLastError();
}

cudaError_t launch_boxmuller(float* data, int64_t n, cudaStream_t st)
{
    const int64_t pairs = (n + 1) / 2;
    if (pairs == 0) return cudaSuccess;
    k_boxmuller<<<(unsigned)((pairs + 255) / 256), 256, 0, st>>>(data, n);
    return cudaGetLastError();
}

cudaError_t launch_a2a_merge(int nfilters, const FilterDesc* d, cudaStream_t st)
{
    k_a2a_merge<<<nfilters, 1024, 0, st>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_exchange_sources(const FilterDesc* d, int32_t* src, cudaStream_t st)
{
    FilterDesc h;
    cudaError_t e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    k_exchange_sources<<<h.N, 256, 0, st>>>(d, src);
    return cudaGetLastError();
}

cudaError_t launch_a2a_merge_step(const FilterDesc* d, const StepState& X, cudaStream_t st)
{
    k_a2a_merge_step<<<1, 1024, 0, st>>>(d, X);
    return cudaGetLastError();
}

// The bounded mbarrier wait of the resampling kernels on a phase that nothing
// completes (initialised for one arrival that never comes): the wait gives up
// after `limit` polls and the kernel reports PF_STATUS_WAIT_TIMEOUT in *status.
__global__ void k_test_bounded_wait(int limit, int32_t* status)
{
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)) : "memory");
    __syncthreads();
    const bool ok = mbar_wait(&mbar, 0, limit);
    if (threadIdx.x == 0) *status = ok ? 0 : PF_STATUS_WAIT_TIMEOUT;
}

cudaError_t launch_test_bounded_wait(int limit, int32_t* status, cudaStream_t st)
{
    k_test_bounded_wait<<<1, 32, 0, st>>>(limit, status);
    return cudaGetLastError();
}

// The CTA-wide wait of the resampling kernels (mbar_wait_cta) with a bulk copy
// really in flight and a poll limit per thread from the host (limits[tid]; 0:
// the thread gives up at once, so some threads run out while others see the
// copy land).  outcome[tid] receives each thread's result (1, 0 or -1; the
// same in every thread when the decision is CTA-wide); *copied is 1 when the
// shared-memory words equal the source once the CTA went on (the copy landed
// before anyone moved on), 0 when they differ, -1 when the outcome was -1.
constexpr int kMixedWaitBytes = 32768;
__global__ void k_test_bounded_wait_mixed(const int32_t* __restrict__ limits, const uint4* __restrict__ src,
                                          int32_t* __restrict__ outcome, int32_t* __restrict__ copied)
{
    __shared__ __align__(128) uint4 buf[kMixedWaitBytes / 16];
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) {
        mbar_init_expect(&mbar, kMixedWaitBytes);
        bulk_g2s(buf, src, kMixedWaitBytes, &mbar);
    }
    __syncthreads();  // the mbarrier is initialised
    const int r = mbar_wait_cta(&mbar, 0, limits[threadIdx.x], kBulkDrainPolls);
    outcome[threadIdx.x] = r;
    if (r < 0) {
        if (threadIdx.x == 0) *copied = -1;
        return;
    }
    int bad = 0;
    for (int i = threadIdx.x; i < kMixedWaitBytes / 16; i += blockDim.x) {
        const uint4 a = buf[i], b = src[i];
        bad |= (a.x != b.x) | (a.y != b.y) | (a.z != b.z) | (a.w != b.w);
    }
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) *copied = bad ? 0 : 1;
}

cudaError_t launch_test_bounded_wait_mixed(const int32_t* limits, int nthreads, const void* src, int32_t* outcome,
                                           int32_t* copied, cudaStream_t st)
{
    k_test_bounded_wait_mixed<<<1, nthreads, 0, st>>>(limits, static_cast<const uint4*>(src), outcome, copied);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Shards (pf_shard_*): the halo export of a step and the group rows.
// ---------------------------------------------------------------------------
// The sorted top t of the shard's last row (block 0, the shard below takes it
// as its top halo) and first row (block 1, the shard above's bottom halo):
// out[h][1+S][dx*t], key row then state rows, slot x*t + j of row sub-filter x.
__global__ void k_shard_pack(const FilterDesc* __restrict__ descs, float* __restrict__ out, int S)
{
    const FilterDesc& D = descs[0];
    const int P = D.dx * D.t, rows = D.N / D.dx;
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < 2 * P; i += blockDim.x * gridDim.x) {
        const int h = i / P, idx = i - h * P, x = idx / D.t, j = idx - x * D.t;
        const int b = (h == 0 ? rows - 1 : 0) * D.dx + x;
        const int64_t g = (int64_t)b * D.M + j;
        float* o = out + (int64_t)h * (1 + S) * P + idx;
        o[0] = D.tkey[g];
        for (int v = 0; v < S; ++v) o[(int64_t)(1 + v) * P] = D.tmp[v * D.T + g];
    }
}

cudaError_t launch_shard_pack(const FilterDesc* d, float* out, int S, int P, cudaStream_t st)
{
    k_shard_pack<<<(2 * P + 255) / 256, 256, 0, st>>>(d, out, S);
    return cudaGetLastError();
}

// Each local group's partial row (kPartStride doubles, its winner as a
// filter-wide index) and that winner's state (the best slot of the winning
// sub-filter).
__global__ void k_shard_rows(const FilterDesc* __restrict__ descs, double* __restrict__ rows, float* __restrict__ states,
                             int S, int NV)
{
    const FilterDesc& D = descs[0];
    const int g = blockIdx.x;
    const double* r = D.gpart + (int64_t)g * kPartStride;
    for (int j = threadIdx.x; j < kPartStride; j += blockDim.x) rows[(int64_t)g * kPartStride + j] = r[j];
    const int b = (int)r[NV + 1] - D.b0;
    for (int v = threadIdx.x; v < S; v += blockDim.x) states[(int64_t)g * S + v] = D.tmp[v * D.T + (int64_t)b * D.M];
}

cudaError_t launch_shard_rows(const FilterDesc* d, int ng, double* rows, float* states, int S, int NV, cudaStream_t st)
{
    k_shard_rows<<<ng, 32, 0, st>>>(d, rows, states, S, NV);
    return cudaGetLastError();
}

// The filter-wide estimate from every shard's group rows, in group order (the
// same combination as a whole filter's last group makes): D.gpart holds the
// rows, best_src[v * D.T + b] the winner states at their sub-filter b.
template <int S>
__global__ void k_shard_estimate(FilterDesc D, const float* __restrict__ best_src, pf_estimate* out, int ng,
                                 int32_t step_no)
{
    if (threadIdx.x >= 32) return;
    estimate_final<S>(D, threadIdx.x, ng, 2 + S + D.na, best_src, *out, step_no);
}

cudaError_t launch_shard_estimate(const FilterDesc& D, int S, const float* best_src, pf_estimate* out, int ng,
                                  int32_t step_no, cudaStream_t st)
{
#define PF_SE(s)                                                                 \
    if (S == s) {                                                                \
        k_shard_estimate<s><<<1, 32, 0, st>>>(D, best_src, out, ng, step_no);    \
        return cudaGetLastError();                                               \
    }
    PF_SE(1) PF_SE(2) PF_SE(3) PF_SE(4) PF_SE(5) PF_SE(6) PF_SE(7) PF_SE(8)
    PF_SE(9) PF_SE(10) PF_SE(11) PF_SE(12) PF_SE(13) PF_SE(14) PF_SE(15) PF_SE(16)
#undef PF_SE
    return cudaErrorInvalidValue;
}

// A run's device step counter, advanced (or set) by a launch of its own once
// every kernel of the step that reads it is enqueued before it.
__global__ void k_counter_update(int32_t* ctr, int32_t set, int32_t value)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *ctr = set ? value : *ctr + 1;
}

cudaError_t launch_counter_inc(int32_t* ctr, cudaStream_t st)
{
    k_counter_update<<<1, 32, 0, st>>>(ctr, 0, 0);
    return cudaGetLastError();
}

cudaError_t launch_counter_set(int32_t* ctr, int32_t value, cudaStream_t st)
{
    k_counter_update<<<1, 32, 0, st>>>(ctr, 1, value);
    return cudaGetLastError();
}

}  // namespace pfdev
