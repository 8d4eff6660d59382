// ref_kernels_harness.cu -- test infrastructure only: a C-ABI around the
// reference's OWN CUDA kernels for the sort, the multinomial resampling, the
// ring exchange and the robot-arm propagate + weight (block_sort, resampling,
// exchange_ring with its bitonic_sort, prefix_sum and binary_search,
// sampling_importance: src/partfilt/cuda/pf_generic_soa.cu:169-323, 400-453 and
// bitonic-sort.cu:11-61; the robot-arm model's types and sampling_iw,
// src/models/robotarm/cuda/pf_model_soa.cuh:33-184), so that the engine's
// kernels and the CPU oracle can be checked against the reference itself on a
// GPU.  Built by oracle/build_ref_kernels.sh straight from the reference tree
// (its main() renamed) into oracle/_ref/; the reference sources are not copied.
//
// The reference kernels move particles with particle_set(); the harness
// stores each particle's own index in the model's `x` variable, so the moved
// `x` values give the permutation / selection / routing directly.  The
// cuRAND build of the reference is used: its uniforms are in [0,1), the MTGP
// build's are the same values + 1 (it subtracts the 1 back,
// pf_generic_soa.cu:424, 442).
#include <vector>

#include "pf_generic_soa.cu"

namespace {

struct Soa {
    state_data d{};
    float* base = nullptr;
    int64_t T = 0;
    bool alloc(int64_t t)
    {
        T = t;
        if (cudaMalloc(&base, sizeof(float) * (size_t)T * NUM_STATE_VARIABLES) != cudaSuccess) return false;
        d.angles = base;
        d.x = base + NUM_ANGLES * T;
        d.y = d.x + T;
        d.vX = d.y + T;
        d.vY = d.vX + T;
        return true;
    }
    ~Soa()
    {
        if (base) cudaFree(base);
    }
    // x[i] = i (or -1), everything else 0
    bool fill_index(bool minus_one)
    {
        std::vector<float> h((size_t)T * NUM_STATE_VARIABLES, 0.0f);
        for (int64_t i = 0; i < T; ++i) h[(size_t)(NUM_ANGLES * T + i)] = minus_one ? -1.0f : (float)i;
        return cudaMemcpy(base, h.data(), h.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    bool read_x(int32_t* out)
    {
        std::vector<float> h((size_t)T);
        if (cudaMemcpy(h.data(), d.x, (size_t)T * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
        for (int64_t i = 0; i < T; ++i) out[i] = (int32_t)h[(size_t)i];
        return true;
    }
};

struct Buf {
    void* p = nullptr;
    ~Buf()
    {
        if (p) cudaFree(p);
    }
};

}  // namespace

// nsub descending sorts of m keys by the reference's block_sort (m/2 threads per
// block): keys sorted in place, perm[i] = the source slot (within the sub-filter).
extern "C" int ref_block_sort(float* keys, int m, int nsub, int32_t* perm)
{
    if (m < 2 || m > MAX_NUM_PARTICLES || (m & (m - 1)) || nsub < 1) return 1;
    const int64_t T = (int64_t)m * nsub;
    Soa src, dst;
    Buf w, win;
    if (!src.alloc(T) || !dst.alloc(T) || !src.fill_index(false) || !dst.fill_index(true)) return 2;
    if (cudaMalloc(&w.p, (size_t)T * 4) != cudaSuccess || cudaMalloc(&win.p, (size_t)nsub * 4) != cudaSuccess) return 2;
    if (cudaMemcpy(w.p, keys, (size_t)T * 4, cudaMemcpyHostToDevice) != cudaSuccess) return 2;
    block_sort<<<nsub, m / 2>>>(dst.d, (float*)w.p, src.d, m, (float*)win.p);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    if (cudaMemcpy(keys, w.p, (size_t)T * 4, cudaMemcpyDeviceToHost) != cudaSuccess || !dst.read_x(perm)) return 2;
    for (int64_t i = 0; i < T; ++i) perm[i] -= (int32_t)((i / m) * m);
    return 0;
}

// The reference's resampling over nsub sub-filters of m weights: random[T + b]
// is sub-filter b's decision uniform, random[i] particle i's, all in [0,1).
// sel[i] = the selected slot within the sub-filter, or -1 where the
// sub-filter skipped (decision uniform > freq).
extern "C" int ref_resampling(const float* weights, const float* random, int m, int nsub, float freq, int32_t* sel)
{
    if (m < 2 || m > MAX_NUM_PARTICLES || (m & (m - 1)) || nsub < 1) return 1;
    const int64_t T = (int64_t)m * nsub;
    Soa data, tmp;
    Buf w, r;
    if (!data.alloc(T) || !tmp.alloc(T) || !data.fill_index(true) || !tmp.fill_index(false)) return 2;
    if (cudaMalloc(&w.p, (size_t)T * 4) != cudaSuccess || cudaMalloc(&r.p, (size_t)(T + nsub) * 4) != cudaSuccess)
        return 2;
    if (cudaMemcpy(w.p, weights, (size_t)T * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(r.p, random, (size_t)(T + nsub) * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return 2;
    resampling<<<nsub, m>>>(data.d, tmp.d, (const float*)w.p, (const float*)r.p, m, freq);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    if (!data.read_x(sel)) return 2;
    for (int64_t i = 0; i < T; ++i)
        if (sel[i] >= 0) sel[i] -= (int32_t)((i / m) * m);
    return 0;
}

// The reference's exchange_ring with t particles: src[i] = the global slot that
// slot i holds afterwards (identity where nothing arrived); keys are moved too.
extern "C" int ref_exchange_ring(float* keys, int m, int nsub, int t, int32_t* src)
{
    if (m < 2 || m > MAX_NUM_PARTICLES || nsub < 1 || t < 1 || 2 * t > m) return 1;
    const int64_t T = (int64_t)m * nsub;
    Soa data;
    Buf w;
    if (!data.alloc(T) || !data.fill_index(false)) return 2;
    if (cudaMalloc(&w.p, (size_t)T * 4) != cudaSuccess) return 2;
    if (cudaMemcpy(w.p, keys, (size_t)T * 4, cudaMemcpyHostToDevice) != cudaSuccess) return 2;
    exchange_ring<<<nsub, t>>>(data.d, (float*)w.p, m, nsub);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    if (cudaMemcpy(keys, w.p, (size_t)T * 4, cudaMemcpyDeviceToHost) != cudaSuccess || !data.read_x(src)) return 2;
    return 0;
}

// The reference's sampling_importance (robot-arm sampling_iw, pf_model_soa.cuh:
// 114-184) over n particles: state SoA [9][n] in/out (angles[5], x, y, vX, vY),
// normals [9][n] (the same variable-major layout), control angle rates [5],
// measurement (angles[5], x, y); weights[n] receives the linear weights.
extern "C" int ref_sampling_importance(float* state, const float* normals, const float* control7,
                                       const float* meas7, float dt, int n, float* weights)
{
    if (n < 1 || n % 64) return 1;
    Soa data;
    Buf w, r;
    if (!data.alloc(n)) return 2;
    if (cudaMalloc(&w.p, (size_t)n * 4) != cudaSuccess || cudaMalloc(&r.p, (size_t)n * 9 * 4) != cudaSuccess) return 2;
    if (cudaMemcpy(data.base, state, (size_t)n * 9 * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(r.p, normals, (size_t)n * 9 * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return 2;
    control c;
    measurement z;
    for (int i = 0; i < NUM_ANGLES; ++i) {
        c.angles[i] = control7[i];
        z.angles[i] = meas7[i];
    }
    z.x = meas7[5];
    z.y = meas7[6];
    sampling_importance<<<n / 64, 64>>>(data.d, (float*)w.p, c, z, (const float*)r.p, dt);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    if (cudaMemcpy(state, data.base, (size_t)n * 9 * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(weights, w.p, (size_t)n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return 2;
    return 0;
}
