// ref_camarm_harness.cu -- test infrastructure only: a C-ABI around the
// reference's OWN pinhole-camera arm model (sampling_iw with its calibration
// and arm lengths, src/models/robotarm/cuda/pf_model_soa_packed_code.cuh:33-145,
// types from pf_model_soa_packed_data.h), so that the engine's camera-arm model
// can be checked against the reference itself on a GPU.  Built by
// oracle/build_ref_camarm.sh straight from the reference tree into
// oracle/_ref/; the reference sources are not copied.  The wrapper kernel
// below only calls the reference's sampling_iw once per particle (its drivers
// pf_generic2*.cu, which call it, do not compile).
#include <vector>

#include "pf_model_soa_packed_code.cuh"

__global__ void harness_sampling_iw(state_data d, control c, measurement z, const float* rnd, float dt, float* w)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    w[idx] = sampling_iw(d, c, z, rnd, dt);
}

// n particles (a multiple of 256), state SoA (9 x n: angles[5], x, y, vX, vY),
// normals SoA (9 x n, the same variable order), controls[5], meas[7]
// (angles[5], pixel x, pixel y).  Returns 0 on success.
extern "C" int ref_camarm_sampling(const float* state, const float* normals, const float* controls,
                                   const float* meas, float dt, int n, float* state_out, float* weight_out)
{
    if (n < 256 || n % 256) return 1;
    std::vector<float4> a1((size_t)n), ps((size_t)n);
    std::vector<float> a2((size_t)n);
    for (int i = 0; i < n; ++i) {
        a1[(size_t)i] = make_float4(state[i], state[n + i], state[2 * n + i], state[3 * n + i]);
        a2[(size_t)i] = state[4 * n + i];
        ps[(size_t)i] = make_float4(state[5 * n + i], state[6 * n + i], state[7 * n + i], state[8 * n + i]);
    }
    float4 *da1 = nullptr, *dps = nullptr;
    float *da2 = nullptr, *dr = nullptr, *dw = nullptr;
    int rc = 2;
    if (cudaMalloc(&da1, sizeof(float4) * n) == cudaSuccess && cudaMalloc(&dps, sizeof(float4) * n) == cudaSuccess &&
        cudaMalloc(&da2, sizeof(float) * n) == cudaSuccess && cudaMalloc(&dr, sizeof(float) * 9 * n) == cudaSuccess &&
        cudaMalloc(&dw, sizeof(float) * n) == cudaSuccess &&
        cudaMemcpy(da1, a1.data(), sizeof(float4) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(dps, ps.data(), sizeof(float4) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(da2, a2.data(), sizeof(float) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(dr, normals, sizeof(float) * 9 * n, cudaMemcpyHostToDevice) == cudaSuccess) {
        state_data d;
        d.angles1 = da1;
        d.angles2 = da2;
        d.pos = dps;
        control c;
        measurement z;
        for (int i = 0; i < NUM_ANGLES; ++i) {
            c.angles[i] = controls[i];
            z.angles[i] = meas[i];
        }
        z.x = meas[5];
        z.y = meas[6];
        harness_sampling_iw<<<n / 256, 256>>>(d, c, z, dr, dt, dw);
        if (cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
            cudaMemcpy(a1.data(), da1, sizeof(float4) * n, cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(a2.data(), da2, sizeof(float) * n, cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(ps.data(), dps, sizeof(float4) * n, cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(weight_out, dw, sizeof(float) * n, cudaMemcpyDeviceToHost) == cudaSuccess) {
            for (int i = 0; i < n; ++i) {
                const float4 a = a1[(size_t)i], p = ps[(size_t)i];
                const float v[9] = {a.x, a.y, a.z, a.w, a2[(size_t)i], p.x, p.y, p.z, p.w};
                for (int k = 0; k < 9; ++k) state_out[(size_t)k * n + i] = v[k];
            }
            rc = 0;
        }
    }
    cudaFree(da1);
    cudaFree(dps);
    cudaFree(da2);
    cudaFree(dr);
    cudaFree(dw);
    return rc;
}
