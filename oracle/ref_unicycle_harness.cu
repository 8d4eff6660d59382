// ref_unicycle_harness.cu -- test infrastructure only: a C-ABI around the
// reference unicycle program's OWN propagate + weight kernel
// (sampling_importance with sampling and importance_weight,
// src/models/unicycle/particle_filter.cu:314-455, its fixed beacons and
// noise constants :60-76), so that the engine's beacon model can be checked
// against the reference itself on a GPU.  Built by oracle/build_ref_unicycle.sh
// straight from the reference tree (its main() renamed, cuRAND build, the
// legacy cutil.h replaced by oracle/cutil_shim/cutil.h) into oracle/_ref/;
// the reference sources are not copied.
//
// The kernel is launched with one particle per block (num_particles = 1), so
// its in-block sort and max/min search are no-ops and every particle comes
// back in place: state out and linear weight (norm * expf(-value)) per particle.
#include <vector>

#include "particle_filter.cu"

// n particles, state SoA (x[n], y[n], theta[n]), normals SoA (3 x n, particle
// i's draws at i, n + i, 2n + i), ten range measurements.  Returns 0 on success.
extern "C" int ref_unicycle_sampling(const float* state, const float* normals, float v, float w, float dt,
                                     const float* ranges, int n, float* state_out, float* weight_out)
{
    if (n < 1) return 1;
    std::vector<robot_state> h((size_t)n);
    std::vector<float> r((size_t)3 * n);
    for (int i = 0; i < n; ++i) {
        h[(size_t)i].x = state[i];
        h[(size_t)i].y = state[n + i];
        h[(size_t)i].theta = state[2 * n + i];
        for (int k = 0; k < 3; ++k) r[(size_t)3 * i + k] = normals[(size_t)k * n + i];  // the program's d_random[3 idx + k]
    }
    robot_state *dp = nullptr, *dwin = nullptr;
    float *dw = nullptr, *dr = nullptr, *dwinw = nullptr;
    int rc = 2;
    if (cudaMalloc(&dp, sizeof(robot_state) * n) == cudaSuccess && cudaMalloc(&dw, sizeof(float) * n) == cudaSuccess &&
        cudaMalloc(&dr, sizeof(float) * 3 * n) == cudaSuccess && cudaMalloc(&dwin, sizeof(robot_state)) == cudaSuccess &&
        cudaMalloc(&dwinw, sizeof(float)) == cudaSuccess &&
        cudaMemcpy(dp, h.data(), sizeof(robot_state) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpy(dr, r.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
        cudaMemcpyToSymbol(d_sensor_data, ranges, sizeof(float) * NUM_SENSORS, 0, cudaMemcpyHostToDevice) == cudaSuccess) {
        control_input c;
        c.velocity = v;
        c.angular_velocity = w;
        sampling_importance<<<n, 1>>>(dp, dw, dwin, dwinw, c, dr, dt, 1, 0);
        if (cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
            cudaMemcpy(h.data(), dp, sizeof(robot_state) * n, cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(weight_out, dw, sizeof(float) * n, cudaMemcpyDeviceToHost) == cudaSuccess) {
            for (int i = 0; i < n; ++i) {
                state_out[i] = h[(size_t)i].x;
                state_out[n + i] = h[(size_t)i].y;
                state_out[2 * n + i] = h[(size_t)i].theta;
            }
            rc = 0;
        }
    }
    cudaFree(dp);
    cudaFree(dw);
    cudaFree(dr);
    cudaFree(dwin);
    cudaFree(dwinw);
    return rc;
}
