// pf_model_lingauss.cu -- a model added through esthera_b200_model.cuh, in
// one file: a linear-Gaussian constant-velocity target, whose exact posterior
// is the Kalman filter's (the engine's statistical end-to-end check).
//
// State (position p, velocity v); per step, with dt from the input (or the
// parameter): p' = p + v dt, v' = v + sigma_v n (the position advances with
// the velocity of the previous step); measurement z = p' + sigma_z e;
// log weight -(z - p')^2 / (2 sigma_z^2).  Registered as PF_MODEL_USER_BASE.
#include "esthera_b200_model.cuh"

struct pf_lingauss_params {
    float dt;
    float sigma_v;        // process noise std on the velocity
    float sigma_z;        // position measurement std
    float init_state[2];  // position, velocity
};

struct LinGauss {
    static constexpr int S = 2, K = 1, NA = 0, C = 0, Z = 1;
    __host__ __device__ static constexpr int angle_var(int) { return 0; }
    struct Consts {
        float dt, sv, iz, z;
    };
    __device__ static void prepare(Consts& c, const pf_step_input& in, const pfdev::ModelParams& mp, int lane)
    {
        if (lane != 0) return;
        const pf_lingauss_params& p = *reinterpret_cast<const pf_lingauss_params*>(mp.raw);
        c.dt = in.dt > 0.0f ? in.dt : p.dt;
        c.sv = p.sigma_v;
        c.iz = 1.0f / p.sigma_z;
        c.z = in.meas[0];
    }
    __device__ static __forceinline__ float step(const Consts& c, float* s, const float* n, float*, float*)
    {
        const float p = fmaf(s[1], c.dt, s[0]);
        s[1] = fmaf(c.sv, n[0], s[1]);
        s[0] = p;
        const float e = (c.z - p) * c.iz;
        return -0.5f * e * e;
    }
};

PF_MODEL(LinGauss, PF_MODEL_USER_BASE, pf_lingauss_params, "lingauss");
