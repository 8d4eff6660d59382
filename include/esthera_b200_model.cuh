/*
 * esthera_b200_model.cuh -- adding a model to the engine from one CUDA file.
 *
 * The reference's model plugin is a header its driver #includes at compile
 * time (src/partfilt/cuda/pf_generic_soa.cu:43 -> src/models/robotarm/cuda/
 * pf_model_soa.cuh:33-316: the state / control / measurement types,
 * sampling_iw, particle_set, read_trace, estimate_error).  Here a model is a
 * struct of device hooks compiled together with the engine's kernels: the
 * model's own .cu file, built into the library, ends with
 *
 *     PF_MODEL(MyModel, PF_MODEL_USER_BASE + k, my_params, "name");
 *
 * which instantiates every kernel of the step for MyModel (sampling,
 * resampling with each resampler, the single-kernel and the phased
 * pipelines, the model test entry) and registers it; pf_create, the batches
 * and pfk_model_step then run it like a built-in model (pf_model_list /
 * pf_model_name list it).  The server runs the built-in models only.
 *
 * The model struct (the reference's sampling_iw + particle_set + types):
 *
 *   static constexpr int S, K, NA, C, Z;
 *       state floats (1..PF_MAX_STATE), standard normals drawn per particle
 *       and step (>= 1), angular state variables (0..S; their posterior mean
 *       is circular; S + NA <= 28), control and measurement floats read from
 *       pf_step_input.
 *   __host__ __device__ static constexpr int angle_var(int a);
 *       the state index of the a-th angular variable.
 *   struct Consts { ... };
 *       per-step constants, in shared memory.
 *   __device__ static void prepare(Consts& c, const pf_step_input& in,
 *                                  const pfdev::ModelParams& mp, int lane);
 *       called by the 32 lanes of one warp before a sub-filter's step; the
 *       model's parameter struct is at mp.raw; each lane fills its own fields.
 *   __device__ static float step(const Consts& c, float* s, const float* n,
 *                                float* sn, float* cs);
 *       one particle: propagate s[S] in place with the normals n[K], return
 *       its FP32 log-likelihood (log weight), and sin / cos of the NA angular
 *       variables of the new state (sn[a], cs[a] of s[angle_var(a)], as
 *       __sincosf gives them: the estimate uses them for circular means).
 *   optional: template <int E, class Noise> __device__ static void
 *       step_batch(const Consts&, float (&s)[E][S], Noise noise,
 *                  float (&sn)[E][NA or 1], float (&cs)[E][NA or 1], float (&ll)[E]);
 *       E particles at once with step()'s arithmetic (noise(e, v) is
 *       particle e's v-th normal), when interleaving them pays.
 *   optional: __device__ static float step_pair(const Consts& c, float* s,
 *                                               const float* n, int h,
 *                                               float* sn, float* cs);
 *       two threads per particle (pf_config.threads_per_particle = 2): the
 *       lanes 2g + h (h = 0, 1) of a pair call it for the same particle; both
 *       must leave identical s / sn / cs and return identical log-likelihoods,
 *       exchanging partial results with __shfl_xor_sync(0xffffffff, x, 1)
 *       (every lane of the warp takes part).  Without it both lanes run step.
 *
 * The parameter struct: standard layout, at most 256 bytes, with a member
 * float init_state[S] (the state pf_set_initial_state and creation use).
 *
 * Ids: PF_MODEL_USER_BASE (64) and above; an id registered twice keeps the
 * first registration.  Random numbers, sorting, exchange, resampling and the
 * estimate are the engine's and need nothing from the model.
 */
#ifndef ESTHERA_B200_MODEL_CUH
#define ESTHERA_B200_MODEL_CUH

#include "esthera_b200.h"

#define PF_PART_K1
#define PF_PART_K2REF
#define PF_PART_K2SYS
#define PF_PART_K2VOSE
#define PF_PART_PHASED
#define PF_PART_STEPREF
#define PF_PART_STEPSYS
#define PF_PART_STEPVOSE
#include "pf_launch_impl.cuh"
#include "pf_host.cuh"

#define PF_MODEL(MDL, ID, PARAMS, NAME)         \
    template struct ::pfdev::Launch<MDL>;       \
    PF_REGISTER_MODEL(MDL, ID, PARAMS, NAME)

#endif
