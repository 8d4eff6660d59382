// Kernel instantiations: the phased kernels and dispatchers for the reference's pinhole-camera arm (lens distortion).
#define PF_PART_PHASED
#include "pf_launch_impl.cuh"
namespace pfdev {
template cudaError_t Launch<CamArm>::sample_weight(int, int, int, cudaStream_t, const FilterDesc*, const int2*, InputRef);
template cudaError_t Launch<CamArm>::block_sort(int, int, int, cudaStream_t, const FilterDesc*, const int2*);
template cudaError_t Launch<CamArm>::exchange_resample(int, int, int, int, cudaStream_t, const FilterDesc*, const int2*, InputRef, int32_t*, int);
template cudaError_t Launch<CamArm>::exchange_inplace(int, int, cudaStream_t, const FilterDesc*, const int2*);
template cudaError_t Launch<CamArm>::test_model(const ModelParams&, const pf_step_input*, int, float*, const float*, float*, cudaStream_t);
template cudaError_t Launch<CamArm>::step(int, int, int, int, cudaStream_t, const FilterDesc*, const StepState&, InputRef, int32_t*, bool);
}  // namespace pfdev
