// Kernel instantiations: the single-kernel step, reference multinomial for the reference's pinhole-camera arm (lens distortion).
#define PF_PART_STEPREF
#include "pf_launch_impl.cuh"
namespace pfdev {
template cudaError_t Launch<CamArm>::step_ref(int, int, int, cudaStream_t, const FilterDesc*, const StepState&, InputRef, int32_t*, bool);
}  // namespace pfdev
