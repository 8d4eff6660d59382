// Kernel instantiations: the single-kernel step, systematic for the reference's pinhole-camera arm (lens distortion).
#define PF_PART_STEPSYS
#include "pf_launch_impl.cuh"
namespace pfdev {
template cudaError_t Launch<CamArm>::step_sys(int, int, int, cudaStream_t, const FilterDesc*, const StepState&, InputRef, int32_t*, bool);
}  // namespace pfdev
