// Kernel instantiations: the single-kernel step, Vose alias for the reference's pinhole-camera arm (lens distortion).
#define PF_PART_STEPVOSE
#include "pf_launch_impl.cuh"
namespace pfdev {
template cudaError_t Launch<CamArm>::step_vose(int, int, int, cudaStream_t, const FilterDesc*, const StepState&, InputRef, int32_t*, bool);
}  // namespace pfdev
