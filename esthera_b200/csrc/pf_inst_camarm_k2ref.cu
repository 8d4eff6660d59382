// Kernel instantiations: the exchange+resample kernel, reference multinomial for the reference's pinhole-camera arm (lens distortion).
#define PF_PART_K2REF
#include "pf_launch_impl.cuh"
namespace pfdev {
template cudaError_t Launch<CamArm>::k2_ref(int, int, int, cudaStream_t, const FilterDesc*, const int2*, InputRef, int32_t*, int);
}  // namespace pfdev
