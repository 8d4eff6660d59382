// Kernel instantiations: the fused sample+weight+sort kernel for the 6-joint Denavit-Hartenberg arm.
#define PF_PART_K1
#include "pf_launch_impl.cuh"
#include "pf_host.cuh"
namespace pfdev {
template cudaError_t Launch<DhArm>::sample_sort(int, int, int, bool, int, cudaStream_t, const FilterDesc*, const int2*, InputRef);
}  // namespace pfdev
// the model registers itself here (once for the library)
PF_REGISTER_MODEL(pfdev::DhArm, PF_MODEL_DHARM, pf_dharm_params, "dharm");
