// Kernel instantiations: the fused sample+weight+sort kernel for the unicycle (range/bearing) model.
#define PF_PART_K1
#include "pf_launch_impl.cuh"
#include "pf_host.cuh"
namespace pfdev {
template cudaError_t Launch<Unicycle>::sample_sort(int, int, int, bool, int, cudaStream_t, const FilterDesc*, const int2*, InputRef);
}  // namespace pfdev
// the model registers itself here (once for the library)
PF_REGISTER_MODEL(pfdev::Unicycle, PF_MODEL_UNICYCLE, pf_unicycle_params, "unicycle");
