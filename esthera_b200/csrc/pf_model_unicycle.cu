// Kernel instantiations for the unicycle (range/bearing) model.
#include "pf_launch.cuh"
namespace pfdev {
template struct Launch<Unicycle>;
}
