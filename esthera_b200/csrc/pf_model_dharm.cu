// Kernel instantiations for the 6-joint Denavit-Hartenberg arm.
#include "pf_launch.cuh"
namespace pfdev {
template struct Launch<DhArm>;
}
