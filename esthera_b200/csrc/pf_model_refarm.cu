// Kernel instantiations for the reference's 5-angle camera arm.
#include "pf_launch.cuh"
namespace pfdev {
template struct Launch<RefArm>;
}
