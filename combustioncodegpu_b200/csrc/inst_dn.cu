// Kernel instantiation: bulk precision double, species count -1 (-1 = runtime).
#include "launch.cuh"
namespace ccb {
CCB_INSTANTIATE(double, -1)
}  // namespace ccb
