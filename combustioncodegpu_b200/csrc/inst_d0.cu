// Kernel instantiation: bulk precision double, species count 0 (-1 = runtime).
#include "launch.cuh"
namespace ccb {
CCB_INSTANTIATE(double, 0)
}  // namespace ccb
